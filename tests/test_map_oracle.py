"""The vector_map oracle against the reference's known answers
(compute/map/tests.rs:56-272, compute/cast.rs:58-98,
map/arithmetic.rs:222-341), and the IR's serialisation."""

import math

import numpy as np
import pytest

from oracle import vector_map as M
from pg_warren_b200 import expr as X


def x(i, t="f64"):
    return X.Vector(t, i)


def lit(v, t="f64"):
    return X.Literal(t, v)


def div(a, b):
    return X.Arithmetic("/", a, b)


def err(fn):
    with pytest.raises(M.MapError) as e:
        fn()
    return e.value.status, e.value.position


def test_nullif_guards_a_division_and_null_stores_nan():
    found = M.vector_map(div(x(0), X.NullIf(x(1), lit(0.0))), 3,
                         [np.array([1.0, 2.0, 3.0]), np.array([2.0, 0.0, 1.0])])
    assert found[0] == 0.5 and math.isnan(found[1]) and found[2] == 3.0


def test_case_with_or_yields_an_integer_vector():
    cond = X.Or([X.Compare("=", x(0), lit(1.0)), X.Compare("<=", x(1), lit(50.0))])
    e = X.Case("i64", [(cond, lit(1, "i64"))], lit(0, "i64"))
    found = M.vector_map(e, 3, [np.array([1.0, 0.0, 0.0]), np.array([99.0, 50.0, 51.0])])
    assert found.tolist() == [1, 1, 0]


def test_broadcast_and_width_checks():
    emb = np.array([[1.0, 2.0], [3.0, 4.0]])
    nbr = np.array([[10.0, 20.0], [30.0, 40.0]])
    smooth = X.Arithmetic("+", X.Arithmetic("*", lit(0.5), x(0)), X.Arithmetic("*", lit(0.25), x(1)))
    assert M.vector_map(smooth, 2, [emb, nbr]).reshape(-1).tolist() == [3.0, 6.0, 9.0, 12.0]
    assert M.vector_map(div(x(0), x(1)), 2, [emb, np.array([2.0, 4.0])]).reshape(-1).tolist() == \
        [0.5, 1.0, 0.75, 1.0]
    assert err(lambda: M.vector_map(X.Arithmetic("+", x(0), x(1)), 2,
                                    [np.ones((2, 2)), np.ones((2, 3))]))[0] == M.WIDTH
    assert err(lambda: M.vector_map(x(0), 4, [np.ones(3)]))[0] == M.ID_SPACE


def test_operand_references_are_checked_even_unevaluated():
    unused = X.Case("f64", [(lit(False, "bool"), x(1))])
    assert err(lambda: M.vector_map(unused, 0, [np.ones(0)]))[0] == M.UNKNOWN_OPERAND
    assert err(lambda: M.vector_map(x(0), 0, [np.ones(0, np.int64)]))[0] == M.OPERAND_TYPE


def test_guarded_branches_are_not_evaluated():
    zero = np.array([0.0, 2.0])
    inv = lambda: div(lit(1.0), x(0))
    case = X.Case("f64", [(X.Compare("=", x(0), lit(0.0)), lit(0.0))], inv())
    assert M.vector_map(case, 2, [zero]).tolist() == [0.0, 0.5]
    when = X.Case("f64", [(X.Compare("<>", x(0), lit(0.0)), inv())], lit(-1.0))
    assert M.vector_map(when, 2, [zero]).tolist() == [-1.0, 0.5]
    conj = X.And([X.Compare("<>", x(0), lit(0.0)), X.Compare(">", inv(), lit(0.0))])
    assert M.vector_map(conj, 2, [zero]).tolist() == [False, True]
    assert M.vector_map(X.Coalesce("f64", [x(0), inv()]), 2, [zero]).tolist() == [0.0, 2.0]
    assert err(lambda: M.vector_map(X.Least("f64", [x(0), inv()]), 2, [zero]))[0] == M.DIV0


def test_the_first_failing_element_decides_the_error():
    a = np.array([1.0, 1, 1, 1, -1, 1, 1, 1, -1, 1])
    b = np.array([1.0, 1, 0, 1, 1, 1, 0, 1, 1, 1])
    e = X.Arithmetic("+", X.Call("sqrt", x(0)), div(lit(1.0), x(1)))
    assert err(lambda: M.vector_map(e, 10, [a, b])) == (M.DIV0, 2)
    assert err(lambda: M.vector_map(e, 10, [a, np.ones(10)])) == (M.SQRT_NEG, 4)


def test_null_results():
    assert err(lambda: M.vector_map(lit(None, "i64"), 1))[0] == M.NULL_RESULT
    assert err(lambda: M.vector_map(lit(None, "bool"), 1))[0] == M.NULL_RESULT
    assert math.isnan(M.vector_map(lit(None, "f32"), 1)[0])
    assert M.vector_map(lit(True, "bool"), 3).tolist() == [True] * 3


def test_bigint_and_real_operations():
    a, b = np.array([7, -7, -2 ** 63], np.int64), np.array([2, 2, -1], np.int64)
    i = lambda k: x(k, "i64")
    assert M.vector_map(X.Modulo(i(0), i(1)), 3, [a, b]).tolist() == [1, -1, 0]
    assert err(lambda: M.vector_map(X.Arithmetic("/", i(0), i(1)), 3, [a, b]))[0] == M.BIGINT
    assert err(lambda: M.vector_map(X.Abs(i(0)), 3, [a, b]))[0] == M.BIGINT
    assert M.vector_map(X.Negate(i(1)), 3, [a, b]).tolist() == [-2, -2, 1]
    real = np.array([1.5, -2.0, 0.1], np.float32)
    r = x(0, "f32")
    assert M.vector_map(X.Abs(r), 3, [real]).tolist() == np.array([1.5, 2.0, 0.1], np.float32).tolist()
    assert M.vector_map(X.Arithmetic("+", r, r), 3, [real]).tolist() == \
        np.array([3.0, -4.0, 0.2], np.float32).tolist()
    widened = X.Arithmetic("+", X.Cast("f64", r), lit(0.0))
    assert M.vector_map(widened, 3, [real])[2] == 0.10000000149011612


def test_three_valued_logic_least_and_greatest():
    t, f, n = lit(True, "bool"), lit(False, "bool"), lit(None, "bool")

    def ev(e):
        c = X.Case("i64", [(e, lit(1, "i64")), (X.Not(e), lit(0, "i64"))], lit(2, "i64"))
        return int(M.vector_map(c, 1)[0])
    assert [ev(X.And([n, f])), ev(X.And([n, t])), ev(X.And([t, t]))] == [0, 2, 1]
    assert [ev(X.Or([n, t])), ev(X.Or([n, f])), ev(X.Or([f, f]))] == [1, 2, 0]
    assert ev(X.Not(n)) == 2 and ev(X.And([])) == 1 and ev(X.Or([])) == 0
    v = lambda e: M.vector_map(e, 1)[0]
    assert v(X.Least("f64", [lit(math.nan), lit(None), lit(1.0)])) == 1.0
    assert math.isnan(v(X.Greatest("f64", [lit(1.0), lit(math.nan)])))
    assert math.copysign(1, v(X.Least("f64", [lit(-0.0), lit(0.0)]))) < 0
    assert math.isnan(v(X.Greatest("f64", [lit(None), lit(None)])))
    assert math.isnan(v(X.Coalesce("f64", [])))


def test_casts_and_functions():
    c = lambda v, frm, to: M.vector_map(X.Cast(to, lit(v, frm)), 1)[0]
    assert c(2.5, "f64", "i64") == 2 and c(-2.5, "f64", "i64") == -2 and c(3.5, "f32", "i64") == 4
    assert err(lambda: c(9.3e18, "f64", "i64"))[0] == M.BIGINT
    assert err(lambda: c(math.nan, "f64", "i64"))[0] == M.BIGINT
    assert err(lambda: c(1e39, "f64", "f32"))[0] == M.OVERFLOW
    assert err(lambda: c(1e-50, "f64", "f32"))[0] == M.UNDERFLOW
    assert c(math.nan, "f64", "bool") and not c(-0.0, "f32", "bool")
    f = lambda name, v: M.vector_map(X.Call(name, lit(v)), 1)[0]
    assert f("round", 2.5) == 2.0 and f("round", 3.5) == 4.0 and f("sign", math.nan) == 0.0
    assert err(lambda: f("ln", 0.0))[0] == M.LOG_ZERO
    assert err(lambda: f("log", -1.0))[0] == M.LOG_NEG
    assert err(lambda: f("exp", 1000.0))[0] == M.OVERFLOW
    assert err(lambda: f("exp", -1000.0))[0] == M.UNDERFLOW
    p = lambda a, b: M.vector_map(X.Power(lit(a), lit(b)), 1)[0]
    assert err(lambda: p(0.0, -1.0))[0] == M.ZERO_NEG_POW
    assert err(lambda: p(-8.0, 1 / 3))[0] == M.COMPLEX_POW
    assert p(-math.inf, 3.0) == -math.inf and p(math.nan, 0.0) == 1.0 and p(1.0, math.nan) == 1.0


def test_serialisation():
    e = X.Case("f64", [(X.Compare("<", x(0), lit(1.0)), x(0))], lit(2.0))
    nodes, children, root = X.serialize(e)
    assert len(nodes) == 6 and root == 5
    assert nodes[root]["kind"] == X.CASE and nodes[root]["has_else"] == 1
    assert nodes[root]["count"] == 3
    kids = children[nodes[root]["first"]:nodes[root]["first"] + 3]
    assert [nodes[k]["kind"] for k in kids] == [X.COMPARE, X.VECTOR, X.LITERAL]


def test_the_oracle_evaluates_random_trees():
    # The device tests' generator, on the host: the oracle either gives a
    # value of the expression's type or a MapError, never anything else.
    from test_gpu_map import gen, operands
    for seed in range(6):
        rng = np.random.default_rng(seed)
        ops = operands(rng, 60)
        for t in ("f64", "i64", "bool", "f32"):
            for _ in range(40):
                e = gen(rng, t, 4, seed % 2 == 0)
                try:
                    out = M.vector_map(e, 60, ops)
                except M.MapError:
                    continue
                assert out.dtype == {"f64": np.float64, "i64": np.int64, "bool": np.bool_,
                                     "f32": np.float32}[t]
