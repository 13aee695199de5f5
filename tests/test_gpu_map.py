"""vector_map on the device against the oracle's row-at-a-time restatement
of compute/map: the reference's examples, and seeded random expression
trees over special values (NaN, signed zeros, infinities, extremes), the
same value bit for bit (NaN payloads aside, which are the hardware's) or
the same first failing element and status; with exp, ln, log or power,
within 2 units in the last place."""

import math

import numpy as np
import pytest

import pg_warren_b200 as W
from oracle import vector_map as M
from pg_warren_b200 import expr as X

pytestmark = pytest.mark.gpu


def version(n):
    return W.GraphVersion(np.zeros(n + 1, np.uint64), np.zeros(0, np.uint32))


def both(e, n, ops):
    gv = version(n)
    try:
        want = M.vector_map(e, n, ops)
    except M.MapError as err:
        want = err
    try:
        got = W.vector_map(gv, e, ops)
    except W.api.WarrenError as err:
        got = err
    return got, want


def same_outcome(got, want, ulps=0):
    if isinstance(want, M.MapError):
        assert isinstance(got, W.api.WarrenError), (got, want.status, want.position)
        assert got.status == want.status
        if want.position is not None:
            assert got.detail.node == want.position
        return
    assert not isinstance(got, Exception), (got, getattr(got, "detail", None) and got.detail.node)
    if want.dtype in (np.float32, np.float64):
        # NaN payloads and signs are the hardware's (SQL sees every NaN as
        # one value): NaN where the oracle has NaN, every other bit equal.
        assert (np.isnan(got) == np.isnan(want)).all()
        got, want = np.where(np.isnan(got), 0, got), np.where(np.isnan(want), 0, want)
    if ulps == 0 or want.dtype not in (np.float64,):
        assert got.tobytes() == want.tobytes()
        return
    g, w = got.reshape(-1), want.reshape(-1)
    both_nan = np.isnan(g) & np.isnan(w)
    exact = (g == w) | both_nan
    close = np.abs(g - w) <= ulps * np.spacing(np.abs(w))
    assert (exact | close).all()


def x(i, t="f64"):
    return X.Vector(t, i)


def lit(v, t="f64"):
    return X.Literal(t, v)


def test_the_reference_examples():
    got, want = both(X.Arithmetic("/", x(0), X.NullIf(x(1), lit(0.0))), 3,
                     [np.array([1.0, 2.0, 3.0]), np.array([2.0, 0.0, 1.0])])
    same_outcome(got, want)
    cond = X.Or([X.Compare("=", x(0), lit(1.0)), X.Compare("<=", x(1), lit(50.0))])
    e = X.Case("i64", [(cond, lit(1, "i64"))], lit(0, "i64"))
    got, want = both(e, 3, [np.array([1.0, 0.0, 0.0]), np.array([99.0, 50.0, 51.0])])
    assert got.tolist() == [1, 1, 0]
    same_outcome(got, want)
    emb = np.array([[1.0, 2.0], [3.0, 4.0]])
    got = W.vector_map(version(2), X.Arithmetic("/", x(0), x(1)), [emb, np.array([2.0, 4.0])])
    assert got.reshape(-1).tolist() == [0.5, 1.0, 0.75, 1.0]
    a = np.array([1.0, 1, 1, 1, -1, 1, 1, 1, -1, 1])
    b = np.array([1.0, 1, 0, 1, 1, 1, 0, 1, 1, 1])
    e = X.Arithmetic("+", X.Call("sqrt", x(0)), X.Arithmetic("/", lit(1.0), x(1)))
    got, want = both(e, 10, [a, b])
    assert got.status == 13 and got.detail.node == 2
    same_outcome(got, want)
    with pytest.raises(W.api.NullResult):
        W.vector_map(version(1), lit(None, "i64"))
    with pytest.raises(W.api.UnknownOperand):
        W.vector_map(version(0), X.Case("f64", [(lit(False, "bool"), x(1))]), [np.ones(0)])
    with pytest.raises(W.api.OperandType):
        W.vector_map(version(0), x(0), [np.ones(0, np.int64)])
    with pytest.raises(W.api.WidthMismatch):
        W.vector_map(version(2), X.Arithmetic("+", x(0), x(1)), [np.ones((2, 2)), np.ones((2, 3))])


SPECIAL = [0.0, -0.0, 1.0, -1.0, 2.5, -2.5, 0.5, 3.0, 1e300, -1e300, 1e-300, 5e-324, math.inf,
           -math.inf, math.nan, 100.0, 7.0, 9.3e18]


def operands(rng, n):
    f = rng.choice(SPECIAL, n)
    g = rng.choice(SPECIAL, n)
    i = rng.choice([0, 1, -1, 2, 7, -7, 3, 2 ** 62, -2 ** 63, 2 ** 63 - 1, 100], n).astype(np.int64)
    b = rng.random(n) < 0.5
    r = rng.choice([0.0, -0.0, 1.5, -2.0, 0.1, 3e38, 1e-30, math.inf, math.nan], n).astype(np.float32)
    return [f, g, i, b, r]


def gen(rng, t, depth, transcendental):
    """A random expression of type `t`."""
    leaf = depth == 0 or rng.random() < 0.25
    if leaf:
        if rng.random() < 0.6:
            return {"f64": lambda: x(int(rng.integers(0, 2))), "i64": lambda: x(2, "i64"),
                    "bool": lambda: x(3, "bool"), "f32": lambda: x(4, "f32")}[t]()
        if rng.random() < 0.1:
            return lit(None, t)
        return lit({"f64": float(rng.choice(SPECIAL)), "i64": int(rng.choice([0, 1, -1, 3, 2 ** 62])),
                    "bool": bool(rng.random() < 0.5), "f32": float(np.float32(rng.choice([1.5, -0.0, 1e-30])))}[t], t)
    d = depth - 1
    sub = lambda tt=t: gen(rng, tt, d, transcendental)
    common = rng.random()
    if common < 0.08:
        return X.Case(t, [(gen(rng, "bool", d, transcendental), sub()) for _ in range(int(rng.integers(1, 3)))],
                      sub() if rng.random() < 0.7 else None)
    if common < 0.13:
        return X.Coalesce(t, [sub() for _ in range(int(rng.integers(0, 3)))])
    if common < 0.18:
        return (X.Least if rng.random() < 0.5 else X.Greatest)(t, [sub() for _ in range(int(rng.integers(0, 4)))])
    if common < 0.22:
        return X.NullIf(sub(), sub())
    if common < 0.3:
        frm = str(rng.choice(["f64", "i64", "bool", "f32"]))
        return X.Cast(t, gen(rng, frm, d, transcendental))
    if t == "bool":
        k = rng.random()
        if k < 0.4:
            tt = str(rng.choice(["f64", "i64", "bool", "f32"]))
            return X.Compare(str(rng.choice(X.COMPARISONS)), gen(rng, tt, d, transcendental),
                             gen(rng, tt, d, transcendental))
        if k < 0.55:
            return X.Not(sub())
        return (X.And if k < 0.8 else X.Or)([sub() for _ in range(int(rng.integers(0, 4)))])
    if t == "i64":
        k = rng.random()
        if k < 0.5:
            return X.Arithmetic(str(rng.choice(X.ARITHMETIC)), sub(), sub())
        if k < 0.7:
            return X.Modulo(sub(), sub())
        return (X.Abs if k < 0.85 else X.Negate)(sub())
    if t == "f32":
        k = rng.random()
        if k < 0.6:
            return X.Arithmetic(str(rng.choice(X.ARITHMETIC)), sub(), sub())
        return (X.Abs if k < 0.8 else X.Negate)(sub())
    k = rng.random()
    if k < 0.45:
        return X.Arithmetic(str(rng.choice(X.ARITHMETIC)), sub(), sub())
    if k < 0.55:
        return X.Negate(sub())
    fns = X.FUNCTIONS if transcendental else ["abs", "sqrt", "floor", "ceil", "round", "sign"]
    if transcendental and k < 0.65:
        return X.Power(sub(), sub())
    return X.Call(str(rng.choice(fns)), sub())


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("t", ["f64", "i64", "bool", "f32"])
def test_random_expressions_match_the_oracle(seed, t):
    rng = np.random.default_rng(seed * 17 + len(t))
    n = 300
    ops = operands(rng, n)
    for _ in range(25):
        e = gen(rng, t, 4, False)
        got, want = both(e, n, ops)
        same_outcome(got, want)


@pytest.mark.parametrize("name", ["exp", "ln", "log", "power"])
def test_transcendental_functions_within_two_ulps(name):
    # Each call on its own: the device's exp, log, log10 and pow against the
    # host's, within 2 units in the last place of the result.
    rng = np.random.default_rng(len(name))
    n = 4000
    a = np.concatenate([rng.uniform(-700, 700, n // 2), rng.standard_normal(n // 2) * 3])
    pos = np.abs(a) + 1e-3
    exps = np.round(rng.uniform(-20, 20, n))
    if name == "exp":
        e, ops = X.Call("exp", x(0)), [a]
    elif name == "power":
        e, ops = X.Power(x(0), x(1)), [rng.uniform(0.01, 3.0, n), exps]
    else:
        e, ops = X.Call(name, x(0)), [pos]
    got, want = both(e, n, ops)
    same_outcome(got, want, ulps=2)


def test_device_operands_and_a_wide_result():
    import torch
    rng = np.random.default_rng(3)
    n = 100_000
    a = rng.standard_normal((n, 4))
    b = rng.standard_normal(n)
    e = X.Case("f64", [(X.Compare(">", x(0), lit(0.0)), X.Arithmetic("*", x(0), x(1)))],
               X.Call("abs", x(1)))
    got = W.vector_map(version(n), e, [torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda")])
    expect = np.where(a > 0, a * b[:, None], np.abs(b)[:, None])
    assert got.tobytes() == expect.tobytes()
