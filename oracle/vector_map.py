"""Test oracle: a row-at-a-time restatement of compute/map (vector_map), the
form the reference's own tests check its columnar evaluator against
(compute/map/tests.rs:296-480).  Pure Python over small vectors; host libm
(math.exp, math.log, math.log10, math.pow) for the transcendental calls.

Semantics followed: map/eval.rs (lazy CASE / COALESCE / AND / OR, NULLIF,
LEAST / GREATEST skipping NULL, the first of equal values kept),
map/arithmetic.rs (float and bigint operators, functions, power),
compute/cast.rs (casts) and map/mod.rs:96-160 (the first failing element in
row-major order decides the error; NULL stores NaN in float results and is
an error in bigint and boolean ones).  Statuses are the C ABI's.
"""

from __future__ import annotations

import math

import numpy as np

from pg_warren_b200 import expr as X

BIGINT, OVERFLOW, UNDERFLOW, DIV0 = 10, 11, 12, 13
SQRT_NEG, LOG_ZERO, LOG_NEG, ZERO_NEG_POW, COMPLEX_POW = 14, 15, 16, 17, 18
ID_SPACE, WIDTH, UNKNOWN_OPERAND, OPERAND_TYPE, NULL_RESULT = 4, 5, 70, 71, 72
I64_MIN, I64_MAX = -(2 ** 63), 2 ** 63 - 1

_NP = {"f32": np.float32, "f64": np.float64, "i64": np.int64, "bool": np.bool_}


class MapError(Exception):
    def __init__(self, status, position=None):
        super().__init__(f"status {status} at {position}")
        self.status = status
        self.position = position


class _Fail(Exception):
    def __init__(self, status):
        self.status = status


def _isnan(x):
    return x != x


def _isinf(x):
    return not _isnan(x) and abs(float(x)) == math.inf


def sql_cmp(t, a, b):
    """SQL order: NaN above every number and equal to itself; -0 = 0."""
    if t in ("f32", "f64"):
        an, bn = bool(_isnan(a)), bool(_isnan(b))
        if an or bn:
            return int(an) - int(bn)
    return int(bool(a > b)) - int(bool(a < b))


def float_op(t, op, a, b):
    """arithmetic.rs:49-79 in the type's precision."""
    F = _NP[t]
    a, b = F(a), F(b)
    if op == 3 and b == 0 and not _isnan(a):
        raise _Fail(DIV0)
    with np.errstate(all="ignore"):
        r = [a + b, a - b, a * b, a / b][op]
    finite = not _isinf(a) if op == 3 else (not _isinf(a) and not _isinf(b))
    if _isinf(r) and finite:
        raise _Fail(OVERFLOW)
    under = (a != 0 and b != 0) if op == 2 else ((a != 0 and not _isinf(b)) if op == 3 else False)
    if r == 0 and under:
        raise _Fail(UNDERFLOW)
    return r


def int_op(op, a, b):
    """arithmetic.rs:83-97: checked; division truncates."""
    if op == 3:
        if b == 0:
            raise _Fail(DIV0)
        q = abs(a) // abs(b)
        r = q if (a >= 0) == (b >= 0) else -q
    else:
        r = [a + b, a - b, a * b][op]
    if not I64_MIN <= r <= I64_MAX:
        raise _Fail(BIGINT)
    return r


def _checked(r, base):
    if _isinf(r):
        raise _Fail(OVERFLOW)
    if r == 0.0 and base != 0.0:
        raise _Fail(UNDERFLOW)
    return r


def call(fn, a):
    """arithmetic.rs:116-169 (call, exp)."""
    name = X.FUNCTIONS[fn]
    if name == "abs":
        return abs(a)
    if name == "floor":
        return float(np.floor(a))
    if name == "ceil":
        return float(np.ceil(a))
    if name == "round":
        return float(np.rint(a))
    if name == "sign":
        return 1.0 if a > 0 else (-1.0 if a < 0 else 0.0)
    if name == "exp":
        if _isnan(a):
            return a
        if _isinf(a):
            return a if a > 0 else 0.0
        try:
            r = math.exp(a)
        except OverflowError:
            r = math.inf
        return _checked(r, a)
    if name == "sqrt":
        if a < 0:
            raise _Fail(SQRT_NEG)
        return math.sqrt(a) if not _isnan(a) else a
    if a == 0:
        raise _Fail(LOG_ZERO)
    if a < 0:
        raise _Fail(LOG_NEG)
    if _isnan(a):
        return a
    return math.log(a) if name == "ln" else math.log10(a)


def power(a, b):
    """arithmetic.rs:171-218 (power)."""
    if _isnan(a):
        return math.nan if (_isnan(b) or b != 0) else 1.0
    if _isnan(b):
        return math.nan if a != 1.0 else 1.0
    if a == 0 and b < 0:
        raise _Fail(ZERO_NEG_POW)
    if a < 0 and not _isinf(b) and math.floor(b) != b:
        raise _Fail(COMPLEX_POW)
    if _isinf(b):
        mag = abs(a)
        if mag == 1.0:
            return 1.0
        return math.inf if (b > 0) == (mag > 1.0) else 0.0
    if _isinf(a):
        if b == 0:
            return 1.0
        if a > 0:
            return a if b > 0 else 0.0
        half = b / 2.0
        odd = math.floor(half) != half
        if b > 0:
            return a if odd else -a
        return -0.0 if odd else 0.0
    try:
        r = math.pow(a, b)
    except OverflowError:
        r = math.inf
    return _checked(r, a)


def cast(frm, to, v):
    """compute/cast.rs."""
    if to == "f64":
        return float(v) if frm != "bool" else (1.0 if v else 0.0)
    if to == "f32":
        if frm == "i64":
            return np.float32(np.int64(v))
        if frm == "bool":
            return np.float32(1.0 if v else 0.0)
        if frm == "f32":
            return np.float32(v)
        with np.errstate(all="ignore"):
            n = np.float32(v)
        if _isinf(n) and not _isinf(v):
            raise _Fail(OVERFLOW)
        if n == 0 and v != 0:
            raise _Fail(UNDERFLOW)
        return n
    if to == "i64":
        if frm == "i64":
            return int(v)
        if frm == "bool":
            return int(bool(v))
        r = float(np.rint(float(v)))
        if not (-9223372036854775808.0 <= r < 9223372036854775808.0):
            raise _Fail(BIGINT)
        return int(r)
    if frm in ("f32", "f64"):
        return bool(float(v) != 0.0)  # NaN is true
    return bool(v)


class _Row:
    def __init__(self, operands, p, row):
        self.operands, self.p, self.row = operands, p, row

    def load(self, e):
        o = self.operands[e.index]
        if o.ndim == 1:
            return o[self.row]
        return o[self.row, 0] if o.shape[1] == 1 else o.reshape(-1)[self.p]


def ev(e, r):
    """The value of `e` at one element (None: NULL); raises _Fail."""
    t, k = e.type, e.kind
    if k == X.LITERAL:
        if e.value is None:
            return None
        return _NP[t](e.value) if t == "f32" else (bool(e.value) if t == "bool" else
                                                   (int(e.value) if t == "i64" else float(e.value)))
    if k == X.VECTOR:
        v = r.load(e)
        return np.float32(v) if t == "f32" else (bool(v) if t == "bool" else
                                                 (int(v) if t == "i64" else float(v)))
    if k == X.CAST:
        v = ev(e.children[0], r)
        return None if v is None else cast(e.children[0].type, t, v)
    if k == X.CASE:
        for cond, val in e.when:
            c = ev(cond, r)
            if c is not None and c:
                return ev(val, r)
        return ev(e.otherwise, r) if e.otherwise is not None else None
    if k == X.NULLIF:
        a, b = ev(e.children[0], r), ev(e.children[1], r)
        if a is not None and b is not None and sql_cmp(t, a, b) == 0:
            return None
        return a
    if k == X.COALESCE:
        for c in e.children:
            v = ev(c, r)
            if v is not None:
                return v
        return None
    if k in (X.LEAST, X.GREATEST):
        want = 1 if k == X.GREATEST else -1
        best = None
        for c in e.children:
            v = ev(c, r)
            if v is not None and (best is None or sql_cmp(t, v, best) == want):
                best = v
        return best
    if k in (X.NEGATE, X.ABS, X.CALL, X.NOT):
        a = ev(e.children[0], r)
        if a is None:
            return None
        if k == X.NOT:
            return not a
        if k == X.CALL:
            return call(e.op, a)
        if t == "i64":
            if a == I64_MIN:
                raise _Fail(BIGINT)
            return -a if k == X.NEGATE else abs(a)
        return -a if k == X.NEGATE else abs(a)
    if k in (X.ARITH, X.MODULO, X.POWER, X.COMPARE):
        a, b = ev(e.children[0], r), ev(e.children[1], r)
        if a is None or b is None:
            return None
        if k == X.COMPARE:
            c = sql_cmp(e.children[0].type, a, b)
            return [c == 0, c != 0, c < 0, c <= 0, c > 0, c >= 0][e.op]
        if k == X.POWER:
            return power(a, b)
        if k == X.MODULO:
            if b == 0:
                raise _Fail(DIV0)
            if b == -1:
                return 0
            m = abs(a) % abs(b)
            return m if a >= 0 else -m
        if t == "i64":
            return int_op(e.op, a, b)
        v = float_op(t, e.op, a, b)
        return np.float32(v) if t == "f32" else float(v)
    if k in (X.AND, X.OR):
        stop = k == X.OR
        null = False
        for c in e.children:
            v = ev(c, r)
            if v is None:
                null = True
            elif bool(v) == stop:
                return stop
        return None if null else (not stop)
    raise ValueError(f"unknown node {e!r}")


def _check_operands(e, operands):
    """Every operand reference, evaluated or not, in evaluation order."""
    if e.kind == X.VECTOR:
        if not 0 <= e.index < len(operands):
            raise MapError(UNKNOWN_OPERAND)
        want = {"f32": np.float32, "f64": np.float64, "i64": np.int64}.get(e.type)
        dt = operands[e.index].dtype
        ok = dt == np.bool_ or dt == np.uint8 if e.type == "bool" else dt == want
        if not ok:
            raise MapError(OPERAND_TYPE)
    for c in e.children:
        _check_operands(c, operands)


def vector_map(expr, id_space, operands=()):
    """map/mod.rs:49-78: the result array, or MapError(status, position)."""
    operands = [np.asarray(o) for o in operands]
    width = max([1] + [1 if o.ndim == 1 else o.shape[1] for o in operands])
    for o in operands:
        if len(o) != id_space:
            raise MapError(ID_SPACE)
        if (1 if o.ndim == 1 else o.shape[1]) not in (1, width):
            raise MapError(WIDTH)
    _check_operands(expr, operands)
    out = np.zeros(id_space * width, _NP[expr.type])
    for p in range(id_space * width):
        try:
            v = ev(expr, _Row(operands, p, p // width))
        except _Fail as f:
            raise MapError(f.status, p)
        if v is None:
            if expr.type in ("f32", "f64"):
                v = math.nan
            else:
                raise MapError(NULL_RESULT, p)
        out[p] = v
    return out.reshape(id_space, width) if width > 1 else out
