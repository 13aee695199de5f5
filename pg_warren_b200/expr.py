"""The vector_map expression IR (compute/map/expr.rs): typed SQL expressions
over operand vectors, built by the adapter from Postgres's analysed tree.

Every node carries its result type, one of "f32" (real), "f64" (double
precision), "i64" (bigint) and "bool"; operators take operands of one type
(an implicit cast is an explicit `Cast`).  `serialize` flattens a tree into
the C ABI's node and child arrays (wc_map_node, include/warren_cuda.h).
"""

from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np

TYPES = {"f32": 0, "f64": 1, "i64": 2, "bool": 3}
ARITHMETIC = ["+", "-", "*", "/"]                       # expr.rs:84-95
COMPARISONS = ["=", "<>", "<", "<=", ">", ">="]         # expr.rs:98-112
FUNCTIONS = ["abs", "sqrt", "exp", "ln", "log", "floor", "ceil", "round", "sign"]  # expr.rs:176-197

(LITERAL, VECTOR, CAST, CASE, NULLIF, COALESCE, LEAST, GREATEST, NEGATE, ARITH, MODULO, ABS,
 CALL, POWER, COMPARE, NOT, AND, OR) = range(18)


class Expr:
    """A node: `type`, its kind and its children in the IR's order."""

    kind = -1

    def __init__(self, type: str, *children: "Expr"):
        if type not in TYPES:
            raise ValueError(f"unknown type {type!r}")
        self.type = type
        self.children: Tuple[Expr, ...] = children

    def __repr__(self):
        return f"{type(self).__name__}({self.type}, {', '.join(map(repr, self.children))})"


class Literal(Expr):
    """A constant; value None is a typed NULL."""
    kind = LITERAL

    def __init__(self, type: str, value=None):
        super().__init__(type)
        self.value = value


class Vector(Expr):
    """Operand vector `index` at the current element."""
    kind = VECTOR

    def __init__(self, type: str, index: int):
        super().__init__(type)
        self.index = index


class Cast(Expr):
    kind = CAST

    def __init__(self, type: str, arg: Expr):
        super().__init__(type, arg)


class Case(Expr):
    """CASE WHEN c1 THEN v1 ... ELSE otherwise END (no ELSE: NULL)."""
    kind = CASE

    def __init__(self, type: str, when: Sequence[Tuple[Expr, Expr]],
                 otherwise: Optional[Expr] = None):
        flat = [x for pair in when for x in pair] + ([otherwise] if otherwise is not None else [])
        super().__init__(type, *flat)
        self.when = list(when)
        self.otherwise = otherwise


class NullIf(Expr):
    kind = NULLIF

    def __init__(self, a: Expr, b: Expr):
        super().__init__(a.type, a, b)


class Coalesce(Expr):
    kind = COALESCE

    def __init__(self, type: str, args: Sequence[Expr]):
        super().__init__(type, *args)


class Least(Expr):
    kind = LEAST

    def __init__(self, type: str, args: Sequence[Expr]):
        super().__init__(type, *args)


class Greatest(Expr):
    kind = GREATEST

    def __init__(self, type: str, args: Sequence[Expr]):
        super().__init__(type, *args)


class Negate(Expr):
    kind = NEGATE

    def __init__(self, a: Expr):
        super().__init__(a.type, a)


class Arithmetic(Expr):
    kind = ARITH

    def __init__(self, op: str, a: Expr, b: Expr):
        super().__init__(a.type, a, b)
        self.op = ARITHMETIC.index(op)


class Modulo(Expr):
    kind = MODULO

    def __init__(self, a: Expr, b: Expr):
        super().__init__("i64", a, b)


class Abs(Expr):
    kind = ABS

    def __init__(self, a: Expr):
        super().__init__(a.type, a)


class Call(Expr):
    kind = CALL

    def __init__(self, function: str, a: Expr):
        super().__init__("f64", a)
        self.op = FUNCTIONS.index(function)


class Power(Expr):
    kind = POWER

    def __init__(self, a: Expr, b: Expr):
        super().__init__("f64", a, b)


class Compare(Expr):
    kind = COMPARE

    def __init__(self, op: str, a: Expr, b: Expr):
        super().__init__("bool", a, b)
        self.op = COMPARISONS.index(op)


class Not(Expr):
    kind = NOT

    def __init__(self, a: Expr):
        super().__init__("bool", a)


class And(Expr):
    kind = AND

    def __init__(self, args: Sequence[Expr]):
        super().__init__("bool", *args)


class Or(Expr):
    kind = OR

    def __init__(self, args: Sequence[Expr]):
        super().__init__("bool", *args)


NODE_DTYPE = np.dtype([("kind", "<i4"), ("type", "<i4"), ("op", "<i4"), ("has_else", "<i4"),
                       ("first", "<u4"), ("count", "<u4"), ("is_null", "<i4"),
                       ("reserved", "<i4"), ("i", "<i8"), ("f", "<f8")])


def serialize(root: Expr):
    """(nodes as a wc_map_node array, children u32, root index)."""
    nodes, children = [], []

    def visit(e: Expr) -> int:
        kids = [visit(c) for c in e.children]
        rec = np.zeros((), NODE_DTYPE)
        rec["kind"], rec["type"] = e.kind, TYPES[e.type]
        rec["op"] = getattr(e, "op", 0)
        rec["has_else"] = int(isinstance(e, Case) and e.otherwise is not None)
        rec["first"], rec["count"] = len(children), len(kids)
        children.extend(kids)
        if isinstance(e, Literal):
            rec["is_null"] = int(e.value is None)
            if e.value is not None:
                if e.type in ("f32", "f64"):
                    rec["f"] = float(e.value)
                else:
                    rec["i"] = int(e.value)
        if isinstance(e, Vector):
            rec["i"] = e.index
        nodes.append(rec)
        return len(nodes) - 1

    root_index = visit(root)
    return (np.array(nodes, NODE_DTYPE), np.array(children, np.uint32), root_index)
