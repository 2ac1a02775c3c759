"""Expression trees on the host: the caller-side data the device path consumes.

Mirrors the constructors of the reference's `expr` module
(`my-version/src/expr.rs`: `node`, `constant`, `input`) for the operators the
device path handles. A tree is serialised as two pre-order arrays, `op[i]`
(int32) and `val[i]` (f64); an operator's arity follows from its code. Codes
0..42 are numerically the device opcodes (`my-version/src/cuda/eval.cu:34-83`,
`my-version/src/gpu.rs:29-73`); 64..66 are the inverse hyperbolics that the
compiler lowers before emission (`my-version/src/gpu.rs:320-345`).
"""
from __future__ import annotations

import numpy as np

CONST, VAR, ADD, SUB, MUL, DIV = 0, 1, 2, 3, 4, 5
SIN, COS, TAN, EXP, LOG, SQRT, ABS, TANH, SIG = 6, 7, 8, 9, 10, 11, 12, 13, 14
SQUARE, CUBE, NEG, GAUSS, STEP, POW, SINH, COSH = 15, 16, 17, 18, 19, 20, 21, 22
FLOOR, CEIL, ROUND, MOD, ATAN2, ERF, ERFC, MIN, MAX, IF = 23, 24, 25, 26, 27, 28, 29, 30, 31, 32
SIGN, EQUAL, LESS, LESS_OR_EQUAL, GREATER, GREATER_OR_EQUAL = 33, 34, 35, 36, 37, 38
AND, OR, XOR, NOT = 39, 40, 41, 42
ASINH, ACOSH, ATANH = 64, 65, 66
HALT = 255

NAMES = {
    CONST: "const", VAR: "var", ADD: "add", SUB: "sub", MUL: "mul", DIV: "div",
    SIN: "sin", COS: "cos", TAN: "tan", EXP: "exp", LOG: "ln", SQRT: "sqrt",
    ABS: "abs", TANH: "tanh", SIG: "logistic", SQUARE: "square", CUBE: "cube",
    NEG: "neg", GAUSS: "gauss", STEP: "step", POW: "pow", SINH: "sinh",
    COSH: "cosh", FLOOR: "floor", CEIL: "ceil", ROUND: "round", MOD: "mod",
    ATAN2: "atan2", ERF: "erf", ERFC: "erfc", MIN: "min", MAX: "max", IF: "if",
    SIGN: "sign", EQUAL: "equal", LESS: "less", LESS_OR_EQUAL: "less_or_equal",
    GREATER: "greater", GREATER_OR_EQUAL: "greater_or_equal", AND: "and",
    OR: "or", XOR: "xor", NOT: "not", ASINH: "asinh", ACOSH: "acosh",
    ATANH: "atanh",
}

BINARY = {ADD, SUB, MUL, DIV, POW, MOD, ATAN2, MIN, MAX, EQUAL, LESS,
          LESS_OR_EQUAL, GREATER, GREATER_OR_EQUAL, AND, OR, XOR}


def arity(op: int) -> int:
    if op in (CONST, VAR):
        return 0
    if op in BINARY:
        return 2
    if op == IF:
        return 3
    return 1


class Node:
    """One tree node: an operator, its value (constant value or input index)
    and its children."""

    __slots__ = ("op", "val", "kids")

    def __init__(self, op: int, val: float = 0.0, kids=None):
        self.op = int(op)
        self.val = float(val)
        self.kids = list(kids or [])
        if len(self.kids) != arity(self.op):
            raise ValueError(f"{NAMES.get(self.op, op)} takes {arity(self.op)} operands, "
                             f"got {len(self.kids)}")

    def clone(self) -> "Node":
        return Node(self.op, self.val, [k.clone() for k in self.kids])

    def prefix(self):
        """Pre-order `(op, val)` arrays (int32, f64)."""
        ops, vals = [], []

        def walk(n):
            ops.append(n.op)
            vals.append(n.val)
            for k in n.kids:
                walk(k)
        walk(self)
        return np.asarray(ops, dtype=np.int32), np.asarray(vals, dtype=np.float64)

    def set_prefix_values(self, vals) -> None:
        """Write pre-order values back (the fitted constants)."""
        it = iter(np.asarray(vals, dtype=np.float64).tolist())

        def walk(n):
            n.val = next(it)
            for k in n.kids:
                walk(k)
        walk(self)

    def constants(self):
        out = []

        def walk(n):
            if n.op == CONST:
                out.append(n.val)
            for k in n.kids:
                walk(k)
        walk(self)
        return out

    def set_constants(self, values) -> None:
        it = iter(list(values))

        def walk(n):
            if n.op == CONST:
                n.val = float(next(it))
            for k in n.kids:
                walk(k)
        walk(self)

    def size(self) -> int:
        return 1 + sum(k.size() for k in self.kids)

    def __repr__(self) -> str:
        if self.op == CONST:
            return repr(self.val)
        if self.op == VAR:
            return f"x{int(self.val)}"
        return f"{NAMES.get(self.op, self.op)}(" + ", ".join(map(repr, self.kids)) + ")"


def node(op: int, kids) -> Node:
    return Node(op, 0.0, kids)


def constant(v: float) -> Node:
    return Node(CONST, v)


def input(i: int) -> Node:  # noqa: A001 - mirrors expr::input
    return Node(VAR, float(i))


def from_prefix(ops, vals) -> Node:
    ops = list(np.asarray(ops).tolist())
    vals = list(np.asarray(vals, dtype=np.float64).tolist())
    pos = 0

    def rec():
        nonlocal pos
        op, v = ops[pos], vals[pos]
        pos += 1
        kids = [rec() for _ in range(arity(op))]
        return Node(op, v, kids)
    t = rec()
    if pos != len(ops):
        raise ValueError("trailing nodes in prefix arrays")
    return t


def from_postfix(words) -> Node:
    """The tree of one postfix program (the words `gpu::emit` writes,
    my-version/src/gpu.rs:320-438, and the device's variation engine builds):
    `[CONST, f32 bits]`, `[VAR, index]`, operator words, up to HALT. A
    constant's value is its f32 word widened to f64. Raises ValueError for a
    program that is not one well-formed expression."""
    w = np.asarray(words, dtype=np.uint32).reshape(-1)
    stack = []
    i = 0
    while i < len(w):
        op = int(w[i])
        i += 1
        if op == HALT:
            break
        if op in (CONST, VAR):
            if i >= len(w):
                raise ValueError("truncated operand")
            a = w[i:i + 1]
            i += 1
            stack.append(Node(CONST, float(a.view(np.float32)[0])) if op == CONST
                         else Node(VAR, float(int(a[0]))))
            continue
        k = arity(op)
        if op not in NAMES or len(stack) < k:
            raise ValueError(f"bad operator word {op}")
        kids = stack[len(stack) - k:]
        del stack[len(stack) - k:]
        stack.append(Node(op, 0.0, kids))
    else:
        raise ValueError("no HALT")
    if len(stack) != 1:
        raise ValueError("program leaves %d values" % len(stack))
    return stack[0]
