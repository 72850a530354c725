"""Symbolic AIRs: the AirBuilder interface of the reference (p3-air 0.5.0's
AirBuilder / ExtensionBuilder / PermutationAirBuilder / PeriodicAirBuilder,
re-exported by p3-miden-lifted-air/src/lib.rs:28-37), recording an
expression DAG the way SymbolicAirBuilder does, so that an AIR written
against it can be handed to the library (p3g_air_create) and proved with a
constraint kernel generated from it.

An AIR is a function ``eval(builder)`` that reads the trace window and emits
constraints, as LiftedAir::eval does (p3-miden-lifted-air/src/air.rs:208)::

    def eval(b):
        local, nxt = b.main()
        b.when_first_row().assert_eq(local[0], b.public_values()[0])
        b.when_transition().assert_eq(nxt[0], local[0] * local[0])

    desc = build_air(eval, width=1, num_public_values=1)

Values are expressions over the Goldilocks field; integers are reduced mod p.
Aux columns, challenges and aux values are extension-field values; a
constraint that involves them is asserted with ``assert_zero_ext`` /
``assert_eq_ext`` (the emission order, base or extension, is what the
reference's ConstraintLayout records).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

P = 0xFFFFFFFF00000001

# node kinds (include/p3g.h, enum p3g_sym_op)
CONST, MAIN, AUX, PUBLIC, RANDOMNESS, AUX_VALUE, PERIODIC = 0, 1, 2, 3, 4, 5, 6
IS_FIRST_ROW, IS_LAST_ROW, IS_TRANSITION, ADD, SUB, MUL, NEG = 7, 8, 9, 10, 11, 12, 13

NODE_DTYPE = np.dtype([("op", "<u4"), ("a", "<u4"), ("b", "<u4"), ("pad", "<u4"), ("value", "<u8")])


class Expr:
    __slots__ = ("b", "i")

    def __init__(self, builder: "SymbolicAirBuilder", index: int):
        self.b = builder
        self.i = index

    def _lift(self, o) -> "Expr":
        if isinstance(o, Expr):
            return o
        return self.b.const(int(o))

    def __add__(self, o):
        return self.b._node(ADD, self.i, self._lift(o).i)

    def __radd__(self, o):
        return self._lift(o) + self

    def __sub__(self, o):
        return self.b._node(SUB, self.i, self._lift(o).i)

    def __rsub__(self, o):
        return self._lift(o) - self

    def __mul__(self, o):
        return self.b._node(MUL, self.i, self._lift(o).i)

    def __rmul__(self, o):
        return self._lift(o) * self

    def __neg__(self):
        return self.b._node(NEG, self.i, 0)

    def __pow__(self, e: int):
        assert isinstance(e, int) and e >= 1
        r, base = None, self
        while e:
            if e & 1:
                r = base if r is None else r * base
            e >>= 1
            if e:
                base = base * base
        return r

    def exp_power_of_2(self, k: int):
        r = self
        for _ in range(k):
            r = r * r
        return r


class _Filtered:
    """FilteredAirBuilder: every assertion is multiplied by the condition."""

    def __init__(self, b: "SymbolicAirBuilder", cond: Expr):
        self.b, self.cond = b, cond

    def assert_zero(self, x):
        self.b.assert_zero(self.cond * x)

    def assert_eq(self, x, y):
        self.assert_zero(self.b._lift(x) - y)

    def assert_one(self, x):
        self.assert_zero(self.b._lift(x) - 1)

    def assert_bool(self, x):
        x = self.b._lift(x)
        self.assert_zero(x * (x - 1))

    def assert_zero_ext(self, x):
        self.b.assert_zero_ext(self.cond * x)

    def assert_eq_ext(self, x, y):
        self.assert_zero_ext(self.b._lift(x) - y)


class SymbolicAirBuilder:
    """Records the constraint DAG of one AIR (dimensions as AirLayout,
    p3-miden-lifted-air/src/air.rs:150-163)."""

    def __init__(self, width: int, aux_width: int = 1, num_randomness: int = 1, num_aux_values: int = 0,
                 num_public_values: int = 0, periodic_columns=()):
        self.width, self.aux_width = width, aux_width
        self.num_randomness, self.num_aux_values = num_randomness, num_aux_values
        self.num_public_values = num_public_values
        self.periodic_columns = [np.asarray(c, dtype=np.uint64) % np.uint64(P) for c in periodic_columns]
        self.nodes: list[tuple] = []
        self._ids: dict[tuple, int] = {}
        self.constraints: list[int] = []
        self.is_ext: list[int] = []

    # -- nodes
    def _node(self, op, a=0, b=0, value=0) -> Expr:
        if op in (ADD, MUL) and a > b:  # commutative: one node per operand pair
            a, b = b, a
        key = (op, a, b, value)
        i = self._ids.get(key)
        if i is None:
            i = len(self.nodes)
            self.nodes.append(key)
            self._ids[key] = i
        return Expr(self, i)

    def _lift(self, o) -> Expr:
        return o if isinstance(o, Expr) else self.const(int(o))

    def const(self, v: int) -> Expr:
        return self._node(CONST, value=int(v) % P)

    # -- AirBuilder
    def main(self):
        """(local, next) rows of the main trace."""
        return ([self._node(MAIN, c, 0) for c in range(self.width)],
                [self._node(MAIN, c, 1) for c in range(self.width)])

    def permutation(self):
        """(local, next) rows of the aux trace (extension field)."""
        return ([self._node(AUX, c, 0) for c in range(self.aux_width)],
                [self._node(AUX, c, 1) for c in range(self.aux_width)])

    def public_values(self):
        return [self._node(PUBLIC, i) for i in range(self.num_public_values)]

    def permutation_randomness(self):
        return [self._node(RANDOMNESS, i) for i in range(self.num_randomness)]

    def permutation_values(self):
        return [self._node(AUX_VALUE, i) for i in range(self.num_aux_values)]

    def periodic_values(self):
        return [self._node(PERIODIC, i) for i in range(len(self.periodic_columns))]

    def is_first_row(self):
        return self._node(IS_FIRST_ROW)

    def is_last_row(self):
        return self._node(IS_LAST_ROW)

    def is_transition(self):
        return self._node(IS_TRANSITION)

    def when(self, cond) -> _Filtered:
        return _Filtered(self, self._lift(cond))

    def when_first_row(self) -> _Filtered:
        return self.when(self.is_first_row())

    def when_last_row(self) -> _Filtered:
        return self.when(self.is_last_row())

    def when_transition(self) -> _Filtered:
        return self.when(self.is_transition())

    def assert_zero(self, x):
        self.constraints.append(self._lift(x).i)
        self.is_ext.append(0)

    def assert_eq(self, x, y):
        self.assert_zero(self._lift(x) - y)

    def assert_one(self, x):
        self.assert_zero(self._lift(x) - 1)

    def assert_bool(self, x):
        x = self._lift(x)
        self.assert_zero(x * (x - 1))

    def assert_zero_ext(self, x):
        self.constraints.append(self._lift(x).i)
        self.is_ext.append(1)

    def assert_eq_ext(self, x, y):
        self.assert_zero_ext(self._lift(x) - y)

    def build(self) -> "AirDesc":
        nodes = np.zeros(len(self.nodes), dtype=NODE_DTYPE)
        for i, (op, a, b, v) in enumerate(self.nodes):
            nodes[i] = (op, a, b, 0, v)
        lengths = np.array([len(c) for c in self.periodic_columns], dtype=np.uint64)
        values = (np.concatenate(self.periodic_columns) if self.periodic_columns
                  else np.zeros(0, dtype=np.uint64)).astype(np.uint64)
        return AirDesc(self.width, self.aux_width, self.num_randomness, self.num_aux_values,
                       self.num_public_values, nodes, np.array(self.constraints, dtype=np.uint32),
                       np.array(self.is_ext, dtype=np.uint8), lengths, values)


@dataclass
class AirDesc:
    """The symbolic form of an AIR, laid out as p3g_air_desc (include/p3g.h)."""
    width: int
    aux_width: int
    num_randomness: int
    num_aux_values: int
    num_public_values: int
    nodes: np.ndarray
    constraints: np.ndarray
    is_ext: np.ndarray
    periodic_lengths: np.ndarray
    periodic_values: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def num_periodic(self) -> int:
        return int(self.periodic_lengths.size)

    @property
    def num_constraints(self) -> int:
        return int(self.constraints.size)


def build_air(eval_fn, width: int, **dims) -> AirDesc:
    """Run ``eval_fn`` on a SymbolicAirBuilder with these dimensions (the
    reference's symbolic pass, p3-miden-lifted-air/src/air.rs:225-247)."""
    b = SymbolicAirBuilder(width, **dims)
    eval_fn(b)
    return b.build()
