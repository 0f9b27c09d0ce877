"""Test-only stand-in for the third-party ``pygrgl`` module (not installable offline).

It supplies only the names that the reference package ``pygrgl_spmv`` imports at module
level or touches on the artifact path, so that the reference's ``ReferenceRuntime``,
``compile_grg`` and ``save_grg_spmv`` can be imported and run from ``make_golden.py``.
Nothing here implements GRG arithmetic; ``load_immutable_grg`` is deliberately unusable.
"""

from enum import Enum

INVALID_NODE = 0x7FFFFFFFFFFFFFFF
COAL_COUNT_NOT_SET = 0xFFFFFFFF


class TraversalDirection(Enum):
    UP = 0
    DOWN = 1


class MutableGRG:  # only used in an isinstance() check
    pass


class ImmutableGRG:  # only used in type annotations
    pass


class Mutation:
    def __init__(self, position, allele, ref_allele, time):
        self.position = position
        self.allele = allele
        self.ref_allele = ref_allele
        self.time = time


def load_immutable_grg(*_args, **_kwargs):
    raise RuntimeError("the pygrgl stand-in cannot load .grg files")
