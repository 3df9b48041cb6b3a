"""Variable types (reference: openjij/variable_type.py, which re-exports dimod's)."""
from __future__ import annotations

import enum


class Vartype(enum.Enum):
    SPIN = frozenset({-1, 1})
    BINARY = frozenset({0, 1})

    def __repr__(self):
        return f"<Vartype.{self.name}>"

    __str__ = __repr__


SPIN = Vartype.SPIN
BINARY = Vartype.BINARY


def cast_vartype(vartype):
    """'SPIN' / 'BINARY' / Vartype -> Vartype (openjij/variable_type.py:23-33)."""
    if isinstance(vartype, Vartype):
        return vartype
    if isinstance(vartype, str):
        if vartype.upper() == "SPIN":
            return SPIN
        if vartype.upper() == "BINARY":
            return BINARY
    raise TypeError("vartype should be SPIN or BINARY")
