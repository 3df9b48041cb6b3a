"""openjij_b200 — B200-native single-spin-flip annealing (SA / SQA) behind
OpenJij's sampler API.

    import openjij_b200 as oj
    res = oj.SASampler().sample_ising(h, J, num_reads=1024, seed=1)

``oj.cxxjij`` keeps OpenJij's C++ binding surface (graph / system /
algorithm / utility / result); every sweep runs on the GPU through the C ABI
of include/openjij_b200.h.  There is no CPU fallback: importing the package
fails when the native extension has not been built.
"""
from __future__ import annotations

import sys as _sys

from . import _cxxjij as cxxjij

for _name in ("graph", "system", "algorithm", "utility", "result"):
    _sys.modules[__name__ + ".cxxjij." + _name] = getattr(cxxjij, _name)
_sys.modules[__name__ + ".cxxjij"] = cxxjij

from .variable_type import BINARY, SPIN, Vartype, cast_vartype  # noqa: E402
from .model.model import BinaryQuadraticModel  # noqa: E402
from .sampler.response import Response  # noqa: E402
from .sampler.sa_sampler import SASampler  # noqa: E402
from .sampler.sqa_sampler import SQASampler  # noqa: E402

__all__ = ["cxxjij", "SPIN", "BINARY", "Vartype", "cast_vartype", "Response", "SASampler",
           "SQASampler", "BinaryQuadraticModel"]
