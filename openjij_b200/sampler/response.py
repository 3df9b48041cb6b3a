"""Sampler result (reference: openjij/sampler/response.py:22-37, a
dimod.SampleSet subclass).  dimod is not a dependency here; the parts of the
SampleSet interface the samplers and their users touch are provided:
``record.sample`` / ``record.energy`` / ``record.num_occurrences``,
``states``, ``energies``, ``first``, ``samples()``, ``variables``, ``vartype``,
``info``, ``change_vartype``."""
from __future__ import annotations

from collections import namedtuple

import numpy as np

from openjij_b200.variable_type import BINARY, SPIN, cast_vartype

Sample = namedtuple("Sample", ["sample", "energy", "num_occurrences"])


class _Record:
    def __init__(self, sample, energy):
        self.sample = sample
        self.energy = energy
        self.num_occurrences = np.ones(len(energy), dtype=np.int64)

    def __len__(self):
        return len(self.energy)


class Response:
    def __init__(self, states, energies, variables, vartype, info=None):
        self.record = _Record(np.asarray(states), np.asarray(energies, dtype=np.float64))
        self.variables = list(variables)
        self.vartype = cast_vartype(vartype)
        self.info = dict(info or {})

    @classmethod
    def from_samples(cls, samples, vartype, energy, info=None, variables=None):
        """``samples``: array [R][n] in the order of ``variables`` (or list of dicts)."""
        if len(samples) and isinstance(samples[0], dict):
            variables = list(samples[0].keys()) if variables is None else list(variables)
            states = np.array([[s[v] for v in variables] for s in samples])
        else:
            states = np.asarray(samples)
            if variables is None:
                variables = list(range(states.shape[1] if states.ndim == 2 else 0))
        if states.ndim == 1:
            states = states.reshape(len(energy), -1)
        return cls(states, energy, variables, vartype, info)

    # ---- openjij Response properties ----------------------------------------
    @property
    def states(self):
        return self.record.sample

    @property
    def energies(self):
        return self.record.energy

    @property
    def indices(self):
        return list(self.variables)

    @property
    def first(self):
        k = int(np.argmin(self.record.energy)) if len(self.record.energy) else 0
        if not len(self.record.energy):
            return Sample({}, 0.0, 0)
        return Sample(dict(zip(self.variables, self.record.sample[k].tolist())),
                      float(self.record.energy[k]), 1)

    @property
    def min_samples(self):
        return self.first.sample

    def samples(self):
        return [dict(zip(self.variables, row.tolist())) for row in self.record.sample]

    def data_vectors(self):
        return {"energy": self.record.energy, "num_occurrences": self.record.num_occurrences}

    def __len__(self):
        return len(self.record.energy)

    def __iter__(self):
        return iter(self.samples())

    def change_vartype(self, vartype, energy_offset: float = 0.0, inplace: bool = True):
        vartype = cast_vartype(vartype)
        states = self.record.sample
        if vartype != self.vartype:
            states = (states + 1) // 2 if vartype == BINARY else 2 * states - 1
        out = self if inplace else Response(states, self.record.energy, self.variables, vartype, self.info)
        out.record.sample = states
        out.record.energy = self.record.energy + energy_offset
        out.vartype = vartype
        return out

    def __repr__(self):
        return f"Response({len(self)} samples, {len(self.variables)} variables, {self.vartype.name})"
