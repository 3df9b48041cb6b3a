"""Binary quadratic model of the sampler path.

Follows the reference's ``openjij.model.model.BinaryQuadraticModel``
(openjij/model/model.py:37-109), whose storage and conversions come from
jij-cimod 1.7.x (not vendored in the reference).  The parts the annealing path
uses are written here: construction from Ising / QUBO dicts and from a numpy
matrix, SPIN <-> BINARY conversion, energies, and the augmented interaction
matrix handed to ``cxxjij`` (upper triangle, h in the last column, 1 in the
corner — pinned by the reference's tests/test_model.py:57-68).

Conventions:
  SPIN:   E(s) = sum_{i<j} J_ij s_i s_j + sum_i h_i s_i + offset
  BINARY: E(x) = sum_{i<j} Q_ij x_i x_j + sum_i Q_ii x_i + offset
  x = (s + 1) / 2.
A numpy QUBO matrix is read as E(x) = x^T Q x: diagonal -> linear, and
Q_ij + Q_ji -> the (i, j) quadratic term.
"""
from __future__ import annotations

from typing import Any

import numpy as np
import scipy.sparse as sp

from openjij_b200.variable_type import BINARY, SPIN, Vartype, cast_vartype


def _sorted_labels(labels):
    labels = list(labels)
    try:
        return sorted(labels)
    except TypeError:
        return sorted(labels, key=lambda v: (type(v).__name__, repr(v)))


class BinaryQuadraticModel:
    """BQM with linear and quadratic biases, an offset and a vartype."""

    def __init__(self, linear: dict, quadratic: dict, *args, **kwargs):
        offset = 0.0
        vartype = kwargs.pop("vartype", None)
        sparse = kwargs.pop("sparse", False)
        if "offset" in kwargs:
            offset = kwargs.pop("offset")
        if kwargs:
            raise TypeError(f"unexpected arguments {sorted(kwargs)}")
        if len(args) == 1:
            if isinstance(args[0], (str, Vartype)):
                vartype = args[0]
            else:
                offset = args[0]
        elif len(args) == 2:
            offset, vartype = args
        elif len(args) > 2:
            raise TypeError("BinaryQuadraticModel(linear, quadratic, [offset], vartype)")
        if vartype is None:
            raise TypeError("vartype is required")
        self.vartype = cast_vartype(vartype)
        self.offset = float(offset)
        self.sparse = bool(sparse)
        self.linear: dict = {}
        self.quadratic: dict = {}
        labels = set()
        for v, b in dict(linear).items():
            self.linear[v] = self.linear.get(v, 0.0) + float(b)
            labels.add(v)
        for (u, v), b in dict(quadratic).items():
            labels.add(u)
            labels.add(v)
            if u == v:
                # a diagonal quadratic term: x*x = x (BINARY), s*s = 1 (SPIN)
                if self.vartype == BINARY:
                    self.linear[u] = self.linear.get(u, 0.0) + float(b)
                else:
                    self.offset += float(b)
                continue
            key = (u, v)
            if (v, u) in self.quadratic:
                key = (v, u)
            self.quadratic[key] = self.quadratic.get(key, 0.0) + float(b)
        for v in labels:
            self.linear.setdefault(v, 0.0)
        self.variables = _sorted_labels(labels)
        self.model_type = "openjij.BinaryQuadraticModel"

    # ---- constructors ------------------------------------------------------
    @classmethod
    def from_ising(cls, h: dict, J: dict, offset: float = 0.0, **kwargs):
        return cls(h, J, offset, vartype=SPIN, **kwargs)

    @classmethod
    def from_qubo(cls, Q: dict, offset: float = 0.0, **kwargs):
        linear, quad = {}, {}
        for (u, v), b in Q.items():
            if u == v:
                linear[u] = linear.get(u, 0.0) + b
            else:
                quad[(u, v)] = quad.get((u, v), 0.0) + b
                linear.setdefault(u, 0.0)
                linear.setdefault(v, 0.0)
        return cls(linear, quad, offset, vartype=BINARY, **kwargs)

    @classmethod
    def from_numpy_matrix(cls, mat, variables=None, offset: float = 0.0, vartype="BINARY",
                          sparse: bool = False, **_):
        M = np.asarray(mat, dtype=np.float64)
        if M.ndim != 2 or M.shape[0] != M.shape[1]:
            raise ValueError("matrix must be square")
        n = M.shape[0]
        labels = list(range(n)) if variables is None else list(variables)
        linear = {labels[i]: float(M[i, i]) for i in range(n)}
        U = np.triu(M, 1) + np.tril(M, -1).T
        rows, cols = np.nonzero(U)
        quad = {(labels[i], labels[j]): float(U[i, j]) for i, j in zip(rows, cols)}
        return cls(linear, quad, offset, cast_vartype(vartype), sparse=sparse)

    # ---- views -------------------------------------------------------------
    @property
    def num_variables(self):
        return len(self.variables)

    @property
    def indices(self):
        return self.variables

    def _index(self):
        return {v: i for i, v in enumerate(self.variables)}

    def copy(self):
        out = BinaryQuadraticModel(dict(self.linear), dict(self.quadratic), self.offset, self.vartype,
                                   sparse=self.sparse)
        out.variables = list(self.variables)
        return out

    # ---- vartype conversion ------------------------------------------------
    def _converted(self, vartype):
        vartype = cast_vartype(vartype)
        if vartype == self.vartype:
            return dict(self.linear), dict(self.quadratic), self.offset
        lin, quad, off = {}, {}, self.offset
        if vartype == BINARY:  # SPIN -> BINARY, s = 2x - 1
            for v, h in self.linear.items():
                lin[v] = lin.get(v, 0.0) + 2.0 * h
                off -= h
            for (u, v), J in self.quadratic.items():
                quad[(u, v)] = 4.0 * J
                lin[u] = lin.get(u, 0.0) - 2.0 * J
                lin[v] = lin.get(v, 0.0) - 2.0 * J
                off += J
        else:  # BINARY -> SPIN, x = (s + 1) / 2
            for v, a in self.linear.items():
                lin[v] = lin.get(v, 0.0) + 0.5 * a
                off += 0.5 * a
            for (u, v), b in self.quadratic.items():
                quad[(u, v)] = 0.25 * b
                lin[u] = lin.get(u, 0.0) + 0.25 * b
                lin[v] = lin.get(v, 0.0) + 0.25 * b
                off += 0.25 * b
        return lin, quad, off

    def change_vartype(self, vartype, inplace: bool = True):
        vartype = cast_vartype(vartype)
        lin, quad, off = self._converted(vartype)
        if inplace:
            self.linear, self.quadratic, self.offset, self.vartype = lin, quad, off, vartype
            return self
        out = BinaryQuadraticModel(lin, quad, off, vartype, sparse=self.sparse)
        out.variables = list(self.variables)
        return out

    def to_ising(self):
        lin, quad, off = self._converted(SPIN)
        return lin, quad, off

    def to_qubo(self):
        lin, quad, off = self._converted(BINARY)
        Q = dict(quad)
        for v, a in lin.items():
            Q[(v, v)] = a
        return Q, off

    # ---- energies -----------------------------------------------------------
    def _vector(self, sample):
        idx = self._index()
        if isinstance(sample, dict):
            x = np.zeros(len(self.variables))
            for v, val in sample.items():
                x[idx[v]] = val
            return x
        return np.asarray(sample, dtype=np.float64)

    def energy(self, sample, **_):
        x = self._vector(sample)
        idx = self._index()
        e = self.offset
        for v, a in self.linear.items():
            e += a * x[idx[v]]
        for (u, v), b in self.quadratic.items():
            e += b * x[idx[u]] * x[idx[v]]
        return float(e)

    calc_energy = energy

    def energies(self, samples, **_):
        return np.array([self.energy(s) for s in samples])

    # ---- matrices ------------------------------------------------------------
    def interaction_matrix(self):
        """(n+1)x(n+1) upper-triangular matrix of the model in its own vartype:
        couplings above the diagonal, linear biases in column n, 1 at (n, n)."""
        n = len(self.variables)
        idx = self._index()
        rows, cols, vals = [], [], []
        for (u, v), b in self.quadratic.items():
            i, j = idx[u], idx[v]
            if i > j:
                i, j = j, i
            rows.append(i)
            cols.append(j)
            vals.append(b)
        for v, a in self.linear.items():
            rows.append(idx[v])
            cols.append(n)
            vals.append(a)
        rows.append(n)
        cols.append(n)
        vals.append(1.0)
        m = sp.csr_matrix((vals, (rows, cols)), shape=(n + 1, n + 1))
        m.sum_duplicates()
        if self.sparse:
            return m
        return m.toarray()

    def get_cxxjij_ising_graph(self):
        """``cxxjij.graph.CSRSparse`` (sparse) or ``cxxjij.graph.Dense`` of the
        Ising form and the energy offset (openjij/model/model.py:72-109)."""
        import openjij_b200.cxxjij as cxxjij
        ising = self.change_vartype(SPIN, inplace=False)
        mat = ising.interaction_matrix()
        if self.sparse:
            return cxxjij.graph.CSRSparse(sp.csr_matrix(mat)), ising.offset
        dense = cxxjij.graph.Dense(len(self.variables))
        dense.set_interaction_matrix(np.asarray(mat))
        return dense, ising.offset

    def __repr__(self):
        return (f"BinaryQuadraticModel({self.linear}, {self.quadratic}, {self.offset}, "
                f"{self.vartype.name})")


def make_BinaryQuadraticModel(linear: Any = None, quadratic: Any = None, sparse: bool = False):
    """The reference's factory (openjij/model/model.py:37-40); one class serves all."""
    return BinaryQuadraticModel
