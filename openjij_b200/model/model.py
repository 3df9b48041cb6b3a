"""Binary quadratic model of the sampler path.

Follows the reference's ``openjij.model.model.BinaryQuadraticModel``
(openjij/model/model.py:37-109), whose storage and conversions come from
jij-cimod 1.7.x (not vendored in the reference).  The parts the annealing path
uses are written here: construction from Ising / QUBO dicts and from a numpy
matrix, SPIN <-> BINARY conversion, energies, and the augmented interaction
matrix handed to ``cxxjij`` (upper triangle, h in the last column, 1 in the
corner — pinned by the reference's tests/test_model.py:57-68).

Storage is by variable index, in numpy arrays (cimod keeps C++ containers):
the sorted labels, the linear biases, and the couplings as (i, j, value) with
i < j, one entry per pair.  ``linear`` / ``quadratic`` are dict views built
on request; conversions, the interaction matrix and energies work on the
arrays, so a dense model of a few thousand variables goes from a numpy matrix
to the GPU graph without per-coupling Python.

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


def _merge_pairs(n, qi, qj, qv):
    """Canonical couplings: i < j, one entry per pair, values of repeated
    pairs summed in input order."""
    a = np.minimum(qi, qj).astype(np.int64)
    b = np.maximum(qi, qj).astype(np.int64)
    qv = np.asarray(qv, np.float64)
    if len(a) == 0:
        return a, b, qv
    w = max(n, 1)
    uniq, inv = np.unique(a * w + b, return_inverse=True)
    vals = np.bincount(inv, weights=qv, minlength=len(uniq))
    return uniq // w, uniq % w, vals


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
        vartype = cast_vartype(vartype)
        lin_items = list(dict(linear).items()) if linear else []
        quad_items = list(dict(quadratic).items()) if quadratic else []
        labels = {v for v, _ in lin_items}
        for (u, v), _ in quad_items:
            labels.add(u)
            labels.add(v)
        variables = _sorted_labels(labels)
        idx = {v: i for i, v in enumerate(variables)}
        n = len(variables)
        lin = np.zeros(n)
        for v, b in lin_items:
            lin[idx[v]] += float(b)
        m = len(quad_items)
        qi = np.fromiter((idx[k[0]] for k, _ in quad_items), np.int64, m)
        qj = np.fromiter((idx[k[1]] for k, _ in quad_items), np.int64, m)
        qv = np.fromiter((float(b) for _, b in quad_items), np.float64, m)
        offset = float(offset)
        diag = qi == qj
        if np.any(diag):
            # a diagonal quadratic term: x*x = x (BINARY), s*s = 1 (SPIN)
            if vartype == BINARY:
                np.add.at(lin, qi[diag], qv[diag])
            else:
                for b in qv[diag]:
                    offset += float(b)
            qi, qj, qv = qi[~diag], qj[~diag], qv[~diag]
        self._set(variables, lin, *_merge_pairs(n, qi, qj, qv), offset, vartype, sparse)

    def _set(self, variables, lin, qi, qj, qv, offset, vartype, sparse):
        self.variables = list(variables)
        self._lin = np.asarray(lin, np.float64)
        self._qi, self._qj, self._qv = qi, qj, np.asarray(qv, np.float64)
        self.offset = float(offset)
        self.vartype = cast_vartype(vartype)
        self.sparse = bool(sparse)
        self.model_type = "openjij.BinaryQuadraticModel"

    @classmethod
    def _from_arrays(cls, variables, lin, qi, qj, qv, offset, vartype, sparse):
        out = cls.__new__(cls)
        out._set(variables, lin, qi, qj, qv, offset, vartype, sparse)
        return out

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
        U = np.triu(M, 1) + np.tril(M, -1).T
        qi, qj = np.nonzero(U)
        qv = U[qi, qj]
        order = _sorted_labels(labels)
        if order == labels:
            return cls._from_arrays(labels, np.diag(M).copy(), qi.astype(np.int64), qj.astype(np.int64), qv,
                                    offset, vartype, sparse)
        pos = {v: k for k, v in enumerate(order)}
        perm = np.array([pos[v] for v in labels], np.int64)
        lin = np.zeros(n)
        lin[perm] = np.diag(M)
        return cls._from_arrays(order, lin, *_merge_pairs(n, perm[qi], perm[qj], qv), offset, vartype, sparse)

    # ---- views -------------------------------------------------------------
    @property
    def linear(self):
        return {v: float(b) for v, b in zip(self.variables, self._lin)}

    @property
    def quadratic(self):
        V = self.variables
        return {(V[i], V[j]): float(b) for i, j, b in zip(self._qi.tolist(), self._qj.tolist(), self._qv)}

    @property
    def num_variables(self):
        return len(self.variables)

    @property
    def indices(self):
        return self.variables

    def get_linear(self):
        return self.linear

    def get_quadratic(self):
        return self.quadratic

    def get_offset(self):
        return self.offset

    def get_vartype(self):
        return self.vartype

    def get_variables(self):
        return list(self.variables)

    def __len__(self):
        return len(self.variables)

    def _index(self):
        return {v: i for i, v in enumerate(self.variables)}

    def copy(self):
        return BinaryQuadraticModel._from_arrays(self.variables, self._lin.copy(), self._qi, self._qj,
                                                 self._qv.copy(), self.offset, self.vartype, self.sparse)

    # ---- vartype conversion ------------------------------------------------
    def _converted_arrays(self, vartype):
        """(lin, qv, offset) in ``vartype``; the coupling pairs stay."""
        vartype = cast_vartype(vartype)
        lin, qv, off = self._lin, self._qv, self.offset
        if vartype == self.vartype:
            return lin.copy(), qv.copy(), off
        n = len(lin)
        adj = np.bincount(self._qi, weights=qv, minlength=n) + np.bincount(self._qj, weights=qv, minlength=n)
        if vartype == BINARY:  # SPIN -> BINARY, s = 2x - 1
            return 2.0 * lin - 2.0 * adj, 4.0 * qv, off - float(np.sum(lin)) + float(np.sum(qv))
        # BINARY -> SPIN, x = (s + 1) / 2
        return 0.5 * lin + 0.25 * adj, 0.25 * qv, off + 0.5 * float(np.sum(lin)) + 0.25 * float(np.sum(qv))

    def _dicts(self, lin, qv):
        V = self.variables
        return ({v: float(b) for v, b in zip(V, lin)},
                {(V[i], V[j]): float(b) for i, j, b in zip(self._qi.tolist(), self._qj.tolist(), qv)})

    def change_vartype(self, vartype, inplace: bool = True):
        vartype = cast_vartype(vartype)
        lin, qv, off = self._converted_arrays(vartype)
        if inplace:
            self._lin, self._qv, self.offset, self.vartype = lin, qv, off, vartype
            return self
        return BinaryQuadraticModel._from_arrays(self.variables, lin, self._qi, self._qj, qv, off, vartype,
                                                 self.sparse)

    def to_ising(self):
        lin, qv, off = self._converted_arrays(SPIN)
        h, J = self._dicts(lin, qv)
        return h, J, off

    def to_qubo(self):
        lin, qv, off = self._converted_arrays(BINARY)
        a, Q = self._dicts(lin, qv)
        for v, b in a.items():
            Q[(v, v)] = b
        return Q, off

    # ---- energies -----------------------------------------------------------
    def _vector(self, sample):
        if isinstance(sample, dict):
            idx = self._index()
            x = np.zeros(len(self.variables))
            for v, val in sample.items():
                x[idx[v]] = val
            return x
        return np.asarray(sample, dtype=np.float64)

    def energy(self, sample, **_):
        x = self._vector(sample)
        return float(self.offset + self._lin @ x + np.sum(self._qv * x[self._qi] * x[self._qj]))

    calc_energy = energy

    def energies(self, samples, **_):
        if isinstance(samples, (list, tuple)) and samples and isinstance(samples[0], dict):
            return np.array([self.energy(s) for s in samples])
        X = np.atleast_2d(np.asarray(samples, dtype=np.float64))
        n = len(self._lin)
        U = sp.csr_matrix((self._qv, (self._qi, self._qj)), shape=(n, n))
        return self.offset + X @ self._lin + np.einsum("rn,rn->r", np.asarray(U @ X.T).T, X)

    # ---- matrices ------------------------------------------------------------
    def _matrix(self, lin, qv, sparse):
        n = len(lin)
        if sparse:
            rows = np.concatenate([self._qi, np.arange(n), [n]])
            cols = np.concatenate([self._qj, np.full(n, n), [n]])
            vals = np.concatenate([qv, lin, [1.0]])
            m = sp.csr_matrix((vals, (rows, cols)), shape=(n + 1, n + 1))
            m.sum_duplicates()
            return m
        M = np.zeros((n + 1, n + 1))
        M[self._qi, self._qj] = qv
        M[:n, n] = lin
        M[n, n] = 1.0
        return M

    def interaction_matrix(self):
        """(n+1)x(n+1) upper-triangular matrix of the model in its own vartype:
        couplings above the diagonal, linear biases in column n, 1 at (n, n)."""
        return self._matrix(self._lin, self._qv, self.sparse)

    def get_cxxjij_ising_graph(self):
        """``cxxjij.graph.CSRSparse`` (sparse) or ``cxxjij.graph.Dense`` of the
        Ising form and the energy offset (openjij/model/model.py:72-109)."""
        import openjij_b200.cxxjij as cxxjij
        lin, qv, off = self._converted_arrays(SPIN)
        mat = self._matrix(lin, qv, self.sparse)
        if self.sparse:
            return cxxjij.graph.CSRSparse(mat), off
        dense = cxxjij.graph.Dense(len(self.variables))
        dense.set_interaction_matrix(mat)
        return dense, off

    def __repr__(self):
        return (f"BinaryQuadraticModel({self.linear}, {self.quadratic}, {self.offset}, "
                f"{self.vartype.name})")


def make_BinaryQuadraticModel(linear: Any = None, quadratic: Any = None, sparse: bool = False):
    """The reference's factory (openjij/model/model.py:37-40); one class serves all."""
    return BinaryQuadraticModel
