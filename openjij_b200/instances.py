"""Seeded synthetic instances with the shapes of the benchmark workloads.

No public dataset is named for this path; these generators (numpy
``default_rng(seed)``) are the workloads.  Every function returns the
symmetric augmented (n+1)x(n+1) interaction matrix as ``scipy.sparse.csr_matrix``
(h in row/column n, 1 at (n, n)) — the layout of the reference's
``get_interactions()`` (include/openjij/graph/dense.hpp:280-282) — plus the
energy offset (non-zero only for QUBO inputs).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def augmented_csr(mat):
    """(n, indptr int64, indices int32, data float64) of a symmetric augmented
    (n+1)x(n+1) matrix, sorted column indices: the arrays oj_graph_create_csr takes."""
    m = sp.csr_matrix(mat, dtype=np.float64)
    m.sort_indices()
    return (m.shape[0] - 1, np.ascontiguousarray(m.indptr, np.int64), np.ascontiguousarray(m.indices, np.int32),
            np.ascontiguousarray(m.data, np.float64))


def augmented_from_ising(h, J_upper_coo, n):
    """h: [n]; J_upper_coo: (rows, cols, vals) with rows < cols (summed)."""
    r, c, v = (np.asarray(x) for x in J_upper_coo)
    rows = np.concatenate([r, c, np.arange(n), np.full(n, n), [n]])
    cols = np.concatenate([c, r, np.full(n, n), np.arange(n), [n]])
    vals = np.concatenate([v, v, h, h, [1.0]]).astype(np.float64)
    m = sp.csr_matrix((vals, (rows, cols)), shape=(n + 1, n + 1))
    m.sum_duplicates()
    m.eliminate_zeros()
    # keep the corner even if eliminate_zeros ran
    m.sort_indices()
    return m


def dense_augmented(J, h):
    """Dense symmetric J (zero diagonal) and h -> dense augmented matrix."""
    n = len(h)
    A = np.zeros((n + 1, n + 1))
    A[:n, :n] = J
    A[:n, n] = h
    A[n, :n] = h
    A[n, n] = 1.0
    return A


def qubo_to_ising(Q):
    """Symmetric Q with energy x^T Q x -> (J (zero diag, symmetric), h, offset).

    x = (1+s)/2: J_ij = Q_ij/2, h_i = Q_ii/2 + sum_{j!=i} Q_ij/2,
    offset = sum_i Q_ii/2 + sum_{i<j} Q_ij/2.
    """
    Q = np.asarray(Q, dtype=np.float64)
    d = np.diag(Q).copy()
    off = Q - np.diag(d)
    J = off / 2.0
    h = d / 2.0 + off.sum(axis=1) / 2.0
    offset = d.sum() / 2.0 + np.triu(off, 1).sum() / 2.0
    return J, h, offset


def lattice_pm_j(L: int, seed: int = 2):
    """2D L x L periodic square lattice, J in {-1,+1} (p = 1/2), h = 0."""
    rng = np.random.default_rng(seed)
    n = L * L
    idx = np.arange(n).reshape(L, L)
    right = np.roll(idx, -1, axis=1)
    down = np.roll(idx, -1, axis=0)
    a = np.concatenate([idx.ravel(), idx.ravel()])
    b = np.concatenate([right.ravel(), down.ravel()])
    v = rng.choice([-1.0, 1.0], size=a.size)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    return augmented_from_ising(np.zeros(n), (lo, hi, v), n), 0.0


def chimera_pm_j(L: int, seed: int = 6, field: float = 0.0):
    """L x L Chimera lattice (unit cells of 8, site 8 L r + 8 c + z, open
    edges as cxxjij.graph.Chimera builds it): sites 0-3 of a cell couple to
    4-7 of the same cell and to the same site of the cells above and below,
    sites 4-7 to the same site of the cells left and right; J in {-1,+1}
    (p = 1/2), fields uniform in [-field, field]."""
    rng = np.random.default_rng(seed)
    ind = lambda r, c, z: 8 * L * r + 8 * c + z  # noqa: E731
    a, b = [], []
    for r in range(L):
        for c in range(L):
            for z in range(4):
                for w in range(4, 8):
                    a.append(ind(r, c, z))
                    b.append(ind(r, c, w))
                if r + 1 < L:
                    a.append(ind(r, c, z))
                    b.append(ind(r + 1, c, z))
            for z in range(4, 8):
                if c + 1 < L:
                    a.append(ind(r, c, z))
                    b.append(ind(r, c + 1, z))
    a, b = np.array(a), np.array(b)
    n = 8 * L * L
    v = rng.choice([-1.0, 1.0], size=a.size)
    h = rng.uniform(-field, field, n) if field else np.zeros(n)
    return augmented_from_ising(h, (np.minimum(a, b), np.maximum(a, b), v), n), 0.0


def random_regular_pm_j(n: int, d: int = 3, seed: int = 4, max_tries: int = 1000):
    """Random d-regular graph (configuration model, multi-edges and loops
    rejected), J in {-1,+1} (p = 1/2), h = 0."""
    rng = np.random.default_rng(seed)
    for _ in range(max_tries):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        a, b = stubs[0::2], stubs[1::2]
        if np.any(a == b):
            continue
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        key = lo.astype(np.int64) * n + hi
        if np.unique(key).size != key.size:
            continue
        v = rng.choice([-1.0, 1.0], size=lo.size)
        return augmented_from_ising(np.zeros(n), (lo, hi, v), n), 0.0
    raise RuntimeError("could not draw a simple regular graph")


def dense_ising_uniform(n: int, seed: int = 1):
    """J_ij (i<j), h_i ~ U(-1, 1), FP64."""
    rng = np.random.default_rng(seed)
    J = np.triu(rng.uniform(-1.0, 1.0, size=(n, n)), 1)
    J = J + J.T
    h = rng.uniform(-1.0, 1.0, size=n)
    return sp.csr_matrix(dense_augmented(J, h)), 0.0


def dense_qubo_int(n: int, lo: int = -8, hi: int = 8, seed: int = 3):
    """Symmetric integer QUBO, Q_ij ~ U{lo..hi}; energy x^T Q x."""
    rng = np.random.default_rng(seed)
    Q = np.triu(rng.integers(lo, hi + 1, size=(n, n)).astype(np.float64))
    Q = Q + np.triu(Q, 1).T
    J, h, offset = qubo_to_ising(Q)
    return sp.csr_matrix(dense_augmented(J, h)), offset


def dense_qubo_normal(n: int, seed: int):
    """Symmetric QUBO, Q_ij ~ N(0, 1) rounded to FP32."""
    rng = np.random.default_rng(seed)
    Q = np.triu(rng.standard_normal(size=(n, n)).astype(np.float32).astype(np.float64))
    Q = Q + np.triu(Q, 1).T
    J, h, offset = qubo_to_ising(Q)
    return sp.csr_matrix(dense_augmented(J, h)), offset


def uneven_qubo_batch(count: int = 512, nmin: int = 64, nmax: int = 1024, seed: int = 5):
    """``count`` dense N(0,1) QUBOs with N ~ U{nmin..nmax}."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [dense_qubo_normal(int(nk), seed * 100003 + k) for k, nk in enumerate(sizes)]


def geometric_betas(beta_min: float, beta_max: float, num_sweeps: int):
    """The schedule SASampler builds when both betas are given
    (openjij/sampler/sa_sampler.py:967-974 -> schedule_list.hpp:165-181):
    num_sweeps//m betas, m = max(1, num_sweeps//1000) sweeps each."""
    m = max(1, num_sweeps // 1000)
    count = num_sweeps // m
    r = (beta_max / beta_min) ** (1.0 / (count - 1)) if count > 1 else 1.0
    betas = np.empty(count)
    b = beta_min
    for k in range(count):
        betas[k] = b
        b *= r
    return betas, np.full(count, m, dtype=np.int32)
