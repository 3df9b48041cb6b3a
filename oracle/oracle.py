"""ORACLE — test infrastructure only (ctypes front end of liboj_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
arm may import this module; the openjij_b200 package never does.  It exposes

* the FP64 restatement of OpenJij's CPU single-spin-flip path with the
  reference's Xorshift stream (``ref_*``), pinned by the reference's own
  known-answer tests (tests/test_cxx.py, tests/cxxtest/sampler/quadraitc.hpp);
* replays of the B200 kernels' update order and Philox stream (``replay_*``).

Graphs are passed as the symmetric augmented (n+1)x(n+1) matrix in CSR form,
exactly what ``Dense.get_interactions()`` / ``CSRSparse.get_interactions()``
return in the reference (include/openjij/graph/dense.hpp:280-282).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboj_oracle.so")
_lib = None

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile liboj_oracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_neglog.argtypes = [C.c_uint32]
        L.orc_neglog.restype = C.c_float
        L.orc_neglog_max.argtypes = []
        L.orc_neglog_max.restype = C.c_float
        L.orc_greedy_colour.argtypes = [C.c_int, _i64p, _i32p, _i32p]
        L.orc_kernel_colour.argtypes = [C.c_int, _i64p, _i32p, _i32p]
        L.orc_gen_spin.argtypes = [C.c_uint64, C.c_int, C.c_int, _i8p]
        L.orc_classical_schedule.argtypes = [C.c_double, C.c_double, C.c_int64, _f64p]
        L.orc_transverse_schedule.argtypes = [C.c_int64, _f64p]
        L.orc_energy.argtypes = [C.c_int, _i64p, _i32p, _f64p, _i8p]
        L.orc_energy.restype = C.c_double
        L.orc_ref_sa.argtypes = [C.c_int, _i64p, _i32p, _f64p, _i8p, _f64p, _i64p, C.c_int64,
                                 C.c_uint64, C.c_int]
        L.orc_ref_sa_many.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _i8p, _f64p, _i64p,
                                      C.c_int64, _u64p, C.c_int]
        L.orc_ref_sqa.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _i8p, C.c_double, _f64p,
                                  _f64p, _i64p, C.c_int64, C.c_uint64, C.c_int, _i8p]
        L.orc_ref_sqa_many.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, C.c_int, _i8p,
                                       C.c_double, _f64p, _f64p, _i64p, C.c_int64, _u64p, C.c_int]
        L.orc_replay_sa.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _i8p, _f32p, C.c_int64,
                                    C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_uint32]
        L.orc_replay_sqa.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, C.c_int, _i8p, _f32p,
                                     _f32p, C.c_int64, C.c_uint64, C.c_int]
        L.orc_replay_sa_msc.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _u32p, _u32p,
                                        C.c_int, _u32p, C.c_int64, C.c_uint64, C.c_int]
        L.orc_msc_thresholds.argtypes = [_f32p, C.c_int64, C.c_double, C.c_int, _u32p, _u32p]
        L.orc_sqa_coefficients.argtypes = [_f64p, _f64p, C.c_int64, C.c_double, C.c_int, _f32p, _f32p]
        L.orc_replay_sqa_msc.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, C.c_int, _u32p, _u32p,
                                         _u32p, C.c_int, C.c_int64, C.c_uint64, C.c_int]
        L.orc_sqa_msc_thresholds.argtypes = [_f32p, _f32p, C.c_int64, C.c_double, C.c_int, _u32p, _u32p]
        L.orc_replay_sqa_split.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, C.c_int, _i8p, _u32p,
                                           _u32p, C.c_int, C.c_int64, C.c_uint64, C.c_int]
        L.orc_replay_sa_batch.argtypes = [C.c_int, _i32p, _i64p, _f64p, _i32p, _i8p, _f32p, C.c_int64,
                                          C.c_uint64, C.c_uint32, C.c_int, C.c_void_p, C.c_uint32, C.c_uint32,
                                          C.c_int, C.c_void_p]
        L.orc_ref_sw.argtypes = [C.c_int, _i64p, _i32p, _f64p, _i8p, _f64p, _i64p, C.c_int64, C.c_uint64]
        L.orc_ref_sw_many.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _i8p, _f64p, _i64p, C.c_int64,
                                      _u64p, C.c_int]
        L.orc_replay_sw.argtypes = [C.c_int, _i64p, _i32p, _f64p, C.c_int, _i8p, _f32p, C.c_int64, C.c_uint64,
                                    C.c_int]
        L.orc_gen_spin_seq.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, _i8p]
        _lib = L
    return _lib


def _threads(threads):
    return int(threads if threads else (os.cpu_count() or 1))


# ---------------------------------------------------------------------------
# instance helpers
# ---------------------------------------------------------------------------

class AugCSR:
    """Symmetric augmented (n+1)x(n+1) matrix (h in row/col n, 1 in the corner)."""

    def __init__(self, mat):
        m = sp.csr_matrix(mat, dtype=np.float64)
        m.sort_indices()
        self.n = m.shape[0] - 1
        self.indptr = np.ascontiguousarray(m.indptr, dtype=np.int64)
        self.indices = np.ascontiguousarray(m.indices, dtype=np.int32)
        self.data = np.ascontiguousarray(m.data, dtype=np.float64)
        self.mat = m

    @staticmethod
    def from_ising(h, J, n=None):
        """h: dict or array; J: dict {(i,j): v} (any i != j order, summed)."""
        if n is None:
            keys = list(h.keys()) if isinstance(h, dict) else list(range(len(h)))
            for (i, j) in J:
                keys += [i, j]
            n = (max(keys) + 1) if keys else 0
        A = np.zeros((n + 1, n + 1))
        hv = h.items() if isinstance(h, dict) else enumerate(h)
        for i, v in hv:
            A[i, n] += v
        for (i, j), v in J.items():
            a, b = min(i, j), max(i, j)
            A[a, b] += v
        A[n, n] = 1.0
        S = np.triu(A) + np.triu(A, 1).T
        return AugCSR(S)

    @staticmethod
    def from_upper(upper):
        """Upper-triangular augmented matrix (reference layout) -> symmetric."""
        U = np.triu(np.asarray(upper, dtype=np.float64))
        return AugCSR(U + np.triu(U, 1).T)

    def args(self):
        return (self.n, self.indptr, self.indices, self.data)


# ---------------------------------------------------------------------------
# building blocks
# ---------------------------------------------------------------------------

def philox4x32_10(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def neglog(x: int) -> float:
    return float(lib().orc_neglog(int(x) & 0xFFFFFFFF))


def neglog_max() -> float:
    """The largest value neglog takes over all 2^32 inputs."""
    return float(lib().orc_neglog_max())


def greedy_colour(g: AugCSR):
    nb = neighbour_csr(g)
    out = np.zeros(g.n, np.int32)
    lib().orc_greedy_colour(g.n, nb[0], nb[1], out)
    return out


def kernel_colour(g: AugCSR):
    """The colouring the colour-class kernels sweep by: greedy, classes evened out."""
    nb = neighbour_csr(g)
    out = np.zeros(g.n, np.int32)
    lib().orc_kernel_colour(g.n, nb[0], nb[1], out)
    return out


def neighbour_csr(g: AugCSR):
    """Neighbour lists without diagonal / dummy column and without zeros."""
    rp = [0]
    ci = []
    for i in range(g.n):
        for p in range(g.indptr[i], g.indptr[i + 1]):
            j = g.indices[p]
            if j != i and j != g.n and g.data[p] != 0.0:
                ci.append(j)
        rp.append(len(ci))
    return np.asarray(rp, np.int64), np.asarray(ci, np.int32)


def gen_spin(seed: int, n: int, engine: str = "xorshift"):
    out = np.zeros(n, np.int8)
    lib().orc_gen_spin(int(seed), n, 0 if engine == "xorshift" else 1, out)
    return out


def gen_spin_seq(seed: int, n: int, count: int, engine: str = "xorshift"):
    out = np.zeros((count, n), np.int8)
    lib().orc_gen_spin_seq(int(seed), n, count, 0 if engine == "xorshift" else 1, out)
    return out


def classical_schedule(beta_min, beta_max, num_call):
    out = np.zeros(num_call, np.float64)
    lib().orc_classical_schedule(float(beta_min), float(beta_max), int(num_call), out)
    return out


def transverse_schedule(num_call):
    out = np.zeros(num_call, np.float64)
    lib().orc_transverse_schedule(int(num_call), out)
    return out


def energy(g: AugCSR, spins):
    s = np.ascontiguousarray(spins, np.int8)
    return float(lib().orc_energy(*g.args(), s))


def energies(g: AugCSR, spins2d):
    return np.array([energy(g, s) for s in np.asarray(spins2d)])


# ---------------------------------------------------------------------------
# reference restatement
# ---------------------------------------------------------------------------

def ref_sa(g: AugCSR, init, betas, mcs, seed, engine="xorshift"):
    s = np.array(init, np.int8, copy=True)
    b = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int64)
    lib().orc_ref_sa(*g.args(), s, b, m, len(b), int(seed), 0 if engine == "xorshift" else 1)
    return s


def ref_sa_many(g: AugCSR, init2d, betas, mcs, seeds, threads=None):
    s = np.array(init2d, np.int8, copy=True, order="C")
    b = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int64)
    sd = np.ascontiguousarray(seeds, np.uint64)
    lib().orc_ref_sa_many(*g.args(), s.shape[0], s, b, m, len(b), sd, _threads(threads))
    return s


def ref_sqa(g: AugCSR, trotter_init, gamma, betas, ss, mcs, seed, engine="xorshift"):
    """trotter_init: [T][n].  Returns (trotter spins [T][n], get_solution spins)."""
    S = np.array(trotter_init, np.int8, copy=True, order="C")
    T = S.shape[0]
    best = np.zeros(g.n, np.int8)
    lib().orc_ref_sqa(*g.args(), T, S, float(gamma), np.ascontiguousarray(betas, np.float64),
                      np.ascontiguousarray(ss, np.float64), np.ascontiguousarray(mcs, np.int64),
                      len(betas), int(seed), 0 if engine == "xorshift" else 1, best)
    return S, best


def ref_sqa_many(g: AugCSR, init3d, gamma, betas, ss, mcs, seeds, threads=None):
    S = np.array(init3d, np.int8, copy=True, order="C")
    R, T, _ = S.shape
    lib().orc_ref_sqa_many(*g.args(), R, T, S, float(gamma),
                           np.ascontiguousarray(betas, np.float64),
                           np.ascontiguousarray(ss, np.float64),
                           np.ascontiguousarray(mcs, np.int64), len(betas),
                           np.ascontiguousarray(seeds, np.uint64), _threads(threads))
    return S


# ---------------------------------------------------------------------------
# replays of the B200 kernels
# ---------------------------------------------------------------------------

def replay_sa(g: AugCSR, init2d, betas_per_sweep, seed, mode="colour", threads=None, rep0=0, sweep0=0):
    """rep0 / sweep0: global index of replica 0 and of the first sweep (shards, split runs)."""
    s = np.array(init2d, np.int8, copy=True, order="C")
    b = np.ascontiguousarray(betas_per_sweep, np.float32)
    lib().orc_replay_sa(*g.args(), s.shape[0], s, b, len(b), int(seed),
                        0 if mode == "colour" else 1, _threads(threads), int(rep0), int(sweep0))
    return s


def sqa_coefficients(betas, ss, gamma, T):
    b = np.ascontiguousarray(betas, np.float64)
    s = np.ascontiguousarray(ss, np.float64)
    a = np.zeros(len(b), np.float32)
    bb = np.zeros(len(b), np.float32)
    lib().orc_sqa_coefficients(b, s, len(b), float(gamma), int(T), a, bb)
    return a, bb


def replay_sqa(g: AugCSR, init3d, coef_a, coef_b, seed, threads=None):
    S = np.array(init3d, np.int8, copy=True, order="C")
    R, T, _ = S.shape
    a = np.ascontiguousarray(coef_a, np.float32)
    bb = np.ascontiguousarray(coef_b, np.float32)
    lib().orc_replay_sqa(*g.args(), R, T, S, a, bb, len(a), int(seed), _threads(threads))
    return S


def pack_words(spins2d):
    """int8 [R][n] (R multiple of 32) -> u32 [R/32][n], bit j = (s == -1)."""
    s = np.asarray(spins2d)
    R, n = s.shape
    G = R // 32
    bits = (s.reshape(G, 32, n) < 0).astype(np.uint64)
    w = np.zeros((G, n), np.uint64)
    for j in range(32):
        w |= bits[:, j, :] << np.uint64(j)
    return w.astype(np.uint32)


def unpack_words(words):
    w = np.asarray(words, np.uint32)
    G, n = w.shape
    out = np.empty((G, 32, n), np.int8)
    for j in range(32):
        out[:, j, :] = np.where((w >> np.uint32(j)) & np.uint32(1), -1, 1)
    return out.reshape(G * 32, n)


def msc_thresholds(betas_per_sweep, c, dmax):
    b = np.ascontiguousarray(betas_per_sweep, np.float32)
    thr = np.zeros((len(b), dmax + 1), np.uint32)
    alw = np.zeros(len(b), np.uint32)
    lib().orc_msc_thresholds(b, len(b), float(c), int(dmax), thr, alw)
    return thr, alw


def replay_sa_msc(g: AugCSR, init2d, thr, always, seed, threads=None):
    """thr: [sweeps][dmax+1] u32; always: [sweeps] u32 bitmask."""
    w = np.ascontiguousarray(pack_words(init2d), np.uint32)
    thr = np.ascontiguousarray(thr, np.uint32)
    alw = np.ascontiguousarray(always, np.uint32)
    lib().orc_replay_sa_msc(*g.args(), w.shape[0], w, thr, thr.shape[1] - 1, alw, thr.shape[0],
                            int(seed), _threads(threads))
    return unpack_words(w)


def pack_slices(spins3d):
    """int8 [R][T][n] (T <= 32) -> u32 [R][n], bit t = (s_t == -1)."""
    s = np.asarray(spins3d)
    R, T, n = s.shape
    w = np.zeros((R, n), np.uint64)
    for t in range(T):
        w |= (s[:, t, :] < 0).astype(np.uint64) << np.uint64(t)
    return w.astype(np.uint32)


def unpack_slices(words, T):
    w = np.asarray(words, np.uint32)
    R, n = w.shape
    out = np.empty((R, T, n), np.int8)
    for t in range(T):
        out[:, t, :] = np.where((w >> np.uint32(t)) & np.uint32(1), -1, 1)
    return out


def sqa_msc_thresholds(coef_a, coef_b, c, dmax):
    a = np.ascontiguousarray(coef_a, np.float32)
    b = np.ascontiguousarray(coef_b, np.float32)
    thr = np.zeros((len(a), (dmax + 1) * 3), np.uint32)
    mode = np.zeros((len(a), 2), np.uint32)
    lib().orc_sqa_msc_thresholds(a, b, len(a), float(c), int(dmax), thr, mode)
    return thr, mode


def replay_sqa_msc(g: AugCSR, init3d, thr, mode, seed, threads=None):
    """Bit-packed SQA replay; thr [sweeps][(dmax+1)*3], mode [sweeps][2]."""
    R, T, _ = np.shape(init3d)
    w = np.ascontiguousarray(pack_slices(init3d), np.uint32)
    thr = np.ascontiguousarray(thr, np.uint32)
    mode = np.ascontiguousarray(mode, np.uint32)
    dmax = thr.shape[1] // 3 - 1
    lib().orc_replay_sqa_msc(*g.args(), R, T, w, thr, mode, dmax, thr.shape[0], int(seed), _threads(threads))
    return unpack_slices(w, T)


def replay_sqa_split(g: AugCSR, init3d, thr, mode, seed, threads=None):
    """Slice-split bit-packed SQA replay on [R][T][n] spins (even T <= 64)."""
    S = np.array(init3d, np.int8, copy=True, order="C")
    R, T, _ = S.shape
    thr = np.ascontiguousarray(thr, np.uint32)
    mode = np.ascontiguousarray(mode, np.uint32)
    dmax = thr.shape[1] // 3 - 1
    lib().orc_replay_sqa_split(*g.args(), R, T, S, thr, mode, dmax, thr.shape[0], int(seed), _threads(threads))
    return S


def replay_sa_batch(mats, reads, spins_flat, betas_per_sweep, seed, inst0=0, threads=None, fields=False,
                    rep0=0, sweep0=0, recompute=16, drift=False):
    """Batched dense SA replay; mats: augmented (n+1)x(n+1) FP64 matrices,
    spins_flat: the instances' [reads[m]][n[m]] int8 blocks concatenated.
    The fields start from (and, before every global sweep that is a multiple
    of ``recompute``, are set anew to) the tensor-core field kernel's
    definition; 0 = never anew.  fields=True also returns the final
    incrementally updated FP32 fields, drift=True the largest |f - f_exact| at
    the recompute points and after the last sweep (per replica).
    inst0 / rep0 / sweep0: global index of instance 0, of every instance's
    replica 0 and of the first sweep (a slice of a larger run)."""
    n = np.array([m.shape[0] - 1 for m in mats], np.int32)
    sizes = np.array([(k + 1) * (k + 1) for k in n], np.int64)
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    flat = np.ascontiguousarray(np.concatenate([np.asarray(m, np.float64).ravel() for m in mats]))
    s = np.array(spins_flat, np.int8, copy=True)
    b = np.ascontiguousarray(betas_per_sweep, np.float32)
    fo = np.zeros(s.shape, np.float32) if fields else None
    dr = np.zeros(int(np.sum(reads)), np.float32) if drift else None
    lib().orc_replay_sa_batch(len(mats), n, offset, flat, np.ascontiguousarray(reads, np.int32), s, b, len(b),
                              int(seed), int(inst0), _threads(threads),
                              None if fo is None else fo.ctypes.data, int(rep0), int(sweep0), int(recompute),
                              None if dr is None else dr.ctypes.data)
    out = (s,)
    if fields:
        out += (fo,)
    if drift:
        out += (dr,)
    return out if len(out) > 1 else s


def ref_sw_many(g: AugCSR, init2d, betas, mcs, seeds, threads=None):
    """Reference Swendsen-Wang reads (Xorshift seeded per read), result s_i * s_dummy."""
    s = np.array(init2d, np.int8, copy=True, order="C")
    lib().orc_ref_sw_many(*g.args(), s.shape[0], s, np.ascontiguousarray(betas, np.float64),
                          np.ascontiguousarray(mcs, np.int64), len(betas),
                          np.ascontiguousarray(seeds, np.uint64), _threads(threads))
    return s


def replay_sw(g: AugCSR, init2d, betas_per_sweep, seed, threads=None):
    """Replay of the B200 Swendsen-Wang kernel."""
    s = np.array(init2d, np.int8, copy=True, order="C")
    b = np.ascontiguousarray(betas_per_sweep, np.float32)
    lib().orc_replay_sw(*g.args(), s.shape[0], s, b, len(b), int(seed), _threads(threads))
    return s


def beta_range_reference(J_aug, beta_max=None, beta_min=None, num_sweeps=1000, seed=None):
    """[beta_max, beta_min] of SASampler's automatic schedule, restated from
    openjij/sampler/sa_sampler.py:872-965 on the augmented matrix J_aug (dense
    ndarray or scipy sparse, as graph.get_interactions() returns it): random
    configurations from np.random, their single-flip energy changes by a
    matrix product, and the smallest |entry| above 1e-8."""
    if seed is not None:
        np.random.seed(seed)
    THRESHOLD = 1e-8
    dE_max = dE_min = 1.0
    rate_dE = 0.5
    dense = isinstance(J_aug, np.ndarray)
    if beta_min is None or beta_max is None:
        if J_aug.shape[0] > 1:
            s = np.random.choice([-1, 1], size=(J_aug.shape[0], 2))
            s[-1, :] = 1
            quad = np.asarray(J_aug[:-1, :-1] @ s[:-1, :]) * (-2 * s[:-1, :])
            hcol = J_aug[:-1, -1][:, np.newaxis] if dense else J_aug[:-1, -1].toarray()
            lin = hcol * s[:-1]
            qa = np.abs(quad)
            if np.any(qa > THRESHOLD):
                rate_dE = np.max(np.abs(lin[qa > THRESHOLD]) / (qa[qa > THRESHOLD].mean() + THRESHOLD))
            pos = quad[quad > THRESHOLD]
            if len(pos) == 0:
                dE_min, dE_max = 1.0, 1.1
            else:
                dE_max = np.median(pos, axis=0).mean()
                dE_min = np.min(pos, axis=0).mean()
    n = J_aug.shape[0]
    prob_init = 9 / 10 - 8 / 10 * np.tanh(rate_dE / 50) + THRESHOLD
    prob_final = 1 / 1000
    if beta_min is None:
        lo, hi = -np.log(prob_init) / dE_max, -np.log(prob_init) / dE_min
        for _ in range(5):
            b = (lo + hi) / 2
            f = 2 * b * prob_init - np.exp(-b * dE_min) + np.exp(-b * dE_max)
            if abs(f) < 1e-8:
                break
            if f > 0:
                hi = b
            else:
                lo = b
        beta_min = lo * 0.8 + (lo * 1.5 - lo * 0.8) * np.tanh(num_sweeps / n)
    if beta_max is None:
        vals = np.abs(J_aug).ravel() if dense else np.abs(sp.csr_matrix(J_aug).data)
        int_min = max(np.min(vals[vals > THRESHOLD]), dE_min / 10.0)
        b_int = -np.log(prob_final) / int_min
        b_dE = -np.log(prob_final) / dE_min
        if rate_dE < 2:
            lo, hi = min(b_dE, b_int), max(b_dE, b_int)
            beta_max = lo + (hi - lo) * np.tanh(num_sweeps / (2 * n))
        else:
            beta_max = -np.log(prob_final) / max(dE_min, int_min) / min(100, num_sweeps // 10 + 1)
        if beta_max < beta_min:
            beta_max = beta_min * 10.0
    if rate_dE > 1:
        beta_min *= rate_dE
        beta_max *= rate_dE
    return [beta_max, beta_min]
