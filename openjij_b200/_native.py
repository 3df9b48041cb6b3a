"""ctypes binding of libojb200.so (the C ABI declared in include/openjij_b200.h).

This is the thin, allocation-free Python view of the C ABI used by the tests
and the benchmark.  It fails loudly when the library is missing: there is no
CPU fallback for the sweep.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libojb200.so")

OJ_OK = 0
OJ_ERR_ARG = 1
OJ_ERR_OOM = 2
OJ_ERR_CUDA = 3
OJ_ERR_TIMEOUT = 4
OJ_ERR_BOUNDS = 5
OJ_ERR_UNSUPPORTED = 6
OJ_ERR_NODEVICE = 7

OJ_DEVICE_POINTERS = 0x1
OJ_AUTOTUNE = 0x2
KERNEL_SHIFT = 4
KERNELS = {"auto": 0, "colour": 1, "dense_plain": 2, "bitpacked": 3, "dense_tc": 4, "dense_jump": 5}
KERNEL_NAMES = {v: k for k, v in KERNELS.items()}
KERNEL_NAMES[6] = "swendsen_wang"

# every symbol the header declares
EXPORTS = [
    "oj_version", "oj_status_string", "oj_ctx_create", "oj_ctx_destroy", "oj_ctx_set_stream",
    "oj_ctx_synchronize", "oj_ctx_last_error", "oj_graph_create_dense", "oj_graph_create_csr",
    "oj_graph_destroy", "oj_graph_query", "oj_sa_run", "oj_sqa_run", "oj_energy",
    "oj_sa_run_bitpacked_noalloc", "oj_batch_create_dense", "oj_batch_destroy", "oj_sa_run_batched",
    "oj_sw_run", "oj_graph_flip_stats", "oj_batch_flip_stats", "oj_ctx_set_field_recompute",
    "oj_ctx_set_wait_limit", "oj_ctx_inject_fault", "oj_host_alloc", "oj_host_free", "oj_host_is_pinned",
]


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_int32), ("nnz", C.c_int64), ("num_colours", C.c_int32),
                ("max_degree", C.c_int32), ("min_degree", C.c_int32), ("bimodal", C.c_int32),
                ("integer_exact", C.c_int32), ("coupling_abs", C.c_double)]


class RunStats(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("launches", C.c_int32), ("sweeps", C.c_int64),
                ("attempts", C.c_double), ("anneal_ms", C.c_float), ("total_ms", C.c_float),
                ("cluster", C.c_int32), ("threads", C.c_int32), ("variant", C.c_int32), ("tuned", C.c_int32),
                ("accepted", C.c_double), ("field_drift", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["kernel"] = KERNEL_NAMES.get(d["kernel"], d["kernel"])
        return d


class OJError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lib = None


def lib():
    """Load libojb200.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libojb200.so not found at {LIB_PATH}; run openjij_b200.build")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, u32, u64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_uint64, C.c_double
        L.oj_version.restype = C.c_char_p
        L.oj_status_string.restype = C.c_char_p
        L.oj_status_string.argtypes = [i32]
        L.oj_ctx_create.argtypes = [i32, C.POINTER(vp)]
        L.oj_ctx_destroy.argtypes = [vp]
        L.oj_ctx_set_stream.argtypes = [vp, vp]
        L.oj_ctx_synchronize.argtypes = [vp]
        L.oj_ctx_set_field_recompute.argtypes = [vp, i32]
        L.oj_ctx_set_wait_limit.argtypes = [vp, i64]
        L.oj_ctx_inject_fault.argtypes = [vp, i32, i64]
        L.oj_ctx_last_error.argtypes = [vp]
        L.oj_ctx_last_error.restype = C.c_char_p
        L.oj_graph_create_dense.argtypes = [vp, i32, vp, C.POINTER(vp)]
        L.oj_graph_create_csr.argtypes = [vp, i32, vp, vp, vp, C.POINTER(vp)]
        L.oj_graph_destroy.argtypes = [vp]
        L.oj_graph_query.argtypes = [vp, C.POINTER(GraphInfo)]
        L.oj_sa_run.argtypes = [vp, vp, i32, vp, vp, vp, i32, u64, i64, i64, u32, vp,
                                C.POINTER(RunStats)]
        L.oj_sqa_run.argtypes = [vp, vp, i32, i32, vp, dbl, vp, vp, vp, i32, u64, i64, i64, u32, vp, vp,
                                 C.POINTER(RunStats)]
        L.oj_energy.argtypes = [vp, vp, i32, vp, u32, vp]
        L.oj_sa_run_bitpacked_noalloc.argtypes = [vp, vp, i32, vp, vp, vp, i32, u64, i64, i64]
        L.oj_host_alloc.argtypes = [C.c_size_t]
        L.oj_host_alloc.restype = vp
        L.oj_host_free.argtypes = [vp]
        L.oj_host_free.restype = None
        L.oj_host_is_pinned.argtypes = [vp]
        L.oj_host_is_pinned.restype = i32
        L.oj_sw_run.argtypes = [vp, vp, i32, vp, vp, vp, i32, u64, i64, i64, u32, vp, C.POINTER(RunStats)]
        L.oj_graph_flip_stats.argtypes = [vp, vp, i32, vp, dbl, vp, vp, C.POINTER(dbl)]
        L.oj_batch_flip_stats.argtypes = [vp, vp, i32, vp, dbl, vp, vp, vp]
        L.oj_batch_create_dense.argtypes = [vp, i32, vp, vp, vp, C.POINTER(vp)]
        L.oj_batch_destroy.argtypes = [vp]
        L.oj_sa_run_batched.argtypes = [vp, vp, vp, vp, vp, vp, i32, u64, i64, i64, u32, vp,
                                        C.POINTER(RunStats)]
        for name in EXPORTS:
            if name not in ("oj_version", "oj_status_string", "oj_ctx_last_error", "oj_host_alloc",
                            "oj_host_free", "oj_host_is_pinned"):
                getattr(L, name).restype = i32
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):  # torch tensor on the device
        return a.data_ptr()
    return a.ctypes.data


class Context:
    """Owns an oj_ctx (device, stream, workspace)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().oj_ctx_create(device, C.byref(self._h))
        if st != OJ_OK:
            raise OJError(st, "oj_ctx_create: " + lib().oj_status_string(st).decode())
        self.device = device

    def check(self, st, what):
        if st != OJ_OK:
            msg = lib().oj_ctx_last_error(self._h).decode()
            raise OJError(st, f"{what}: {lib().oj_status_string(st).decode()}: {msg}")

    def set_stream(self, stream_handle: int):
        self.check(lib().oj_ctx_set_stream(self._h, C.c_void_p(stream_handle)), "set_stream")

    def synchronize(self):
        self.check(lib().oj_ctx_synchronize(self._h), "synchronize")

    def set_field_recompute(self, sweeps: int):
        """Full field recompute every `sweeps` sweeps of batched / dense-jump runs (0 = never)."""
        self.check(lib().oj_ctx_set_field_recompute(self._h, int(sweeps)), "set_field_recompute")

    def inject_alloc_failure(self, after):
        """Host-side fault injection: the after-th device allocation from now
        fails as out of memory (None clears it)."""
        kind, n = (0, 0) if after is None else (1, int(after))
        self.check(lib().oj_ctx_inject_fault(self._h, kind, n), "inject_fault")

    def set_wait_limit(self, iterations: int):
        """Iterations of the field kernel's bounded pipeline waits (< 0: the default)."""
        self.check(lib().oj_ctx_set_wait_limit(self._h, int(iterations)), "set_wait_limit")

    def close(self):
        if self._h:
            lib().oj_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """Owns an oj_graph built from the symmetric augmented (n+1)x(n+1) matrix."""

    def __init__(self, ctx: Context, n: int, indptr, indices, data):
        self.ctx = ctx
        self._h = C.c_void_p()
        self._keep = (np.ascontiguousarray(indptr, np.int64), np.ascontiguousarray(indices, np.int32),
                      np.ascontiguousarray(data, np.float64))
        ip, ix, dv = self._keep
        ctx.check(lib().oj_graph_create_csr(ctx._h, int(n), _ptr(ip), _ptr(ix), _ptr(dv),
                                            C.byref(self._h)), "oj_graph_create_csr")
        self._keep = None
        self.n = int(n)

    @staticmethod
    def from_dense(ctx: Context, J_aug):
        J = np.ascontiguousarray(J_aug, np.float64)
        g = Graph.__new__(Graph)
        g.ctx = ctx
        g._h = C.c_void_p()
        ctx.check(lib().oj_graph_create_dense(ctx._h, J.shape[0] - 1, _ptr(J), C.byref(g._h)),
                  "oj_graph_create_dense")
        g.n = J.shape[0] - 1
        g._keep = None
        return g

    def info(self) -> dict:
        inf = GraphInfo()
        self.ctx.check(lib().oj_graph_query(self._h, C.byref(inf)), "oj_graph_query")
        return {k: getattr(inf, k) for k, _ in inf._fields_}

    def close(self):
        if self._h:
            lib().oj_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _flags(kernel, device, tune=False):
    f = KERNELS[kernel] << KERNEL_SHIFT
    if device:
        f |= OJ_DEVICE_POINTERS
    if tune:
        f |= OJ_AUTOTUNE
    return f


def sa_run(g: Graph, spins, betas, mcs, seed, kernel="auto", energies=None, device=False,
           first_sweep=0, replica_offset=0, tune=False):
    """spins: int8 [R][n] numpy (in/out) or device tensor/pointer with device=True."""
    R = spins.shape[0] if hasattr(spins, "shape") else None
    b = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int32)
    st = RunStats()
    g.ctx.check(lib().oj_sa_run(g.ctx._h, g._h, int(R), _ptr(spins), _ptr(b), _ptr(m), len(b),
                                int(seed) & 0xFFFFFFFFFFFFFFFF, int(first_sweep), int(replica_offset),
                                _flags(kernel, device, tune), _ptr(energies), C.byref(st)), "oj_sa_run")
    return st.as_dict()


def sw_run(g: Graph, spins, betas, mcs, seed, energies=None, device=False, first_sweep=0, replica_offset=0):
    """Swendsen-Wang annealing of spins [R][n] (oj_sw_run)."""
    R = spins.shape[0]
    b = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int32)
    st = RunStats()
    g.ctx.check(lib().oj_sw_run(g.ctx._h, g._h, int(R), _ptr(spins), _ptr(b), _ptr(m), len(b),
                                int(seed) & 0xFFFFFFFFFFFFFFFF, int(first_sweep), int(replica_offset),
                                _flags("auto", device), _ptr(energies), C.byref(st)), "oj_sw_run")
    return st.as_dict()


def sqa_run(g: Graph, spins, gamma, betas, s, mcs, seed, energies=None, best=None, kernel="auto",
            device=False, first_sweep=0, replica_offset=0, tune=False):
    """spins: int8 [R][T][n]."""
    R, T = spins.shape[0], spins.shape[1]
    b = np.ascontiguousarray(betas, np.float64)
    sv = np.ascontiguousarray(s, np.float64)
    m = np.ascontiguousarray(mcs, np.int32)
    st = RunStats()
    g.ctx.check(lib().oj_sqa_run(g.ctx._h, g._h, int(R), int(T), _ptr(spins), float(gamma), _ptr(b),
                                 _ptr(sv), _ptr(m), len(b), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                 int(first_sweep), int(replica_offset), _flags(kernel, device, tune),
                                 _ptr(energies), _ptr(best), C.byref(st)),
                "oj_sqa_run")
    return st.as_dict()


def sa_run_bitpacked_noalloc(g: Graph, spins_dev, betas, mcs, seed, first_sweep=0, replica_offset=0):
    """The allocation-free bit-packed run; spins_dev is a device tensor [R][n]."""
    b = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int32)
    g.ctx.check(lib().oj_sa_run_bitpacked_noalloc(g.ctx._h, g._h, int(spins_dev.shape[0]), _ptr(spins_dev),
                                                  _ptr(b), _ptr(m), len(b), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                                  int(first_sweep), int(replica_offset)),
                "oj_sa_run_bitpacked_noalloc")


def energy(g: Graph, spins, out=None, device=False):
    R = spins.shape[0]
    if out is None:
        out = np.zeros(R, np.float64)
    g.ctx.check(lib().oj_energy(g.ctx._h, g._h, int(R), _ptr(spins),
                                OJ_DEVICE_POINTERS if device else 0, _ptr(out)), "oj_energy")
    return out


def flip_stats(g: Graph, spins, threshold=1e-8):
    """Single-flip energy changes of spins [n][K] and the smallest coupling
    magnitude above threshold (oj_graph_flip_stats): (quad, lin, abs_min)."""
    s = np.ascontiguousarray(spins, np.int8)
    n, K = s.shape
    quad = np.zeros((n, K), np.float64)
    lin = np.zeros((n, K), np.float64)
    amin = C.c_double(0.0)
    g.ctx.check(lib().oj_graph_flip_stats(g.ctx._h, g._h, int(K), _ptr(s), float(threshold), _ptr(quad),
                                          _ptr(lin), C.byref(amin)), "oj_graph_flip_stats")
    return quad, lin, amin.value


class Batch:
    """Owns an oj_batch: dense instances of uneven size, given as their
    augmented (n+1)x(n+1) matrices (numpy arrays)."""

    def __init__(self, ctx: Context, mats):
        self.ctx = ctx
        self.n = np.array([m.shape[0] - 1 for m in mats], np.int32)
        sizes = np.array([(k + 1) * (k + 1) for k in self.n], np.int64)
        self.offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        flat = np.concatenate([np.ascontiguousarray(m, np.float64).ravel() for m in mats]) if len(mats) \
            else np.zeros(1)
        self._h = C.c_void_p()
        ctx.check(lib().oj_batch_create_dense(ctx._h, len(mats), _ptr(self.n), _ptr(self.offset), _ptr(flat),
                                              C.byref(self._h)), "oj_batch_create_dense")

    def flip_stats(self, spins, threshold=1e-8):
        """oj_batch_flip_stats: spins are the instances' [n[k]][K] blocks back
        to back; returns (quad, lin) of the same shape and abs_min[count]."""
        s = np.ascontiguousarray(spins, np.int8)
        if s.ndim != 2 or s.shape[0] != int(self.n.sum()):
            raise ValueError("spins must have shape (sum(n), K)")
        quad = np.zeros(s.shape, np.float64)
        lin = np.zeros(s.shape, np.float64)
        amin = np.zeros(len(self.n), np.float64)
        self.ctx.check(lib().oj_batch_flip_stats(self.ctx._h, self._h, int(s.shape[1]), _ptr(s), float(threshold),
                                                 _ptr(quad), _ptr(lin), _ptr(amin)), "oj_batch_flip_stats")
        return quad, lin, amin

    def close(self):
        if self._h:
            lib().oj_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sa_run_batched(b: Batch, reads, spins, betas, mcs, seed, energies=None, device=False, first_sweep=0,
                   instance_offset=0, tune=False):
    """spins: int8, the instances' [reads[k]][n[k]] blocks concatenated."""
    r = np.ascontiguousarray(reads, np.int32)
    bb = np.ascontiguousarray(betas, np.float64)
    m = np.ascontiguousarray(mcs, np.int32)
    st = RunStats()
    b.ctx.check(lib().oj_sa_run_batched(b.ctx._h, b._h, _ptr(r), _ptr(spins), _ptr(bb), _ptr(m), len(bb),
                                        int(seed) & 0xFFFFFFFFFFFFFFFF, int(first_sweep), int(instance_offset),
                                        _flags("auto", device, tune), _ptr(energies), C.byref(st)),
                "oj_sa_run_batched")
    d = st.as_dict()
    d["kernel"] = "batched"
    return d
