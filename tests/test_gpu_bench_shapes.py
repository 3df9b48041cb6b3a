"""Spin-for-spin parity at the benchmarked workloads and launch shapes.

The throughput numbers come from the full-size instances with many replicas,
clusters and work items; these tests run exactly those instances, replica
counts and launch shapes (the default, the autotuner's and forced
alternatives) on a shortened schedule over the same beta / gamma range, and
compare with the kernels' CPU replays — on every replica for the lattice and
SQA kernels, on replica slices at both ends of the work queue for the dense
kernel, and on a sample of instances for the batch.  Last, an equilibrium
check of the lattice kernel against the restatement of the reference's CPU
path on the benchmark lattice itself."""
import os

import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _init(shape, seed):
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=shape)


def _per_sweep(betas, mcs):
    return np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)


def _env(monkeypatch, **kv):
    for k, v in kv.items():
        if v is None:
            monkeypatch.delenv(k, raising=False)
        else:
            monkeypatch.setenv(k, str(v))


# ---- config 2: L = 128 +-J lattice, 1024 replicas, bit-packed kernel ------------

def test_lattice_L128_R1024_every_shape(ctx, monkeypatch):
    m, _ = I.lattice_pm_j(128, seed=2)
    g = O.AugCSR(m)
    R = 1024
    betas, mcs = I.geometric_betas(0.1, 5.0, 12)  # the benchmark's beta range in 12 sweeps
    s0 = _init((R, g.n), 21)
    thr, alw = O.msc_thresholds(_per_sweep(betas, mcs), 1.0, 4)
    ref = O.replay_sa_msc(g, s0, thr, alw, 777)
    want_e = O.energies(g, ref)
    seen = set()
    for cluster, threads, tune in [(None, None, False), (4, 1024, False), (2, 512, False), (8, 256, False),
                                   (16, 1024, False), (None, None, True)]:
        _env(monkeypatch, OJ_MSC_CLUSTER=cluster, OJ_MSC_THREADS=threads)
        dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
        s = s0.copy()
        e = np.zeros(R)
        st = N.sa_run(dg, s, betas, mcs, seed=777, kernel="bitpacked", energies=e, tune=tune)
        assert st["kernel"] == "bitpacked"
        if cluster:
            assert (st["cluster"], st["threads"]) == (cluster, threads)
        seen.add((st["cluster"], st["threads"]))
        np.testing.assert_array_equal(s, ref, err_msg=f"shape {st['cluster']} x {st['threads']}")
        np.testing.assert_allclose(e, want_e, rtol=0, atol=1e-9)
        dg.close()
    assert (4, 512) in seen  # the planner's shape for 32 groups on 148 SMs


# ---- config 4: SQA on the 3-regular n = 4096 graph, T = 32, 256 replicas -------

def test_sqa_3regular_N4096_T32_R256_every_shape(ctx, monkeypatch):
    m, _ = I.random_regular_pm_j(4096, 3, seed=4)
    g = O.AugCSR(m)
    R, T, S = 256, 32, 12
    ss = np.linspace(0.0, 1.0, S)  # Gamma (1 - s): 1 -> 0, as the benchmark, in 12 sweeps
    betas = np.full(S, 10.0)
    mcs = np.ones(S, np.int32)
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    thr, mode = O.sqa_msc_thresholds(a, b, 1.0, 3)
    t0 = _init((R, T, g.n), 22)
    ref = O.replay_sqa_split(g, t0, thr, mode, 4242)
    want_e = O.energies(g, ref.reshape(R * T, g.n)).reshape(R, T)
    for cluster, threads, tune in [(None, None, False), (1, 256, False), (2, 512, False), (4, 256, False),
                                   (None, None, True)]:
        _env(monkeypatch, OJ_SQA_CLUSTER=cluster, OJ_SQA_THREADS=threads)
        dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
        t = t0.copy()
        e = np.zeros((R, T))
        best = np.zeros(R, np.int32)
        st = N.sqa_run(dg, t, 1.0, betas, ss, mcs, seed=4242, kernel="bitpacked", energies=e, best=best,
                       tune=tune)
        assert st["kernel"] == "bitpacked"
        if cluster:
            assert (st["cluster"], st["threads"]) == (cluster, threads)
        np.testing.assert_array_equal(t, ref, err_msg=f"shape {st['cluster']} x {st['threads']}")
        np.testing.assert_allclose(e, want_e, rtol=0, atol=1e-9)
        np.testing.assert_array_equal(best, np.argmin(want_e, axis=1))
        dg.close()


# ---- config 3: dense integer QUBO n = 2048, 4096 replicas, dense jump kernel ----

@pytest.mark.parametrize("variant", [None, 82, 45, 162])
def test_dense_qubo_N2048_R4096_hot_sweeps(ctx, monkeypatch, variant):
    """The flip-heavy first sweeps from a random state (about half the spins
    flip), int8 dp4a initial fields, FP16 flip rows, in-kernel energies."""
    _env(monkeypatch, OJ_BATCH_VARIANT=variant)
    m, _ = I.dense_qubo_int(2048, seed=3)
    g = O.AugCSR(m)
    A = m.toarray()
    R, n = 4096, 2048
    bf, mf = I.geometric_betas(0.05, 5.0, 1000)
    betas, mcs = bf[:3], mf[:3]  # the schedule's first three sweeps
    s0 = _init((R, n), 23)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    s = s0.copy()
    e = np.zeros(R)
    st = N.sa_run(dg, s, betas, mcs, seed=99, kernel="dense_jump", energies=e)
    assert st["kernel"] == "dense_jump"
    if variant:
        assert st["variant"] == variant
    per = _per_sweep(betas, mcs)
    for r0 in (0, 2048, R - 64):
        ref = O.replay_sa_batch([A], [64], s0[r0:r0 + 64].ravel(), per, 99, rep0=r0).reshape(64, n)
        np.testing.assert_array_equal(s[r0:r0 + 64], ref, err_msg=f"replicas {r0}..{r0 + 63}")
        np.testing.assert_allclose(e[r0:r0 + 64], O.energies(g, ref), rtol=0, atol=1e-9)
    assert np.mean(s != s0) > 0.2  # the hot phase: many flips
    dg.close()


# ---- config 5: 512 uneven N(0,1) QUBOs, 32 reads each, batched kernel -----------

@pytest.fixture(scope="module")
def uneven_batch():
    mats = [q.toarray() for q, _ in I.uneven_qubo_batch(512, 64, 1024, seed=5)]
    return mats


@pytest.mark.parametrize("variant", [None, 82, 45, 321])
def test_uneven_batch_512x32_sample(ctx, monkeypatch, uneven_batch, variant):
    _env(monkeypatch, OJ_BATCH_VARIANT=variant)
    mats = uneven_batch
    reads = np.full(len(mats), 32, np.int32)
    sizes = np.array([q.shape[0] - 1 for q in mats])
    soff = np.concatenate([[0], np.cumsum(reads * sizes)])
    bf, mf = I.geometric_betas(0.1, 10.0, 500)
    betas, mcs = bf[:5], mf[:5]
    per = _per_sweep(betas, mcs)
    s0 = _init(int(soff[-1]), 24)
    b = N.Batch(ctx, mats)
    s = s0.copy()
    e = np.zeros(int(reads.sum()))
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=5, energies=e)
    if variant:
        assert st["variant"] == variant
    for k in range(0, len(mats), 16):  # 32 instances across the longest-first queue
        lo, hi = int(soff[k]), int(soff[k + 1])
        ref = O.replay_sa_batch([mats[k]], [32], s0[lo:hi], per, 5, inst0=k)
        np.testing.assert_array_equal(s[lo:hi], ref, err_msg=f"instance {k} (n = {sizes[k]})")
        gk = O.AugCSR(mats[k])
        want = O.energies(gk, ref.reshape(32, sizes[k]))
        np.testing.assert_allclose(e[32 * k:32 * k + 32], want, rtol=1e-12, atol=1e-9)
    b.close()


# ---- statistics on the benchmark lattice ----------------------------------------

def test_lattice_L128_equilibrium_matches_reference(ctx):
    """At a fixed temperature the energy per spin of the bit-packed kernel's
    1024 replicas and of the reference's CPU path (FP64, Xorshift, sequential
    order; 64 reads) agree: the checkerboard order changes the dynamics, not
    the equilibrium."""
    m, _ = I.lattice_pm_j(128, seed=2)
    g = O.AugCSR(m)
    beta, S = 0.44, 300
    betas, mcs = np.array([beta]), np.array([S], np.int32)
    R = 1024
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    s = _init((R, g.n), 25)
    e_gpu = np.zeros(R)
    N.sa_run(dg, s, betas, mcs, seed=31, kernel="bitpacked", energies=e_gpu)
    reads = 64
    init = _init((reads, g.n), 26)
    ref = O.ref_sa_many(g, init, betas, mcs, np.arange(1, reads + 1, dtype=np.uint64),
                        threads=os.cpu_count())
    e_ref = O.energies(g, ref)
    a, b = e_gpu / g.n, e_ref / g.n
    # difference of means against the combined standard error
    se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    assert abs(a.mean() - b.mean()) < 5.0 * se + 1e-4, (a.mean(), b.mean(), se)
    from scipy.stats import ks_2samp
    assert ks_2samp(a, b).pvalue > 1e-4
    dg.close()


def test_sqa_3regular_N4096_equilibrium_matches_reference(ctx):
    """The SQA benchmark instance (3-regular, n = 4096, T = 32) at a fixed point
    of the schedule (beta = 10, Gamma = 1, s = 0.3): the slice-split kernel's
    256 replicas and 64 reads of the reference's CPU path (FP64, Xorshift,
    slice-parity groups, sequential sites) agree in the classical energy per
    spin averaged over the slices; the update order changes the dynamics, not
    the equilibrium of the Trotter system."""
    m, _ = I.random_regular_pm_j(4096, 3, seed=4)
    g = O.AugCSR(m)
    T, S = 32, 300
    betas, ss, mcs = np.array([10.0]), np.array([0.3]), np.array([S], np.int32)
    R = 256
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    s = _init((R, T, g.n), 41)
    e_gpu = np.zeros((R, T))
    st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=43, kernel="bitpacked", energies=e_gpu)
    assert st["kernel"] == "bitpacked"
    reads = 64
    init = _init((reads, T, g.n), 42)
    ref = O.ref_sqa_many(g, init, 1.0, betas, ss, mcs, np.arange(1, reads + 1, dtype=np.uint64),
                         threads=os.cpu_count())
    e_ref = np.array([O.energies(g, ref[r]) for r in range(reads)])
    a, b = e_gpu.mean(axis=1) / g.n, e_ref.mean(axis=1) / g.n
    se = np.sqrt(a.var(ddof=1) / a.size + b.var(ddof=1) / b.size)
    assert abs(a.mean() - b.mean()) < 5.0 * se + 1e-4, (a.mean(), b.mean(), se)
    from scipy.stats import ks_2samp
    assert ks_2samp(a, b).pvalue > 1e-4
    dg.close()
