"""The tensor-core kernel of the flip-heavy first sweeps (oj_k_hot_tc.cu).

Exact one-digit batches (integer couplings) start every call in it: the
replicas of a 32-replica tile decide a 128-site chunk in lock step and the
chunk's spin changes reach all fields as int8 MMAs; a tile hands its spins and
fields to the dense-jump / batched sweep kernel after the first sweep with
fewer flips per replica than a floor (OJ_HOT_FLOOR, default n/16).  Whatever the
hand-over sweep, the spins, energies and accepted-flip counts must be the
replay's (the sequential sweep of the jump kernel,
include/openjij/updater/single_spin_flip.hpp:66-95, with its uniforms).
OJ_HOT_FLOOR=0 keeps every tile in the tensor-core kernel for the whole call,
a huge floor makes every tile leave after its first sweep, OJ_HOT=0 disables it.
"""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FLOORS = [None, "0", "40", "1000000"]


def _per_sweep(betas, mcs):
    return np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)


def _set_floor(monkeypatch, floor):
    if floor is None:
        monkeypatch.delenv("OJ_HOT_FLOOR", raising=False)
    else:
        monkeypatch.setenv("OJ_HOT_FLOOR", floor)


@pytest.mark.parametrize("floor", FLOORS)
def test_dense_jump_hot_sweeps_match_replay(ctx, monkeypatch, floor):
    """n = 300 (three chunks, the last ragged), 40 replicas (a full and a
    partial 32-replica tile), 24 sweeps from a random state."""
    _set_floor(monkeypatch, floor)
    m, _ = I.dense_qubo_int(300, seed=11)
    A = m.toarray()
    g = O.AugCSR(m)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.05, 4.0, 24)
    R = 40
    s0 = np.random.default_rng(2).choice(np.array([-1, 1], np.int8), size=(R, g.n))
    s = s0.copy()
    e = np.zeros(R)
    st = N.sa_run(dg, s, betas, mcs, seed=21, kernel="dense_jump", energies=e)
    want = O.replay_sa_batch([A], [R], s0.ravel(), _per_sweep(betas, mcs), 21).reshape(R, g.n)
    np.testing.assert_array_equal(s, want)
    np.testing.assert_allclose(e, O.energies(g, want), rtol=0, atol=1e-9)
    monkeypatch.setenv("OJ_HOT", "0")
    s2 = s0.copy()
    st2 = N.sa_run(dg, s2, betas, mcs, seed=21, kernel="dense_jump")
    np.testing.assert_array_equal(s2, want)
    assert st["accepted"] == st2["accepted"] > 0


@pytest.mark.parametrize("floor", FLOORS)
def test_batched_mixed_sizes_hot_sweeps_match_replay(ctx, monkeypatch, floor):
    """Instances with one chunk (no tensor-core sweeps), 2..16 chunks and more
    than 16 chunks (no tensor-core sweeps) in one exact batch."""
    _set_floor(monkeypatch, floor)
    sizes = [100, 130, 700, 2048, 2200]
    reads = [3, 40, 33, 5, 2]
    mats = [I.dense_qubo_int(n, seed=40 + k)[0].toarray() for k, n in enumerate(sizes)]
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.05, 5.0, 12)
    total = sum(r * n for r, n in zip(reads, sizes))
    s0 = np.random.default_rng(5).choice(np.array([-1, 1], np.int8), size=total)
    s = s0.copy()
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=8)
    np.testing.assert_array_equal(s, O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 8))
    assert st["field_drift"] == 0.0


def test_split_call_continues_the_stream(ctx):
    """A run split over two calls (first_sweep) equals the whole run: each call
    starts in the tensor-core kernel at its own global sweep index."""
    m, _ = I.dense_qubo_int(520, seed=12)
    g = O.AugCSR(m)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.05, 4.0, 30)
    s0 = np.random.default_rng(3).choice(np.array([-1, 1], np.int8), size=(64, g.n))
    whole = s0.copy()
    N.sa_run(dg, whole, betas, mcs, seed=5, kernel="dense_jump")
    part = s0.copy()
    N.sa_run(dg, part, betas[:7], mcs[:7], seed=5, kernel="dense_jump")
    N.sa_run(dg, part, betas[7:], mcs[7:], seed=5, kernel="dense_jump", first_sweep=7)
    np.testing.assert_array_equal(part, whole)


def test_hot_sweep_wait_time_out_is_reported():
    """A wait limit of zero makes the bounded waits give up at once: the call
    reports OJ_ERR_TIMEOUT and the context then runs the call correctly."""
    ctx = N.Context(0)
    m, _ = I.dense_qubo_int(260, seed=13)
    A = m.toarray()
    g = O.AugCSR(m)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.1, 3.0, 5)
    s0 = np.random.default_rng(4).choice(np.array([-1, 1], np.int8), size=(33, g.n))
    ctx.set_wait_limit(0)
    with pytest.raises(N.OJError) as ei:
        N.sa_run(dg, s0.copy(), betas, mcs, seed=1, kernel="dense_jump")
    assert ei.value.status == N.OJ_ERR_TIMEOUT
    ctx.set_wait_limit(-1)
    s = s0.copy()
    N.sa_run(dg, s, betas, mcs, seed=1, kernel="dense_jump")
    np.testing.assert_array_equal(s, O.replay_sa_batch([A], [33], s0.ravel(), _per_sweep(betas, mcs), 1).reshape(33, g.n))
    ctx.close()
