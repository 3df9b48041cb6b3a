"""The tensor-core field kernel (oj_k_field_tc.cu) behind the batched and
dense-jump runs: fields of the initial spins, the full recompute every K
sweeps for couplings whose FP32 sums are not exact, the drift statistic, and
the bounded waits' time-out path.  Everything against the oracle's replay,
which restates the same field definition (integers on a per-instance grid,
one rounding) and recompute points."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _normal_batch(sizes, seed):
    return [I.dense_qubo_normal(int(n), seed=seed + k)[0].toarray() for k, n in enumerate(sizes)]


def _spins(mats, reads, seed):
    total = sum(r * (m.shape[0] - 1) for r, m in zip(reads, mats))
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=total)


def _per_sweep(betas, mcs):
    return np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)


@pytest.mark.parametrize("K", [16, 5, 0])
def test_recompute_and_drift_match_replay(K):
    """N(0,1) couplings, uneven sizes (one and several 128-site tiles, reads
    above and below a replica tile): spins and the drift statistic equal the
    replay's, bit for bit, for recompute intervals 16 (default), 5 and 0."""
    ctx = N.Context(0)
    if K != 16:
        ctx.set_field_recompute(K)
    sizes = [7, 130, 300, 64, 515]
    reads = [3, 40, 9, 17, 2]
    mats = _normal_batch(sizes, 90)
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 8.0, 37)
    s0 = _spins(mats, reads, 4)
    s = s0.copy()
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=13)
    ref, drift = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 13, recompute=K, drift=True)
    np.testing.assert_array_equal(s, ref)
    assert st["field_drift"] == float(drift.max())
    assert 0.0 < st["field_drift"] < 1e-2
    b.close()
    ctx.close()


@pytest.mark.parametrize("K", [16, 5])
def test_one_chunk_batch_recomputes_in_the_sweep_kernel(K):
    """Instances of at most 128 sites run in the one-chunk kernel, which sets
    the fields anew itself (int64 sums of the grid integers) at the same global
    sweeps: spins and drift equal the replay's, and a run split over two calls
    at a multiple of K equals the whole run."""
    ctx = N.Context(0)
    ctx.set_field_recompute(K)
    sizes = [7, 100, 128, 64, 33]
    reads = [3, 40, 9, 17, 70]
    mats = _normal_batch(sizes, 120)
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 8.0, 3 * K + 4)
    s0 = _spins(mats, reads, 9)
    s = s0.copy()
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=31)
    ref, drift = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 31, recompute=K, drift=True)
    np.testing.assert_array_equal(s, ref)
    assert st["field_drift"] == float(drift.max())
    assert 0.0 < st["field_drift"] < 1e-2
    part = s0.copy()
    N.sa_run_batched(b, reads, part, betas[:2 * K], mcs[:2 * K], seed=31)
    N.sa_run_batched(b, reads, part, betas[2 * K:], mcs[2 * K:], seed=31, first_sweep=2 * K)
    np.testing.assert_array_equal(part, ref)
    b.close()
    ctx.close()


def test_dense_jump_n100_real_couplings_drift(ctx):
    """The benchmark's 100-spin dense instance (uniform couplings) on the
    dense-jump path: the one-chunk kernel with its own recompute."""
    m, _ = I.dense_ising_uniform(100, seed=1)
    g = O.AugCSR(m)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.1, 10.0, 70)
    s0 = np.random.default_rng(11).choice(np.array([-1, 1], np.int8), size=(100, g.n))
    s = s0.copy()
    st = N.sa_run(dg, s, betas, mcs, seed=5, kernel="dense_jump")
    ref, drift = O.replay_sa_batch([m.toarray()], [100], s0.ravel(), _per_sweep(betas, mcs), 5, drift=True)
    np.testing.assert_array_equal(s, ref.reshape(100, g.n))
    assert st["field_drift"] == float(drift.max())
    assert st["launches"] <= 4  # no launch per recompute


def test_graph_replay_equals_direct_launches(monkeypatch):
    """A batched run's launches are captured as a CUDA graph and replayed (the
    executable graph kept and updated by the next call, instantiated anew when
    the launch sequence changes): calls of different lengths and seeds in a
    row give the spins, drift and counts of the same calls launched directly
    (OJ_GRAPH=0)."""
    sizes = [90, 300, 140]
    reads = [5, 33, 17]
    mats = _normal_batch(sizes, 210)
    s0 = _spins(mats, reads, 12)
    runs = [(37, 3), (37, 4), (20, 5), (52, 6)]  # sweeps, seed

    def go():
        ctx = N.Context(0)
        b = N.Batch(ctx, mats)
        out = []
        for S, seed in runs:
            betas, mcs = I.geometric_betas(0.1, 8.0, S)
            s = s0.copy()
            st = N.sa_run_batched(b, reads, s, betas, mcs, seed=seed)
            out.append((s, st["field_drift"], st["accepted"]))
        b.close()
        ctx.close()
        return out

    monkeypatch.delenv("OJ_GRAPH", raising=False)
    graph = go()
    monkeypatch.setenv("OJ_GRAPH", "0")
    direct = go()
    for (sg, dg_, ag), (sd, dd, ad), (S, seed) in zip(graph, direct, runs):
        np.testing.assert_array_equal(sg, sd)
        assert dg_ == dd and ag == ad
        betas, mcs = I.geometric_betas(0.1, 8.0, S)
        np.testing.assert_array_equal(sg, O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), seed))


def test_exact_batches_report_no_drift(ctx):
    mats = [I.dense_qubo_int(n, seed=n)[0].toarray() for n in (100, 260)]
    reads = [5, 33]
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 5.0, 40)
    s0 = _spins(mats, reads, 5)
    s = s0.copy()
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=2)
    np.testing.assert_array_equal(s, O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 2))
    assert st["field_drift"] == 0.0


def test_dense_jump_real_couplings_recompute(ctx):
    """The dense-jump kernel (one graph) takes the same recompute: a run split
    over two calls at a multiple of 16 sweeps equals the whole run."""
    m, _ = I.dense_ising_uniform(300, seed=8)
    g = O.AugCSR(m)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.1, 10.0, 48)
    s0 = np.random.default_rng(6).choice(np.array([-1, 1], np.int8), size=(20, g.n))
    whole = s0.copy()
    st = N.sa_run(dg, whole, betas, mcs, seed=3, kernel="dense_jump")
    ref, drift = O.replay_sa_batch([m.toarray()], [20], s0.ravel(), _per_sweep(betas, mcs), 3, drift=True)
    np.testing.assert_array_equal(whole, ref.reshape(20, g.n))
    assert st["field_drift"] == float(drift.max())
    part = s0.copy()
    N.sa_run(dg, part, betas[:32], mcs[:32], seed=3, kernel="dense_jump")
    N.sa_run(dg, part, betas[32:], mcs[32:], seed=3, kernel="dense_jump", first_sweep=32)
    np.testing.assert_array_equal(part, whole)


def test_wait_time_out_is_reported_and_context_recovers():
    """A pipeline wait limit of zero iterations makes the field kernel give up
    at its first wait: it drains its copies, frees its tensor memory and
    returns, the call reports OJ_ERR_TIMEOUT, and the same context then runs
    the same call correctly."""
    ctx = N.Context(0)
    mats = _normal_batch([200, 90], 30)
    reads = [8, 3]
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 5.0, 6)
    s0 = _spins(mats, reads, 7)
    ctx.set_wait_limit(0)
    with pytest.raises(N.OJError) as ei:
        N.sa_run_batched(b, reads, s0.copy(), betas, mcs, seed=1)
    assert ei.value.status == N.OJ_ERR_TIMEOUT
    ctx.set_wait_limit(-1)
    s = s0.copy()
    N.sa_run_batched(b, reads, s, betas, mcs, seed=1)
    np.testing.assert_array_equal(s, O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 1))
    b.close()
    ctx.close()
