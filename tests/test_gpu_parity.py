"""Spin-for-spin parity of every sweep kernel with the oracle's replay, through
the C ABI (libojb200.so).  Integer and real couplings alike: the kernels and
the replay perform the same FP32 operations in the same order."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _graph(ctx, m):
    g = O.AugCSR(m)
    return g, N.Graph(ctx, g.n, g.indptr, g.indices, g.data)


def _init(R, n, seed):
    rng = np.random.default_rng(seed)
    return rng.choice(np.array([-1, 1], np.int8), size=(R, n))


def _per_sweep(betas, mcs):
    return np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)


@pytest.mark.parametrize("R", [1, 5, 8])
def test_sa_colour_lattice_bit_exact(ctx, R):
    m, _ = I.lattice_pm_j(8, seed=11)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 5.0, 40)
    s0 = _init(R, g.n, 1)
    s = s0.copy()
    st = N.sa_run(dg, s, betas, mcs, seed=1234, kernel="colour")
    assert st["kernel"] == "colour"
    ref = O.replay_sa(g, s0, _per_sweep(betas, mcs), 1234, mode="colour")
    np.testing.assert_array_equal(s, ref)


def test_sa_colour_real_sparse_bit_exact(ctx):
    rng = np.random.default_rng(3)
    n = 60
    J = np.triu(rng.uniform(-1, 1, (n, n)) * (rng.random((n, n)) < 0.1), 1)
    h = rng.uniform(-1, 1, n)
    A = I.dense_augmented(J + J.T, h)
    g, dg = _graph(ctx, A)
    betas, mcs = I.geometric_betas(0.1, 10.0, 30)
    s0 = _init(7, n, 2)
    s = s0.copy()
    N.sa_run(dg, s, betas, mcs, seed=99, kernel="colour")
    ref = O.replay_sa(g, s0, _per_sweep(betas, mcs), 99, mode="colour")
    np.testing.assert_array_equal(s, ref)


@pytest.mark.parametrize("n,R", [(40, 6), (100, 3), (33, 9)])
def test_sa_dense_plain_bit_exact(ctx, n, R):
    m, _ = I.dense_ising_uniform(n, seed=n)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 10.0, 25)
    s0 = _init(R, n, 5)
    s = s0.copy()
    st = N.sa_run(dg, s, betas, mcs, seed=77, kernel="dense_plain")
    assert st["kernel"] == "dense_plain"
    ref = O.replay_sa(g, s0, _per_sweep(betas, mcs), 77, mode="dense")
    np.testing.assert_array_equal(s, ref)


@pytest.mark.parametrize("maker,R", [(lambda: I.lattice_pm_j(16, seed=2), 64),
                                     (lambda: I.lattice_pm_j(12, seed=3), 40),
                                     (lambda: I.random_regular_pm_j(96, 3, seed=4), 32)])
def test_sa_bitpacked_bit_exact(ctx, maker, R):
    m, _ = maker()
    g, dg = _graph(ctx, m)
    info = dg.info()
    assert info["bimodal"] == 1
    betas, mcs = I.geometric_betas(0.1, 5.0, 30)
    bs = _per_sweep(betas, mcs)
    s0 = _init(R, g.n, 9)
    s = s0.copy()
    st = N.sa_run(dg, s, betas, mcs, seed=2024, kernel="bitpacked")
    assert st["kernel"] == "bitpacked"
    thr, alw = O.msc_thresholds(bs, info["coupling_abs"], info["max_degree"])
    Rp = ((R + 31) // 32) * 32
    s0p = np.ones((Rp, g.n), np.int8)
    s0p[:R] = s0
    ref = O.replay_sa_msc(g, s0p, thr, alw, 2024)[:R]
    np.testing.assert_array_equal(s, ref)


@pytest.mark.parametrize("T", [8, 5, 2, 33])
def test_sqa_colour_bit_exact(ctx, T):
    m, _ = I.random_regular_pm_j(48, 3, seed=7)
    g, dg = _graph(ctx, m)
    R = 3
    nsched = 20
    ss = np.linspace(0.0, 1.0, nsched)
    betas = np.full(nsched, 10.0)
    mcs = np.ones(nsched, np.int32)
    s0 = np.ascontiguousarray(np.broadcast_to(_init(R, g.n, 4)[:, None, :], (R, T, g.n)))
    s = s0.copy()
    best = np.zeros(R, np.int32)
    en = np.zeros((R, T))
    st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=5, energies=en, best=best, kernel="colour")
    assert st["kernel"] == "colour"
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    ref = O.replay_sqa(g, s0, a, b, 5)
    np.testing.assert_array_equal(s, ref)
    for r in range(R):
        e = O.energies(g, ref[r])
        np.testing.assert_allclose(en[r], e, rtol=0, atol=1e-9)
        assert best[r] == int(np.argmin(e))


def test_energy_matches_oracle(ctx):
    m, _ = I.dense_ising_uniform(50, seed=8)
    g, dg = _graph(ctx, m)
    s = _init(11, 50, 3)
    e = N.energy(dg, s)
    ref = O.energies(g, s)
    np.testing.assert_allclose(e, ref, rtol=1e-12, atol=1e-12)


def test_zero_sweeps_and_empty(ctx):
    m, _ = I.lattice_pm_j(4, seed=1)
    g, dg = _graph(ctx, m)
    s0 = _init(3, g.n, 1)
    s = s0.copy()
    N.sa_run(dg, s, np.zeros(0), np.zeros(0, np.int32), seed=1)
    np.testing.assert_array_equal(s, s0)
    s = np.zeros((0, g.n), np.int8)
    N.sa_run(dg, s, [1.0], [1], seed=1)


def test_bitpacked_rejects_non_bimodal(ctx):
    m, _ = I.dense_ising_uniform(10, seed=1)
    g, dg = _graph(ctx, m)
    s = _init(2, 10, 1)
    with pytest.raises(N.OJError) as ei:
        N.sa_run(dg, s, [1.0], [1], seed=1, kernel="bitpacked")
    assert ei.value.status == N.OJ_ERR_UNSUPPORTED


def test_sqa_rejects_one_slice(ctx):
    m, _ = I.lattice_pm_j(4, seed=1)
    g, dg = _graph(ctx, m)
    s = np.ones((1, 1, g.n), np.int8)
    with pytest.raises(N.OJError) as ei:
        N.sqa_run(dg, s, 1.0, [1.0], [0.5], [1], seed=1)
    assert ei.value.status == N.OJ_ERR_ARG


@pytest.mark.parametrize("kernel,maker", [
    ("bitpacked", lambda: I.lattice_pm_j(16, seed=5)),
    ("colour", lambda: I.lattice_pm_j(8, seed=6)),
    ("dense_plain", lambda: I.dense_ising_uniform(30, seed=7)),
])
def test_split_run_equals_single_run(ctx, kernel, maker):
    """A schedule run in two calls (first_sweep = sweeps of the first call)
    reproduces the one-call run bit for bit."""
    m, _ = maker()
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 5.0, 24)
    s0 = _init(64, g.n, 3)
    whole = s0.copy()
    N.sa_run(dg, whole, betas, mcs, seed=11, kernel=kernel)
    part = s0.copy()
    N.sa_run(dg, part, betas[:10], mcs[:10], seed=11, kernel=kernel)
    N.sa_run(dg, part, betas[10:], mcs[10:], seed=11, kernel=kernel, first_sweep=int(np.sum(mcs[:10])))
    np.testing.assert_array_equal(part, whole)


@pytest.mark.parametrize("kernel", ["bitpacked", "colour", "dense_plain"])
def test_replica_shards_equal_whole(ctx, kernel):
    """Replicas [32, 96) run alone with replica_offset=32 equal the same
    replicas of a 96-replica run: results do not depend on the sharding."""
    m, _ = I.lattice_pm_j(8, seed=8) if kernel != "dense_plain" else I.dense_ising_uniform(20, seed=8)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 5.0, 12)
    s0 = _init(96, g.n, 4)
    whole = s0.copy()
    N.sa_run(dg, whole, betas, mcs, seed=21, kernel=kernel)
    shard = s0[32:].copy()
    N.sa_run(dg, shard, betas, mcs, seed=21, kernel=kernel, replica_offset=32)
    np.testing.assert_array_equal(shard, whole[32:])


def _scaled(m, c):
    m = m.tocsr(copy=True) * c
    m[m.shape[0] - 1, m.shape[0] - 1] = 1.0
    return m


def _sqa_bitpacked_replay(g, s0, betas, ss, mcs, c, D, seed):
    """Even T: slice-split layout; odd T: one replica per word."""
    T = s0.shape[1]
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    thr, mode = O.sqa_msc_thresholds(np.repeat(a, mcs), np.repeat(b, mcs), c, D)
    if T % 2 == 0:
        return O.replay_sqa_split(g, s0, thr, mode, seed)
    return O.replay_sqa_msc(g, s0, thr, mode, seed)


@pytest.mark.parametrize("T,R", [(2, 3), (2, 40), (5, 3), (10, 9), (31, 3), (32, 3), (64, 2)])
@pytest.mark.parametrize("which", ["regular3", "lattice", "regular5_real"])
def test_sqa_bitpacked_bit_exact(ctx, T, R, which):
    """Bit-packed SQA against its replay (even T: even / odd slices of several
    replicas in two words; odd T: the slices of one replica in one word), with
    a schedule ending at s = 1 (B = -inf: NaN and +-inf energy differences)."""
    if which == "regular3":
        m, c, D = I.random_regular_pm_j(48, 3, seed=7)[0], 1.0, 3
    elif which == "lattice":
        m, c, D = I.lattice_pm_j(8, seed=3)[0], 1.0, 4
    else:
        m, c, D = _scaled(I.random_regular_pm_j(60, 5, seed=2)[0], 0.37), 0.37, 5
    g, dg = _graph(ctx, m)
    nsched = 16
    ss = np.linspace(0.0, 1.0, nsched)
    betas = np.full(nsched, 6.0)
    mcs = np.where(np.arange(nsched) % 3 == 0, 2, 1).astype(np.int32)
    s0 = np.ascontiguousarray(np.broadcast_to(_init(R, g.n, 4)[:, None, :], (R, T, g.n)))
    s0 = s0.copy()
    s0[:, T // 2, :] = _init(R, g.n, 8)
    s = s0.copy()
    best = np.zeros(R, np.int32)
    en = np.zeros((R, T))
    st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=9, energies=en, best=best, kernel="bitpacked")
    assert st["kernel"] == "bitpacked"
    ref = _sqa_bitpacked_replay(g, s0, betas, ss, mcs, c, D, 9)
    np.testing.assert_array_equal(s, ref)
    for r in range(R):
        e = O.energies(g, ref[r])
        np.testing.assert_allclose(en[r], e, rtol=0, atol=1e-9)
        # real couplings: equal-energy slices may differ in the last bits, so the
        # first minimum is taken over the kernel's own energies
        assert best[r] == int(np.argmin(en[r]))
        assert e[best[r]] == pytest.approx(e.min(), abs=1e-9)


def _trotter_dominated(mode, D):
    """Per sweep: no live class with no aligned Trotter neighbour, and none with
    one aligned neighbour and u >= ceil(D/2) (the slice-split kernel's shorter
    threshold-plane evaluation applies)."""
    bad = 0
    for u in range(D + 1):
        bad |= 1 << (3 * u)
        if u >= (D + 1) // 2:
            bad |= 1 << (3 * u + 1)
    live = np.asarray(mode).reshape(-1, 2)[:, 1]
    return [(int(v) & bad) == 0 for v in live]


@pytest.mark.parametrize("which,T,beta", [("regular3", 4, 10.0), ("lattice", 8, 20.0), ("regular3", 32, 10.0)])
def test_sqa_slice_split_both_threshold_evaluations(ctx, which, T, beta):
    """Sweeps where the Trotter term makes every class without an aligned
    Trotter neighbour accept (the kernel then reads the threshold planes from
    fewer table words) and sweeps where it does not, in one run: the replay's
    spins either way."""
    if which == "lattice":
        m, D = I.lattice_pm_j(24, seed=14)[0], 4
    else:
        m, D = I.random_regular_pm_j(600, 3, seed=15)[0], 3
    g, dg = _graph(ctx, m)
    nsched = 12
    ss = np.concatenate([np.linspace(0.0, 0.9, nsched // 2), np.linspace(0.95, 0.0, nsched // 2)])
    betas = np.full(nsched, beta)
    mcs = np.ones(nsched, np.int32)
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    _, mode = O.sqa_msc_thresholds(a, b, 1.0, D)
    dom = _trotter_dominated(mode, D)
    if T < 32:
        assert any(dom) and not all(dom), dom
    s0 = np.random.default_rng(8).choice(np.array([-1, 1], np.int8), size=(9, T, g.n))
    s = s0.copy()
    st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=17, kernel="bitpacked")
    assert st["kernel"] == "bitpacked"
    np.testing.assert_array_equal(s, _sqa_bitpacked_replay(g, s0, betas, ss, mcs, 1.0, D, 17))


@pytest.mark.parametrize("cluster", [None, "3", "16"])
@pytest.mark.parametrize("which,T,R", [("lattice", 16, 4), ("regular3", 8, 20), ("regular3", 32, 6)])
def test_sqa_slice_split_clusters(ctx, monkeypatch, cluster, which, T, R):
    """Sites split over the CTAs of a cluster (halo refresh through distributed
    shared memory) give the replay's spins."""
    if cluster:
        monkeypatch.setenv("OJ_SQA_CLUSTER", cluster)
    if which == "lattice":
        m, D = I.lattice_pm_j(32, seed=12)[0], 4
    else:
        m, D = I.random_regular_pm_j(1200, 3, seed=13)[0], 3
    g, dg = _graph(ctx, m)
    nsched = 10
    ss = np.linspace(0.0, 0.9, nsched)
    betas = np.full(nsched, 4.0)
    mcs = np.ones(nsched, np.int32)
    s0 = np.random.default_rng(3).choice(np.array([-1, 1], np.int8), size=(R, T, g.n))
    s = s0.copy()
    st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=21, kernel="bitpacked")
    assert st["kernel"] == "bitpacked"
    np.testing.assert_array_equal(s, _sqa_bitpacked_replay(g, s0, betas, ss, mcs, 1.0, D, 21))


@pytest.mark.parametrize("R", [16, 37])
def test_sqa_slice_split_two_halves_equal_one_pass(ctx, monkeypatch, R):
    """Host buffers: the replica groups annealed in two halves on two streams
    (each half's copies overlapping the other's kernel) give the spins,
    energies and best slices of the single pass (OJ_PIPE=0), an even and an
    odd number of groups with a partial last group among them."""
    m, _ = I.random_regular_pm_j(1200, 3, seed=16)
    g, dg = _graph(ctx, m)
    T, nsched = 8, 10
    ss = np.linspace(0.0, 0.9, nsched)
    betas = np.full(nsched, 4.0)
    mcs = np.ones(nsched, np.int32)
    s0 = np.random.default_rng(5).choice(np.array([-1, 1], np.int8), size=(R, T, g.n))
    out = []
    for pipe in (None, "0"):
        if pipe:
            monkeypatch.setenv("OJ_PIPE", pipe)
        else:
            monkeypatch.delenv("OJ_PIPE", raising=False)
        s, en, best = s0.copy(), np.zeros((R, T)), np.full(R, -1, np.int32)
        st = N.sqa_run(dg, s, 1.0, betas, ss, mcs, seed=23, energies=en, best=best, kernel="bitpacked")
        assert st["kernel"] == "bitpacked"
        out.append((s, en, best))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(out[0][0], _sqa_bitpacked_replay(g, s0, betas, ss, mcs, 1.0, 3, 23))


def test_sqa_auto_picks_bitpacked_on_regular_pm_j(ctx):
    m, _ = I.random_regular_pm_j(40, 3, seed=1)
    g, dg = _graph(ctx, m)
    s = np.ones((2, 8, g.n), np.int8)
    assert N.sqa_run(dg, s, 1.0, [5.0], [0.5], [1], seed=1)["kernel"] == "bitpacked"
    s = np.ones((2, 33, g.n), np.int8)
    assert N.sqa_run(dg, s, 1.0, [5.0], [0.5], [1], seed=1)["kernel"] == "colour"
    with pytest.raises(N.OJError) as ei:
        N.sqa_run(dg, s, 1.0, [5.0], [0.5], [1], seed=1, kernel="bitpacked")
    assert ei.value.status == N.OJ_ERR_UNSUPPORTED


@pytest.mark.parametrize("kernel", ["bitpacked", "colour"])
def test_sqa_split_and_shard(ctx, kernel):
    m, _ = I.random_regular_pm_j(40, 3, seed=9)
    g, dg = _graph(ctx, m)
    T, nsched = (6 if kernel == "bitpacked" else 5), 12
    ss = np.linspace(0.0, 1.0, nsched)
    betas = np.full(nsched, 8.0)
    mcs = np.ones(nsched, np.int32)
    s0 = np.ascontiguousarray(np.broadcast_to(_init(64, g.n, 5)[:, None, :], (64, T, g.n)))
    whole = s0.copy()
    N.sqa_run(dg, whole, 1.0, betas, ss, mcs, seed=3, kernel=kernel)
    part = s0[32:].copy()
    N.sqa_run(dg, part, 1.0, betas[:5], ss[:5], mcs[:5], seed=3, replica_offset=32, kernel=kernel)
    N.sqa_run(dg, part, 1.0, betas[5:], ss[5:], mcs[5:], seed=3, replica_offset=32, first_sweep=5,
              kernel=kernel)
    np.testing.assert_array_equal(part, whole[32:])


def test_replica_offset_must_be_multiple_of_32(ctx):
    m, _ = I.lattice_pm_j(4, seed=1)
    g, dg = _graph(ctx, m)
    s = _init(4, g.n, 1)
    with pytest.raises(N.OJError) as ei:
        N.sa_run(dg, s, [1.0], [1], seed=1, replica_offset=5)
    assert ei.value.status == N.OJ_ERR_ARG


@pytest.mark.parametrize("n,R", [(200, 128), (700, 130), (1100, 64)])
def test_sa_dense_tc_bit_exact_integer(ctx, n, R):
    """Tensor-core delayed updates: for half-integer couplings every product and
    sum is exact, so the trajectory equals the sequential replay spin for spin."""
    m, _ = I.dense_qubo_int(n, seed=n)
    g, dg = _graph(ctx, m)
    assert dg.info()["integer_exact"] == 1
    betas, mcs = I.geometric_betas(0.05, 5.0, 12)
    s0 = _init(R, n, 3)
    s = s0.copy()
    st = N.sa_run(dg, s, betas, mcs, seed=4242, kernel="dense_tc")
    assert st["kernel"] == "dense_tc"
    ref = O.replay_sa(g, s0, _per_sweep(betas, mcs), 4242, mode="dense")
    np.testing.assert_array_equal(s, ref)


def test_sa_dense_tc_equals_plain_integer(ctx):
    m, _ = I.dense_qubo_int(512, seed=9)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.05, 5.0, 30)
    s0 = _init(160, 512, 8)
    a, b = s0.copy(), s0.copy()
    N.sa_run(dg, a, betas, mcs, seed=77, kernel="dense_tc")
    N.sa_run(dg, b, betas, mcs, seed=77, kernel="dense_plain")
    np.testing.assert_array_equal(a, b)


def test_sa_dense_tc_real_couplings_statistics(ctx):
    """Real couplings: the BF16 hi/lo split is not exact, so trajectories may
    part from the FP32 plain kernel after a near-tie; the final-energy
    distributions must agree (two-sample comparison of the means)."""
    m, _ = I.dense_qubo_normal(300, seed=11)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 10.0, 60)
    s0 = _init(256, 300, 2)
    a, b = s0.copy(), s0.copy()
    ea, eb = np.zeros(256), np.zeros(256)
    N.sa_run(dg, a, betas, mcs, seed=5, kernel="dense_tc", energies=ea)
    N.sa_run(dg, b, betas, mcs, seed=6, kernel="dense_plain", energies=eb)
    se = np.sqrt(ea.var() / len(ea) + eb.var() / len(eb))
    assert abs(ea.mean() - eb.mean()) < 4 * se + 1e-9
    np.testing.assert_allclose(ea, O.energies(g, a), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("which", ["lattice", "regular_h", "sparse_real"])
def test_swendsen_wang_bit_exact(ctx, which):
    """oj_sw_run against its replay: bonds, clusters (union-find) and cluster
    coins; with fields (bonds to the dummy spin) and real couplings."""
    if which == "lattice":
        m = I.lattice_pm_j(16, seed=4)[0]
    elif which == "regular_h":
        m = I.random_regular_pm_j(300, 3, seed=5)[0].tolil()
        rng = np.random.default_rng(1)
        n = m.shape[0] - 1
        for i in range(0, n, 3):
            m[i, n] = m[n, i] = float(rng.choice([-0.5, 0.7]))
        m = m.tocsr()
    else:
        m, _ = I.dense_ising_uniform(60, seed=9)
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.1, 3.0, 12)
    s0 = _init(40, g.n, 7)
    s = s0.copy()
    e = np.zeros(40)
    st = N.sw_run(dg, s, betas, mcs, seed=19, energies=e)
    assert st["kernel"] == "swendsen_wang"
    ref = O.replay_sw(g, s0, _per_sweep(betas, mcs), 19)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_allclose(e, O.energies(g, ref), rtol=1e-12, atol=1e-9)


def test_swendsen_wang_split_run(ctx):
    m = I.lattice_pm_j(8, seed=2)[0]
    g, dg = _graph(ctx, m)
    betas, mcs = I.geometric_betas(0.2, 2.0, 10)
    s0 = _init(64, g.n, 3)
    whole = s0.copy()
    N.sw_run(dg, whole, betas, mcs, seed=4)
    part = s0[32:].copy()
    N.sw_run(dg, part, betas[:4], mcs[:4], seed=4, replica_offset=32)
    N.sw_run(dg, part, betas[4:], mcs[4:], seed=4, replica_offset=32, first_sweep=int(np.sum(mcs[:4])))
    np.testing.assert_array_equal(part, whole[32:])


def test_swendsen_wang_large_graph_global_forest(ctx):
    """Above the shared-memory size (n > 45,000) the forest lives in global
    scratch; same bonds, clusters and coins as the replay."""
    m = I.lattice_pm_j(224, seed=6)[0]
    g, dg = _graph(ctx, m)
    assert g.n > 45000
    betas, mcs = I.geometric_betas(0.2, 1.5, 3)
    s0 = _init(3, g.n, 8)
    s = s0.copy()
    N.sw_run(dg, s, betas, mcs, seed=21)
    np.testing.assert_array_equal(s, O.replay_sw(g, s0, _per_sweep(betas, mcs), 21))


def test_graph_validation(ctx):
    """Graph upload: an asymmetric matrix, a non-zero diagonal and a corner
    other than 1 are refused; unsorted rows and repeated entries (summed, as
    scipy does) are taken."""
    def csr(rows, n):
        indptr, indices, data = [0], [], []
        for r in rows:
            for j, v in r:
                indices.append(j)
                data.append(v)
            indptr.append(len(indices))
        return (n, np.array(indptr, np.int64), np.array(indices, np.int32), np.array(data, np.float64))
    good = [[(2, 0.5), (1, -1.0)], [(0, -1.0), (2, 0.5), (2, 0.5)], [(1, 1.0), (0, 0.5)], [(3, 1.0)]]
    g = N.Graph(ctx, *csr(good, 3))
    assert g.info()["nnz"] == 6
    for bad in ([[(1, -1.0)], [(0, -2.0)], [], [(3, 1.0)]],  # J_01 != J_10
                [[(0, 1.0)], [], [], [(3, 1.0)]],             # diagonal
                [[], [], [], [(3, 2.0)]]):                    # corner
        with pytest.raises(N.OJError) as ei:
            N.Graph(ctx, *csr(bad, 3))
        assert ei.value.status == N.OJ_ERR_ARG
