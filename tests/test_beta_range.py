"""SASampler's automatic beta range (sa_sampler.py:853-976): the flip
statistics come from the GPU (oj_graph_flip_stats / oj_batch_flip_stats), the
rest is host arithmetic; both are checked against the oracle's restatement of
the reference's numpy procedure."""
import numpy as np
import pytest
import scipy.sparse as sp

import openjij_b200 as oj
import openjij_b200.cxxjij.graph as G
from openjij_b200 import _native as N
from openjij_b200 import instances as I
from openjij_b200.sampler.sa_sampler import _THRESHOLD, _beta_range, _flip_spins, geometric_ising_beta_schedule
from oracle import oracle as O


def _np_stats(J, spins):
    """The reference's matrix-product statistics for spins [n][K]."""
    J = J.toarray() if sp.issparse(J) else J
    quad = (J[:-1, :-1] @ spins.astype(np.float64)) * (-2.0 * spins)
    lin = J[:-1, -1][:, None] * spins
    a = np.abs(J)
    return quad, lin, a[a > _THRESHOLD].min() if np.any(a > _THRESHOLD) else np.inf


def _augs():
    rng = np.random.default_rng(5)
    out = {}
    q = I.dense_qubo_int(120, seed=2)[0]
    out["dense_int"] = q.toarray() if sp.issparse(q) else q
    d = I.dense_ising_uniform(90, seed=3)[0]
    out["dense_real"] = d.toarray() if sp.issparse(d) else d
    out["lattice"] = I.lattice_pm_j(8, seed=1)[0]
    h_only = np.zeros((31, 31))
    h_only[:30, 30] = h_only[30, :30] = rng.choice([-1.0, 2.0], 30)
    h_only[30, 30] = 1.0
    out["fields_only"] = h_only
    big_h = I.lattice_pm_j(6, seed=4)[0].tolil()
    for i in range(36):
        big_h[i, 36] = big_h[36, i] = 9.0
    out["strong_fields"] = big_h.tocsr()
    return out


@pytest.mark.parametrize("name", list(_augs()))
@pytest.mark.parametrize("ends", [(None, None), (None, 5.0), (0.3, None)])
def test_beta_range_host_logic_matches_reference(name, ends):
    """CPU: _flip_spins + _beta_range on numpy statistics equal the oracle."""
    J = _augs()[name]
    bmin, bmax = ends
    for S in (10, 1000, 5000):
        np.random.seed(7)
        spins = _flip_spins(J.shape[0])
        got = _beta_range(*_np_stats(J, spins), J.shape[0], S, bmin, bmax)
        want = O.beta_range_reference(J, beta_max=bmax, beta_min=bmin, num_sweeps=S, seed=7)
        np.testing.assert_allclose(got, want, rtol=1e-13)


def _cxxgraph(J):
    if sp.issparse(J):
        return G.CSRSparse(J)
    g = G.Dense(J.shape[0] - 1)
    g.set_interaction_matrix(J)
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_augs()))
def test_flip_stats_kernel(ctx, name):
    J = _augs()[name]
    aug = J if sp.issparse(J) else sp.csr_matrix(J)
    g = N.Graph(ctx, *I.augmented_csr(aug))
    spins = np.random.default_rng(1).choice(np.array([-1, 1], np.int8), size=(J.shape[0] - 1, 3))
    quad, lin, amin = N.flip_stats(g, spins)
    wq, wl, wa = _np_stats(J, spins)
    exact = name != "dense_real"
    np.testing.assert_allclose(quad, wq, rtol=0 if exact else 1e-12, atol=0 if exact else 1e-12)
    np.testing.assert_array_equal(lin, wl)
    assert amin == wa


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_augs()))
@pytest.mark.parametrize("ends", [(None, None), (None, 5.0), (0.3, None)])
def test_geometric_schedule_matches_reference(name, ends):
    J = _augs()[name]
    bmin, bmax = ends
    g = _cxxgraph(J)
    for S in (10, 1000):
        _, got = geometric_ising_beta_schedule(g, beta_max=bmax, beta_min=bmin, num_sweeps=S, seed=11)
        want = O.beta_range_reference(g.get_interactions(), beta_max=bmax, beta_min=bmin, num_sweeps=S, seed=11)
        if name == "dense_real":
            np.testing.assert_allclose(got, want, rtol=1e-12)
        else:
            assert [float(x) for x in got] == [float(x) for x in want]


@pytest.mark.gpu
def test_empty_graph_schedule():
    g = G.Dense(0)
    _, got = geometric_ising_beta_schedule(g, num_sweeps=100, seed=1)
    assert [float(x) for x in got] == [float(x) for x in O.beta_range_reference(g.get_interactions(), num_sweeps=100,
                                                                              seed=1)]


@pytest.mark.gpu
def test_batch_flip_stats_and_sample_batch_range(ctx):
    mats = [I.dense_qubo_normal(n, seed=20 + n)[0].toarray() for n in (5, 64, 200)]
    mats.append(np.eye(1))  # an empty model
    b = N.Batch(ctx, mats)
    rng = np.random.default_rng(2)
    spins = rng.choice(np.array([-1, 1], np.int8), size=(sum(a.shape[0] - 1 for a in mats), 2))
    quad, lin, amin = b.flip_stats(spins)
    pos = 0
    for k, a in enumerate(mats):
        nk = a.shape[0] - 1
        wq, wl, wa = _np_stats(a, spins[pos:pos + nk])
        np.testing.assert_allclose(quad[pos:pos + nk], wq, rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(lin[pos:pos + nk], wl)
        assert amin[k] == wa
        pos += nk
    models = [{(i, j): float(a[i, j]) for i in range(a.shape[0] - 1) for j in range(i, a.shape[0] - 1)
               if a[i, j] != 0} for a in mats[:3]]
    res = oj.SASampler().sample_batch(models, num_sweeps=50, num_reads=2, seed=4)
    ranges = []
    for m in models:
        bqm = oj.BinaryQuadraticModel.from_qubo(m)
        graph, _ = bqm.get_cxxjij_ising_graph()
        ranges.append(O.beta_range_reference(graph.get_interactions(), num_sweeps=50, seed=4))
    sched = res[0].info["schedule"]
    np.testing.assert_allclose(sched["beta_max"], max(r[0] for r in ranges), rtol=1e-12)
    np.testing.assert_allclose(sched["beta_min"], min(r[1] for r in ranges), rtol=1e-12)
