"""The launch-shape autotuner (OJ_AUTOTUNE): the tuned run gives the same spins
as the default run, the choice is cached for later calls, and the stats report
the shape that ran."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I

pytestmark = pytest.mark.gpu


def _graph(ctx, m):
    return N.Graph(ctx, *I.augmented_csr(m))


def test_tuned_bitpacked_sa_equals_default(ctx):
    m, _ = I.lattice_pm_j(32, seed=3)
    betas, mcs = I.geometric_betas(0.1, 4.0, 40)
    s0 = np.random.default_rng(1).choice(np.array([-1, 1], np.int8), size=(256, 1024))
    plain = s0.copy()
    st0 = N.sa_run(_graph(ctx, m), plain, betas, mcs, seed=8, kernel="bitpacked")
    g = _graph(ctx, m)
    tuned = s0.copy()
    st1 = N.sa_run(g, tuned, betas, mcs, seed=8, kernel="bitpacked", tune=True)
    np.testing.assert_array_equal(tuned, plain)
    assert st0["tuned"] == 0 and st1["tuned"] == 1
    assert st1["cluster"] >= 1 and st1["threads"] in (256, 512, 1024)
    again = s0.copy()
    st2 = N.sa_run(g, again, betas, mcs, seed=8, kernel="bitpacked", tune=True)
    assert st2["tuned"] == 0 and (st2["cluster"], st2["threads"]) == (st1["cluster"], st1["threads"])
    np.testing.assert_array_equal(again, plain)


def test_tuned_slice_split_sqa_equals_default(ctx):
    m, _ = I.random_regular_pm_j(1200, 3, seed=13)
    T, R, nsched = 16, 20, 12
    ss = np.linspace(0.0, 0.9, nsched)
    betas = np.full(nsched, 4.0)
    mcs = np.ones(nsched, np.int32)
    s0 = np.random.default_rng(2).choice(np.array([-1, 1], np.int8), size=(R, T, 1200))
    plain = s0.copy()
    N.sqa_run(_graph(ctx, m), plain, 1.0, betas, ss, mcs, seed=4, kernel="bitpacked")
    tuned = s0.copy()
    st = N.sqa_run(_graph(ctx, m), tuned, 1.0, betas, ss, mcs, seed=4, kernel="bitpacked", tune=True)
    assert st["tuned"] == 1 and st["cluster"] in (1, 2, 4) and st["threads"] in (256, 512)
    np.testing.assert_array_equal(tuned, plain)


def test_tuned_batch_equals_default(ctx):
    mats = [I.dense_qubo_normal(n, seed=80 + k)[0].toarray() for k, n in enumerate((70, 300, 129))]
    reads = [9, 3, 16]
    betas, mcs = I.geometric_betas(0.1, 5.0, 12)
    total = sum(r * (a.shape[0] - 1) for r, a in zip(reads, mats))
    s0 = np.random.default_rng(3).choice(np.array([-1, 1], np.int8), size=total)
    plain = s0.copy()
    N.sa_run_batched(N.Batch(ctx, mats), reads, plain, betas, mcs, seed=6)
    tuned = s0.copy()
    st = N.sa_run_batched(N.Batch(ctx, mats), reads, tuned, betas, mcs, seed=6, tune=True)
    assert st["tuned"] == 1 and st["variant"] in (45, 82, 83, 84, 162, 321)
    np.testing.assert_array_equal(tuned, plain)
