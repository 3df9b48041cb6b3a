"""Per-call accepted-flip counts (oj_run_stats.accepted) of every
single-spin-flip kernel.  In one sweep each site (each site and slice, for
SQA) is visited once, so the count of a one-sweep call equals the number of
spins that differ from the initial state; over more sweeps it is at least
that."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I

pytestmark = pytest.mark.gpu


def _init(shape, seed):
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=shape)


@pytest.mark.parametrize("kernel,maker,R", [
    ("bitpacked", lambda: I.lattice_pm_j(32, seed=2), 64),
    ("colour", lambda: I.lattice_pm_j(16, seed=2), 7),
    ("colour", lambda: I.dense_ising_uniform(60, seed=3), 5),
    ("dense_plain", lambda: I.dense_ising_uniform(200, seed=3), 9),
    ("dense_jump", lambda: I.dense_qubo_int(300, seed=3), 40),
    ("dense_tc", lambda: I.dense_qubo_int(256, seed=3), 130),
])
def test_sa_accepted_flips_one_sweep(ctx, kernel, maker, R):
    m, _ = maker()
    g = N.Graph(ctx, *I.augmented_csr(m))
    for beta in (0.05, 0.8):
        s0 = _init((R, g.n), 3)
        s = s0.copy()
        st = N.sa_run(g, s, [beta], [1], seed=11, kernel=kernel)
        assert st["kernel"] == kernel
        assert st["accepted"] == np.count_nonzero(s != s0)
    s = s0.copy()
    st = N.sa_run(g, s, [0.1, 1.0, 3.0], [2, 2, 2], seed=12, kernel=kernel)
    assert st["accepted"] >= np.count_nonzero(s != s0)


@pytest.mark.parametrize("kernel,T", [("bitpacked", 8), ("bitpacked", 5), ("colour", 6)])
def test_sqa_accepted_flips_one_sweep(ctx, kernel, T):
    m, _ = I.random_regular_pm_j(256, 3, seed=7)
    g = N.Graph(ctx, *I.augmented_csr(m))
    R = 8 if kernel == "bitpacked" and T == 8 else 3  # slice-split groups of 8 replicas at T = 8
    t0 = _init((R, T, g.n), 4)
    t = t0.copy()
    st = N.sqa_run(g, t, 1.0, [2.0], [0.5], [1], seed=5, kernel=kernel)
    assert st["accepted"] == np.count_nonzero(t != t0)


def test_batched_accepted_flips_one_sweep(ctx):
    mats = [I.dense_qubo_normal(k, seed=k)[0].toarray() for k in (40, 130, 300)]
    reads = [3, 5, 8]
    total = sum(r * (a.shape[0] - 1) for r, a in zip(reads, mats))
    s0 = _init(total, 6)
    s = s0.copy()
    st = N.sa_run_batched(N.Batch(ctx, mats), reads, s, [0.3], [1], seed=9)
    assert st["accepted"] == np.count_nonzero(s != s0)


def test_swendsen_wang_reports_no_count(ctx):
    m, _ = I.lattice_pm_j(8, seed=2)
    g = N.Graph(ctx, *I.augmented_csr(m))
    st = N.sw_run(g, _init((2, g.n), 1), [0.5], [2], seed=1)
    assert st["accepted"] == -1.0
