"""Statistical agreement of the B200 update schemes with the reference samplers.

The GPU kernels draw their random numbers from Philox and visit the sites in
colour-class (or bit-packed) order, so their runs are not the reference's runs;
the GPU parity tests pin every kernel spin for spin to its CPU replay, and
these tests compare the replays' statistics with the restated reference
(sequential site order, Xorshift, `SASampler` / `SQASampler` semantics), on
the same seeded instances:

* at a fixed temperature, after enough sweeps to equilibrate, the final-energy
  distribution is the Boltzmann distribution whatever the update order, so the
  two histograms must agree (chi-square / Kolmogorov-Smirnov, p > 1e-4);
* under annealing (not at equilibrium) the ground-state hit rates and mean
  final energies must agree within 4 standard errors plus a stated allowance
  for the different visiting order (0.05 in hit rate).

With a seed the reference runs every read from the same state and seed
(sampler.py:103-104); here every read r gets seed + r, as independent reads.
"""
import itertools

import numpy as np
import pytest
from scipy import stats

from openjij_b200 import instances as I
from oracle import oracle as O

P_MIN = 1e-4


def _lattice4():
    return O.AugCSR(I.lattice_pm_j(4, seed=21)[0])


def _ground_energy(g):
    best = np.inf
    n = g.n
    for bits in itertools.product([-1, 1], repeat=n - 1):
        s = np.array((1,) + bits, np.int8)  # global flip symmetry (h = 0)
        best = min(best, O.energy(g, s))
    return best


def _chi2_p(a, b):
    a = np.round(np.asarray(a, np.float64), 6)
    b = np.round(np.asarray(b, np.float64), 6)
    vals = np.union1d(a, b)
    table = np.array([[np.sum(a == v) for v in vals], [np.sum(b == v) for v in vals]])
    keep = table.sum(axis=0) >= 20
    merged = np.column_stack([table[:, keep], table[:, ~keep].sum(axis=1)]) if (~keep).any() else table[:, keep]
    merged = merged[:, merged.sum(axis=0) > 0]
    return stats.chi2_contingency(merged)[1]


def _init(R, n, seed):
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=(R, n))


def _two_prop_ok(k1, n1, k2, n2, allowance):
    p1, p2 = k1 / n1, k2 / n2
    se = np.sqrt(max(p1 * (1 - p1), 1e-4) / n1 + max(p2 * (1 - p2), 1e-4) / n2)
    return abs(p1 - p2) <= allowance + 4 * se, (p1, p2)


@pytest.mark.parametrize("scheme", ["colour", "dense", "bitpacked"])
def test_sa_equilibrium_energy_distribution(scheme):
    g = _lattice4()
    R, S, beta = 4096, 200, 0.6
    s0 = _init(R, g.n, 1)
    ref = O.ref_sa_many(g, s0, [beta], [S], np.arange(R, dtype=np.uint64) + 1000)
    per = np.full(S, beta, np.float32)
    if scheme == "bitpacked":
        thr, alw = O.msc_thresholds(per, 1.0, 4)
        got = O.replay_sa_msc(g, s0, thr, alw, 77)
    else:
        got = O.replay_sa(g, s0, per, 77, mode=scheme)
    p = _chi2_p(O.energies(g, got), O.energies(g, ref))
    assert p > P_MIN, p


def test_sa_equilibrium_real_couplings():
    m, _ = I.dense_ising_uniform(14, seed=31)
    g = O.AugCSR(m)
    R, S, beta = 4000, 200, 1.5
    s0 = _init(R, g.n, 2)
    ref = O.ref_sa_many(g, s0, [beta], [S], np.arange(R, dtype=np.uint64) + 5000)
    per = np.full(S, beta, np.float32)
    for mode in ("colour", "dense"):
        got = O.replay_sa(g, s0, per, 91, mode=mode)
        p = stats.ks_2samp(O.energies(g, got), O.energies(g, ref)).pvalue
        assert p > P_MIN, (mode, p)


@pytest.mark.parametrize("scheme", ["colour", "dense", "bitpacked"])
def test_sa_annealing_ground_state_rate(scheme):
    g = _lattice4()
    e0 = _ground_energy(g)
    R = 2048
    betas, mcs = I.geometric_betas(0.1, 3.0, 12)
    s0 = _init(R, g.n, 3)
    ref = O.ref_sa_many(g, s0, betas, mcs, np.arange(R, dtype=np.uint64) + 11)
    per = np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)
    if scheme == "bitpacked":
        thr, alw = O.msc_thresholds(per, 1.0, 4)
        got = O.replay_sa_msc(g, s0, thr, alw, 5)
    else:
        got = O.replay_sa(g, s0, per, 5, mode=scheme)
    eg, er = O.energies(g, got), O.energies(g, ref)
    ok, rates = _two_prop_ok(np.sum(np.isclose(eg, e0)), R, np.sum(np.isclose(er, e0)), R, 0.05)
    assert ok, rates
    assert 0.02 < rates[1] < 0.98  # the schedule leaves room to differ
    se = np.sqrt(eg.var() / R + er.var() / R)
    assert abs(eg.mean() - er.mean()) <= 0.05 * abs(e0) + 4 * se


def _sqa_replay(scheme, g, s0, gamma, betas, ss, mcs, seed):
    T = s0.shape[1]
    a, b = O.sqa_coefficients(betas, ss, gamma, T)
    a, b = np.repeat(a, mcs), np.repeat(b, mcs)
    if scheme == "colour":
        return O.replay_sqa(g, s0, a, b, seed)
    thr, mode = O.sqa_msc_thresholds(a, b, 1.0, 4)
    if scheme == "bitpacked_slices":
        return O.replay_sqa_split(g, s0, thr, mode, seed)
    return O.replay_sqa_msc(g, s0, thr, mode, seed)


@pytest.mark.parametrize("scheme", ["colour", "bitpacked_word", "bitpacked_slices"])
def test_sqa_equilibrium_slice_energy_distribution(scheme):
    g = _lattice4()
    R, T, S = 2048, 8, 200
    gamma, beta, s = 1.0, 2.0, 0.5
    s0 = np.ascontiguousarray(np.broadcast_to(_init(R, g.n, 4)[:, None, :], (R, T, g.n)))
    ref = O.ref_sqa_many(g, s0, gamma, [beta], [s], [S], np.arange(R, dtype=np.uint64) + 300)
    got = _sqa_replay(scheme, g, s0, gamma, [beta], [s], [S], 17)
    # slice 0 (all slices are equivalent by the periodic Trotter symmetry)
    p = _chi2_p(O.energies(g, got[:, 0, :]), O.energies(g, ref[:, 0, :]))
    assert p > P_MIN, p
    # and the mean classical energy over the slices
    mg = np.array([O.energies(g, x).mean() for x in got])
    mr = np.array([O.energies(g, x).mean() for x in ref])
    assert stats.ks_2samp(mg, mr).pvalue > P_MIN


@pytest.mark.parametrize("scheme", ["colour", "bitpacked_word", "bitpacked_slices"])
def test_sqa_annealing_ground_state_rate(scheme):
    g = _lattice4()
    e0 = _ground_energy(g)
    R, T, S = 1024, 8, 12
    gamma, beta = 1.0, 6.0
    ss = np.linspace(0.0, 1.0, S)
    betas = np.full(S, beta)
    mcs = np.ones(S, np.int64)
    s0 = np.ascontiguousarray(np.broadcast_to(_init(R, g.n, 6)[:, None, :], (R, T, g.n)))
    ref = O.ref_sqa_many(g, s0, gamma, betas, ss, mcs, np.arange(R, dtype=np.uint64) + 900)
    got = _sqa_replay(scheme, g, s0, gamma, betas, ss, mcs.astype(np.int32), 23)

    def best(x):  # get_solution: the first slice of minimum energy
        return np.array([O.energies(g, r).min() for r in x])

    bg, br = best(got), best(ref)
    ok, rates = _two_prop_ok(np.sum(np.isclose(bg, e0)), R, np.sum(np.isclose(br, e0)), R, 0.05)
    assert ok, rates
    assert 0.02 < rates[1] < 0.98


def test_batched_fp32_field_drift_is_stated():
    """The batched / dense-jump kernels update FP32 fields incrementally (one
    rounding per accepted flip) and, for couplings whose FP32 sums are not
    exact, set them anew from the spins on the tensor cores every 16 sweeps
    (the library's default).  Their replay performs the same operations, so its
    fields are the kernel's.  On N(0,1) QUBOs (n = 512 and 1024, 500 sweeps,
    beta 0.1 -> 10), against the FP64 fields of the final spins: without the
    recompute the error grows to about 4e-6 of the field scale; with it the
    final fields are within 2e-7 of the scale (about one FP32 unit in the last
    place), and the largest drift between two recomputes (the hot first
    sweeps) stays below 5e-4 absolute.  Integer couplings: zero."""
    from openjij_b200 import instances as I
    betas, mcs = I.geometric_betas(0.1, 10.0, 500)
    per = np.repeat(betas, mcs).astype(np.float32)
    for integer in (False, True):
        for n in (512, 1024):
            A = (I.dense_qubo_int(n, seed=n) if integer else I.dense_qubo_normal(n, seed=n))[0].toarray()
            R = 4
            s0 = _init(R, n, n)
            A32 = A.astype(np.float32).astype(np.float64)  # the kernel's own inputs
            for K, tol in ((0, 1e-5), (16, 2e-7)):
                s, f32, dr = O.replay_sa_batch([A], [R], s0.ravel(), per, 7, fields=True, drift=True, recompute=K)
                S = s.reshape(R, n).astype(np.float64)
                f64r = A32[:n, n][None, :] + S @ A32[:n, :n]
                err = np.abs(f32.reshape(R, n).astype(np.float64) - f64r).max()
                scale = np.abs(f64r).max()
                if integer:
                    assert err == 0.0 and dr.max() == 0.0, (n, K, err, dr.max())
                    continue
                assert err / scale <= tol, (n, K, err / scale)
                assert dr.max() >= err * (1 - 1e-6) - 1e-5  # the statistic covers the final error
                if K:
                    assert dr.max() <= 5e-4, (n, dr.max())


def test_swendsen_wang_equilibrium_and_annealing():
    """Swendsen-Wang replay against the reference updater (swendsen_wang.hpp):
    the equilibrium energy histogram at a fixed beta, and the ground-state rate
    of a short anneal."""
    g = _lattice4()
    R, S, beta = 4096, 100, 0.6
    s0 = _init(R, g.n, 11)
    ref = O.ref_sw_many(g, s0, [beta], [S], np.arange(R, dtype=np.uint64) + 77)
    got = O.replay_sw(g, s0, np.full(S, beta, np.float32), 5)
    p = _chi2_p(O.energies(g, got), O.energies(g, ref))
    assert p > P_MIN, p
    e0 = _ground_energy(g)
    betas, mcs = I.geometric_betas(0.1, 3.0, 8)
    ref = O.ref_sw_many(g, s0[:2048], betas, mcs, np.arange(2048, dtype=np.uint64) + 3)
    got = O.replay_sw(g, s0[:2048], np.repeat(betas, mcs).astype(np.float32), 6)
    eg, er = O.energies(g, got), O.energies(g, ref)
    ok, rates = _two_prop_ok(np.sum(np.isclose(eg, e0)), 2048, np.sum(np.isclose(er, e0)), 2048, 0.05)
    assert ok, rates
