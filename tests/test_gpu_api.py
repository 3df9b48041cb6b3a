"""The reference-facing API on the GPU: cxxjij bindings (after the reference's
tests/test_cxx.py) and the samplers (after tests/test_sampler.py), plus
end-to-end parity of the sampler path with the oracle replay."""
import numpy as np
import pytest
from scipy import sparse

import openjij_b200 as oj
import openjij_b200.cxxjij.algorithm as A
import openjij_b200.cxxjij.graph as G
import openjij_b200.cxxjij.result as R
import openjij_b200.cxxjij.system as S
import openjij_b200.cxxjij.utility as U
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GROUND8 = [-1, -1, 1, 1, 1, 1, 1, -1]
CASE8 = {(0, 0): -0.1, (0, 1): -0.9, (0, 2): 0.2, (0, 3): 0.1, (0, 4): 1.3, (0, 5): 0.8, (0, 6): 0.9,
         (0, 7): 0.4, (1, 1): -0.7, (1, 2): -1.6, (1, 3): 1.5, (1, 4): 1.5, (1, 5): 1.2, (1, 6): -1.5,
         (1, 7): -1.7, (2, 2): -0.6, (2, 3): 1.2, (2, 4): -1.3, (2, 5): -0.5, (2, 6): -1.9, (2, 7): 1.2,
         (3, 3): 0.8, (3, 4): -0.5, (3, 5): -0.4, (3, 6): -1.8, (3, 7): -2.0, (4, 4): 0.6, (4, 5): -2.0,
         (4, 6): -1.9, (4, 7): 0.5, (5, 5): -1.8, (5, 6): -1.2, (5, 7): 1.8, (6, 6): 0.3, (6, 7): 1.4,
         (7, 7): 1.8}


def dense8():
    d = G.Dense(8)
    for (i, j), v in CASE8.items():
        d[i, j] = v
    return d


def test_classical_dense_and_csr_find_ground_state():
    # tests/test_cxx.py:224-275
    d = dense8()
    csr = G.CSRSparse(sparse.csr_matrix(np.triu(d.get_interactions())))
    for graph in (d, csr):
        system = S.make_classical_ising(d.gen_spin(1234), graph)
        A.Algorithm_SingleSpinFlip_run(system, 5678, U.make_classical_schedule_list(0.1, 100.0, 100, 100))
        assert R.get_solution(system) == GROUND8


def test_transverse_dense_and_csr_find_ground_state():
    # tests/test_cxx.py:419-469
    d = dense8()
    csr = G.CSRSparse(sparse.csr_matrix(np.triu(d.get_interactions())))
    for graph in (d, csr):
        system = S.make_transverse_ising(d.gen_spin(1234), graph, 1.0, 10)
        A.Algorithm_SingleSpinFlip_run(system, 5678, U.make_transverse_field_schedule_list(10, 100, 100))
        assert R.get_solution(system) == GROUND8


def test_callback_run_equals_plain_run():
    d = dense8()
    sched = U.make_classical_schedule_list(0.1, 10.0, 3, 20)
    a = S.make_classical_ising(d.gen_spin(7), d)
    A.Algorithm_SingleSpinFlip_run(a, 99, sched)
    seen = []
    b = S.make_classical_ising(d.gen_spin(7), d)
    A.Algorithm_SingleSpinFlip_run(b, 99, sched, lambda sys, beta: seen.append(beta))
    assert len(seen) == 60
    assert R.get_solution(a) == R.get_solution(b)
    # transverse, tuple-list schedule
    tl = [((10.0, s), 2) for s in np.linspace(0, 1, 10)]
    a = S.make_transverse_ising(d.gen_spin(3), d, 1.0, 4)
    A.Algorithm_SingleSpinFlip_run(a, 5, tl)
    seen = []
    b = S.make_transverse_ising(d.gen_spin(3), d, 1.0, 4)
    A.Algorithm_SingleSpinFlip_run(b, 5, tl, lambda sys, p: seen.append(p))
    assert len(seen) == 20 and seen[0] == (10.0, 0.0)
    np.testing.assert_array_equal(a.trotter_spins, b.trotter_spins)


def test_system_properties():
    d = dense8()
    s = S.make_classical_ising(d.gen_spin(1), d)
    assert s.spin.shape == (9,) and s.spin[-1] == 1
    assert s.num_spins == 8
    t = S.make_transverse_ising(d.gen_spin(1), d, 1.0, 5)
    assert t.trotter_spins.shape == (9, 5)
    assert np.all(t.trotter_spins[-1] == 1)
    t.gamma = 2.0
    assert t.gamma == 2.0


def test_sampler_path_matches_replay():
    """SASampler.sample_ising on a +-J lattice (bit-packed kernel) equals the
    oracle's replay of that kernel from the same seed and initial state."""
    m, _ = I.lattice_pm_j(8, seed=3)
    g = O.AugCSR(m)
    h = {}
    J = {}
    mat = m.tocoo()
    for i, j, v in zip(mat.row, mat.col, mat.data):
        if i < j < g.n:
            J[(int(i), int(j))] = float(v)
    res = oj.SASampler().sample_ising(h, J, beta_min=0.1, beta_max=5.0, num_sweeps=40, num_reads=32,
                                      seed=17)
    assert res.info["run"]["kernel"] == "bitpacked"
    init = np.tile(O.gen_spin(17, g.n), (32, 1))
    betas, mcs = I.geometric_betas(0.1, 5.0, 40)
    per = np.repeat(betas, mcs).astype(np.float32)
    thr, alw = O.msc_thresholds(per, 1.0, 4)
    ref = O.replay_sa_msc(g, init, thr, alw, 17)
    np.testing.assert_array_equal(res.states, ref)
    np.testing.assert_allclose(res.energies, O.energies(g, ref), atol=1e-9)


def test_system_spins_page_locked_or_not_give_the_same_samples(monkeypatch):
    """The systems keep their spins in page-locked blocks of the library's
    host allocator (a freed block serves the next request of its size); the
    samples equal those of a run from ordinary memory (OJ_HOST_PINNED=0)."""
    from openjij_b200 import _native as N

    L = N.lib()
    ctx = N.Context(0)  # blocks are page-locked once a context exists
    size = (5 << 20) + 7
    p = L.oj_host_alloc(size)
    assert p and L.oj_host_is_pinned(p) == 1
    L.oj_host_free(p)
    q = L.oj_host_alloc(size)
    assert q == p
    L.oj_host_free(q)
    m, _ = I.lattice_pm_j(16, seed=4)
    mat = m.tocoo()
    n = m.shape[0] - 1
    J = {(int(i), int(j)): float(v) for i, j, v in zip(mat.row, mat.col, mat.data) if i < j < n}
    out = []
    for pinned in ("1", "0"):
        monkeypatch.setenv("OJ_HOST_PINNED", pinned)
        res = oj.SASampler().sample_ising({}, J, beta_min=0.1, beta_max=5.0, num_sweeps=30, num_reads=64, seed=5)
        out.append((np.asarray(res.states), np.asarray(res.energies)))
        res = oj.SQASampler().sample_ising({}, J, beta=5.0, gamma=1.0, trotter=8, num_sweeps=20, num_reads=16,
                                           seed=6)
        out.append((np.asarray(res.states), np.asarray(res.energies)))
    r = L.oj_host_alloc(1 << 20)
    assert r and L.oj_host_is_pinned(r) == 0
    L.oj_host_free(r)
    for a, b in zip(out[:2], out[2:]):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])
    ctx.close()


# ---- tests/test_sampler.py ------------------------------------------------

NUM_H = {0: -1, 1: -1, 2: 1, 3: 1}
NUM_J = {(0, 1): -1, (3, 4): -1}
GROUND5 = [1, 1, -1, -1, -1]
QUBO = {(0, 0): -1, (1, 1): -1, (2, 2): 1, (3, 3): 1, (4, 4): 1, (0, 1): -1, (3, 4): 1}
QUBO_ND = np.array([[-1, -1, 0, 0, 0], [0, -1, 0, 0, 0], [0, 0, 1, 0, 0], [0, 0, 0, 1, 1], [0, 0, 0, 0, 1]])


def basic(res, n=1):
    assert len(res.states) == n and len(res.energies) == n
    assert len(res.record.sample) == n and len(res.record.energy) == n
    assert isinstance(float(res.energies[0]), float)


def run_samplers(sampler, init=None, qinit=None, schedule=None):
    res = sampler.sample_ising(NUM_H, NUM_J, schedule=schedule, initial_state=init, seed=1)
    basic(res)
    res = sampler.sample_qubo(QUBO, initial_state=qinit, schedule=schedule, seed=2)
    basic(res)
    res = sampler.sample_qubo(QUBO_ND, initial_state=qinit, schedule=schedule, seed=2)
    basic(res)


def test_sa_sampler_reference_cases():
    s = oj.SASampler()
    run_samplers(s)
    run_samplers(s, init=[1] * 5, qinit=[1] * 5)
    run_samplers(s, init={i: 1 for i in range(5)})
    run_samplers(s, init={i: 1 for i in range(5)}, schedule=[[0.1, 10], [1, 10], [10, 10]])
    run_samplers(s, init={i: 1 for i in range(5)}, schedule=[(0.1, 10), (1, 10), (10, 10)])
    res = s.sample_ising(NUM_H, NUM_J, num_reads=10, seed=2)
    basic(res, 10)
    res = oj.SASampler().sample_ising(NUM_H, NUM_J, num_reads=10)
    basic(res, 10)
    # ground states and energies found
    res = oj.SASampler().sample_ising(NUM_H, NUM_J, num_reads=8, seed=3)
    assert list(res.first.sample.values()) == GROUND5 and res.first.energy == -6
    res = oj.SASampler().sample_qubo(QUBO, num_reads=8, seed=3)
    assert list(res.first.sample.values()) == [1, 1, 0, 0, 0] and res.first.energy == -3


def test_sa_afm_chain_and_sparse():
    afih = {0: -10}
    afij = {(i, i + 1): 1 for i in range(29)}
    for sparse_opt in (True, False):
        res = oj.SASampler().sample_ising(afih, afij, seed=1, num_reads=100, sparse=sparse_opt)
        assert len(res.states) == 100
        best = res.first.sample
        assert best == {i: (-1) ** i for i in range(30)}


def test_sa_energies_match_model():
    rng = np.random.default_rng(0)
    h = {i: float(rng.uniform(-1, 1)) for i in range(20)}
    J = {(i, j): float(rng.uniform(-1, 1)) for i in range(20) for j in range(i + 1, 20) if rng.random() < 0.3}
    for sparse_opt in (True, False):
        res = oj.SASampler().sample_ising(h, J, num_reads=16, seed=4, sparse=sparse_opt)
        bqm = oj.BinaryQuadraticModel.from_ising(h, J)
        for st, e in zip(res.samples(), res.energies):
            assert e == pytest.approx(bqm.energy(st), abs=1e-9)
    Q = {(i, j): float(rng.integers(-8, 9)) for i in range(12) for j in range(i, 12)}
    res = oj.SASampler().sample_qubo(Q, num_reads=8, seed=5)
    bqm = oj.BinaryQuadraticModel.from_qubo(Q)
    for st, e in zip(res.samples(), res.energies):
        assert e == pytest.approx(bqm.energy(st), abs=1e-9)


def test_response_info_states_flips_and_field_drift():
    """Response.info carries the call's accepted flips and, for the dense
    kernels, the largest deviation of the incremental FP32 fields from the
    exact fields (recomputed on the tensor cores): positive and small for real
    couplings, zero for integer ones, -1 for the sparse kernels."""
    rng = np.random.default_rng(11)
    n = 300
    Qr = rng.standard_normal((n, n))
    Qi = rng.integers(-8, 9, (n, n)).astype(np.float64)
    for Q, exact in ((np.triu(Qr), False), (np.triu(Qi), True)):
        res = oj.SASampler().sample_qubo(Q, num_reads=16, num_sweeps=64, seed=3)
        assert res.info["run"]["kernel"] == "dense_jump"
        assert res.info["accepted_flips"] > 0
        if exact:
            assert res.info["field_drift"] == 0.0
        else:
            assert 0.0 < res.info["field_drift"] < 1e-2
    h = {i: 0.0 for i in range(16)}
    J = {(i, (i + 1) % 16): -1.0 for i in range(16)}
    res = oj.SASampler().sample_ising(h, J, num_reads=4, num_sweeps=20, seed=1)
    assert res.info["accepted_flips"] > 0 and res.info["field_drift"] == -1.0


def test_sqa_sampler_reference_cases():
    s = oj.SQASampler()
    run_samplers(s)
    run_samplers(s, init=[1] * 5, qinit=[1] * 5)
    run_samplers(s, init={i: 1 for i in range(5)}, schedule=[[0.1, 10], [0.5, 10], [0.9, 10]])
    run_samplers(s, init={i: 1 for i in range(5)}, schedule=[(0.1, 0.1, 10), (0.5, 1, 10), (0.9, 10, 10)])
    res = s.sample_ising(NUM_H, NUM_J, num_reads=10, seed=2)
    basic(res, 10)
    assert res.info["system"]["trotter_state"].shape == (10, 4, 5)
    res = oj.SQASampler().sample_ising({0: -10}, {(i, i + 1): 1 for i in range(29)}, seed=1, num_reads=100)
    assert len(res.states) == 100


@pytest.mark.parametrize("sampler", [oj.SASampler, oj.SQASampler])
def test_empty_and_small(sampler):
    for sp in (True, False):
        res = sampler().sample_ising({}, {}, sparse=sp)
        assert len(res.first.sample) == 0
        res = sampler().sample_qubo({}, sparse=sp)
        assert len(res.first.sample) == 0
    sampler().sample_ising({}, {(0, 1): -1})
    sampler().sample_ising({2: -1}, {(0, 1): -1})


def test_two_variable_cases():
    # tests/test_sampler.py:281-313
    for q, want in [({(0, 0): 1, (1, 1): 1}, [0, 0]), ({(0, 0): -1, (1, 1): -1}, [1, 1]),
                    ({(0, 0): 1, (1, 1): 1, (0, 1): 1e-7}, [0, 0]),
                    ({(0, 0): -1, (1, 1): -1, (0, 1): 1e-7}, [1, 1])]:
        res = oj.SASampler().sample_qubo(q, seed=1)
        assert list(res.states[0]) == want


def test_reverse_annealing_chains_reads():
    s = oj.SASampler()
    res = s.sample_ising(NUM_H, NUM_J, num_reads=4, initial_state=[1, 1, -1, -1, -1],
                         reinitialize_state=False, schedule=[(5.0, 5)], seed=1)
    assert len(res.states) == 4
    assert all(e == -6 for e in res.energies)


def test_unknown_parameter_and_updater():
    with pytest.raises(ValueError):
        oj.SASampler().sample_ising(NUM_H, NUM_J, updater="heat bath")


def test_swendsen_wang_sampler():
    """updater="swendsen wang" (sa_sampler.py:98-107): ground states of the
    reference's 5-spin case and the AFM chain with a field, on the GPU cluster kernel."""
    res = oj.SASampler().sample_ising(NUM_H, NUM_J, updater="swendsen wang", num_reads=16, seed=3)
    assert res.info["run"]["kernel"] == "swendsen_wang"
    assert list(res.first.sample.values()) == GROUND5 and res.first.energy == -6
    res = oj.SASampler().sample_ising({0: -10}, {(i, i + 1): 1 for i in range(29)}, updater="swendsen_wang",
                                      num_reads=32, seed=1, sparse=False)
    assert res.first.sample == {i: (-1) ** i for i in range(30)}
    # the cxxjij binding exists for sparse systems only, as in the reference
    d = G.Dense(4)
    with pytest.raises(TypeError):
        A.Algorithm_SwendsenWang_run(S.make_classical_ising([1, 1, 1, 1], d), 1, U.make_classical_schedule_list(0.1, 1.0, 1, 4))


def test_sa_sample_batch():
    """SASampler.sample_batch: many models of uneven size in one GPU launch, one
    Response per model, energies equal to the models' own."""
    rng = np.random.default_rng(11)
    rand_q = {(i, j): float(rng.standard_normal()) for i in range(40) for j in range(i, 40)}
    models = [oj.BinaryQuadraticModel.from_ising(NUM_H, NUM_J), QUBO, rand_q,
              oj.BinaryQuadraticModel.from_ising({0: -10}, {(i, i + 1): 1 for i in range(29)})]
    out = oj.SASampler().sample_batch(models, num_reads=16, num_sweeps=300, seed=5)
    assert len(out) == 4
    for mdl, res in zip(models, out):
        bqm = mdl if isinstance(mdl, oj.BinaryQuadraticModel) else oj.BinaryQuadraticModel.from_qubo(mdl)
        assert len(res.states) == 16
        for st, e in zip(res.samples(), res.energies):
            assert e == pytest.approx(bqm.energy(st), abs=1e-9)
    assert list(out[0].first.sample.values()) == GROUND5 and out[0].first.energy == -6
    assert list(out[1].first.sample.values()) == [1, 1, 0, 0, 0] and out[1].first.energy == -3
    assert out[3].first.sample == {i: (-1) ** i for i in range(30)}
