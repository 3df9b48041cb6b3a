"""BinaryQuadraticModel and graph hand-off (CPU only), after the reference's
tests/test_model.py."""
import numpy as np
import pytest

import openjij_b200 as oj
import openjij_b200.cxxjij as cj


def ising_energy(h, J, s):
    return sum(v * s[i] * s[j] for (i, j), v in J.items()) + sum(v * s[i] for i, v in h.items())


def qubo_energy(Q, x):
    return sum(v * x[i] * x[j] for (i, j), v in Q.items())


H = {0: 1, 1: -2}
J = {(0, 1): -1, (1, 2): -3, (2, 3): 0.5}
SPINS = {0: 1, 1: -1, 2: 1, 3: 1}
Q = {(0, 0): 1, (1, 2): -1, (2, 0): -0.2, (1, 3): 3}
BINS = {0: 0, 1: 1, 2: 1, 3: 0}


def test_variable_type():
    assert oj.cast_vartype("SPIN") == oj.SPIN
    assert oj.cast_vartype("BINARY") == oj.BINARY


def test_bqm_constructor():
    bqm = oj.BinaryQuadraticModel(H, J, "SPIN", sparse=False)
    assert isinstance(bqm.interaction_matrix(), np.ndarray)
    assert bqm.vartype == oj.SPIN
    g, off = bqm.get_cxxjij_ising_graph()
    assert isinstance(g, cj.graph.Dense)
    assert off == 0
    assert oj.BinaryQuadraticModel.from_qubo(Q=Q).vartype == oj.BINARY


def test_interaction_matrix_layout():
    # tests/test_model.py:57-68
    want = np.array([[0, -1, 0, 0, 1], [0, 0, -3, 0, -2], [0, 0, 0, 0.5, 0], [0, 0, 0, 0, 0],
                     [0, 0, 0, 0, 1]])
    np.testing.assert_array_equal(oj.BinaryQuadraticModel(H, J, "SPIN").interaction_matrix(), want)


@pytest.mark.parametrize("sparse", [False, True])
def test_transfer_to_cxxjij(sparse):
    bqm = oj.BinaryQuadraticModel(H, J, "SPIN", sparse=sparse)
    g, off = bqm.get_cxxjij_ising_graph()
    assert g.size() == len(bqm.variables)
    M = bqm.interaction_matrix()
    M = M.toarray() if hasattr(M, "toarray") else M
    G = g.get_interactions()
    G = G.toarray() if hasattr(G, "toarray") else G
    n = len(bqm.variables)
    for i in range(n + 1):
        for j in range(i + 1, n + 1):
            assert M[i, j] == pytest.approx(G[i, j])
            assert G[i, j] == pytest.approx(G[j, i])
    qb = oj.BinaryQuadraticModel.from_qubo(Q=Q)
    g, off = qb.get_cxxjij_ising_graph()
    assert off == pytest.approx(qb.change_vartype("SPIN", inplace=False).offset)


def test_energies():
    assert oj.BinaryQuadraticModel(H, J, "SPIN").energy(SPINS) == ising_energy(H, J, SPINS)
    qb = oj.BinaryQuadraticModel.from_qubo(Q=Q)
    assert qb.energy(BINS) == qubo_energy(Q, BINS)
    s = {0: 1, 1: 1, 2: -1, 3: 1}
    x = {0: 1, 1: 1, 2: 0, 3: 1}
    e = qb.energy(x)
    qb.change_vartype("SPIN")
    assert qb.energy(s) == pytest.approx(e)


def test_energy_consistency_dense_csr():
    d, _ = oj.BinaryQuadraticModel(H, J, "SPIN", sparse=False).get_cxxjij_ising_graph()
    c, _ = oj.BinaryQuadraticModel(H, J, "SPIN", sparse=True).get_cxxjij_ising_graph()
    spins = [-1, -1, -1, -1]
    assert d.calc_energy(spins) == pytest.approx(c.calc_energy(spins))
    assert d.calc_energy(spins) == pytest.approx(ising_energy(H, J, dict(enumerate(spins))))


def test_dense_validation_errors():
    d = cj.graph.Dense(3)
    bad = np.zeros((4, 4))
    with pytest.raises(RuntimeError):
        d.set_interaction_matrix(bad)  # corner must be 1
    bad[3, 3] = 1
    bad[1, 1] = 0.5
    with pytest.raises(RuntimeError):
        d.set_interaction_matrix(bad)  # zero diagonal
    with pytest.raises(RuntimeError):
        d.set_interaction_matrix(np.zeros((3, 3)))
    with pytest.raises(IndexError):
        d.calc_energy([1, 1])


def test_gen_spin_matches_reference_stream():
    from oracle import oracle as O
    d = cj.graph.Dense(40)
    assert list(d.gen_spin(1234)) == list(O.gen_spin(1234, 40))


def test_schedules():
    from oracle import oracle as O
    s = cj.utility.make_classical_schedule_list(0.1, 100.0, 3, 50)
    np.testing.assert_array_equal([e.updater_parameter.beta for e in s], O.classical_schedule(0.1, 100.0, 50))
    assert all(e.one_mc_step == 3 for e in s)
    t = cj.utility.make_transverse_field_schedule_list(10.0, 1, 20)
    np.testing.assert_array_equal([e.updater_parameter.s for e in t], O.transverse_schedule(20))


def test_sampler_constructor_rejects_parameters():
    # tests/test_sampler.py:263-279
    for kw in [dict(num_reads=100), dict(num_sweeps=100), dict(beta_min=10), dict(beta_max=10)]:
        with pytest.raises(TypeError):
            oj.SASampler(**kw)
    for kw in [dict(num_reads=100), dict(num_sweeps=100), dict(beta=10), dict(trotter=10)]:
        with pytest.raises(TypeError):
            oj.SQASampler(**kw)


def test_transverse_needs_two_slices():
    d = cj.graph.Dense(3)
    with pytest.raises(ValueError):
        cj.system.make_transverse_ising([1, 1, 1], d, 1.0, 1)


def test_system_spins_from_int8_and_float_inputs_agree():
    """int8 arrays (read in place) and float / list inputs (converted) give
    the same system spins; a value other than +-1 raises ValueError and leaves
    the system's spins as they were; a trailing dummy spin column is dropped."""
    rng = np.random.default_rng(4)
    n, R, T = 12, 5, 3
    d = cj.graph.Dense(n)
    s8 = rng.choice(np.array([-1, 1], np.int8), size=(R, n))
    a = cj.system.make_classical_ising(s8, d)
    b = cj.system.make_classical_ising(s8.astype(np.float64), d)
    np.testing.assert_array_equal(a._spins_int8(), s8)
    np.testing.assert_array_equal(b._spins_int8(), s8)
    a.reset_spins(np.concatenate([s8, np.ones((R, 1), np.int8)], 1))
    np.testing.assert_array_equal(a._spins_int8(), s8)
    a.reset_spins(s8[2])
    np.testing.assert_array_equal(a._spins_int8(), s8[2:3])
    b.reset_spins(list(s8[3].astype(int)))
    np.testing.assert_array_equal(b._spins_int8(), s8[3:4])
    for bad_value in (0, 3, -128, 127):
        bad = s8.copy()
        bad[1, 4] = bad_value
        with pytest.raises(ValueError):
            a.reset_spins(bad)
        np.testing.assert_array_equal(a._spins_int8(), s8[2:3])
    t8 = rng.choice(np.array([-1, 1], np.int8), size=(R, T, n))
    t = cj.system.make_transverse_ising(t8, d, 1.0)
    u = cj.system.make_transverse_ising(t8.astype(np.float32), d, 1.0)
    np.testing.assert_array_equal(t._spins_int8(), t8)
    np.testing.assert_array_equal(u._spins_int8(), t8)
    bad = t8.copy()
    bad[0, 1, 2] = 2
    with pytest.raises(ValueError):
        t.reset_spins(bad)
    np.testing.assert_array_equal(t._spins_int8(), t8)
    c = cj.system.make_transverse_ising(s8, d, 1.0, 4)
    np.testing.assert_array_equal(c._spins_int8(), np.repeat(s8[:, None, :], 4, 1))
    # views: broadcast (zero strides), permuted axes, reversed rows, a strided last axis
    one = s8[0]
    a.reset_spins(np.broadcast_to(one, (R, n)))
    np.testing.assert_array_equal(a._spins_int8(), np.tile(one, (R, 1)))
    a.reset_spins(s8[::-1])
    np.testing.assert_array_equal(a._spins_int8(), s8[::-1])
    wide = rng.choice(np.array([-1, 1], np.int8), size=(R, 2 * n))
    a.reset_spins(wide[:, ::2])
    np.testing.assert_array_equal(a._spins_int8(), wide[:, ::2])
    t.reset_spins(np.broadcast_to(one, (R, T, n)))
    np.testing.assert_array_equal(t._spins_int8(), np.broadcast_to(one, (R, T, n)))
    perm = t8.transpose(1, 0, 2).copy().transpose(1, 0, 2)
    t.reset_spins(perm)
    np.testing.assert_array_equal(t._spins_int8(), t8)
