"""Lattice graphs and models: cxxjij.graph.Sparse / Square / Chimera
(include/openjij/graph/{sparse,square,chimera}.hpp), ChimeraModel and
KingGraph (openjij/model/{chimera_model,king_graph}.py) and the GPU anneal of
a Chimera system, the job of the reference's retired Chimera GPU kernel, here
on the colour-class kernels."""
import itertools

import numpy as np
import pytest

import openjij_b200 as oj
import openjij_b200.cxxjij.algorithm as A
import openjij_b200.cxxjij.graph as G
import openjij_b200.cxxjij.result as R
import openjij_b200.cxxjij.system as S
import openjij_b200.cxxjij.utility as U
from openjij_b200.model.chimera_model import ChimeraModel
from openjij_b200.model.king_graph import KingGraph
from openjij_b200.utils import chimera_to_ind, qubo_to_ising
from oracle import oracle as O

D = G.ChimeraDir


def chimera_case():
    """tests/cxxtest/testcase.hpp:270-300 (generate_chimera_interaction)."""
    c = G.Chimera(2, 2)
    for r, col, i in itertools.product(range(2), range(2), range(4)):
        for d in (D.IN_0or4, D.IN_1or5, D.IN_2or6, D.IN_3or7):
            c[r, col, i, d] = +0.25
    c[0, 0, 0] = +1
    c[0, 0, 6, D.PLUS_C] = +1
    c[0, 0, 3, D.PLUS_R] = -1
    c[1, 0, 5, D.PLUS_C] = +1
    return c


def chimera_ground(c):
    """tests/cxxtest/testcase.hpp:351-391 (get_true_chimera_groundstate)."""
    s = [0] * c.size()
    for (r, col), left in {(0, 0): -1, (0, 1): +1, (1, 0): -1, (1, 1): +1}.items():
        for i in range(8):
            s[c.to_ind(r, col, i)] = left if i < 4 else -left
    return s


# ---- graph classes (CPU) ---------------------------------------------------

def test_chimera_indexing_and_bonds():
    c = G.Chimera(2, 3)
    assert c.size() == 48 and c.get_num_row() == 2 and c.get_num_column() == 3 and c.get_num_in_chimera() == 8
    for ind in range(c.size()):
        assert c.to_ind(*c.to_rci(ind)) == ind
    assert c.to_ind(-1, 0, 1) == c.to_ind(1, 0, 1) and c.to_ind(0, 3, 4) == c.to_ind(0, 0, 4)
    with pytest.raises(RuntimeError):
        c.to_ind(3, 0, 0)
    with pytest.raises(RuntimeError):
        c.to_ind(0, 0, 8)
    c[0, 1, 2, D.IN_1or5] = 0.5  # (0,1,2)-(0,1,5), seen from both ends
    assert c[0, 1, 5, D.IN_2or6] == 0.5
    c[0, 0, 3, D.PLUS_R] = -1.5
    assert c[1, 0, 3, D.MINUS_R] == -1.5
    c[1, 2, 6, D.PLUS_C] = 2.0  # wraps to column 0
    assert c[1, 0, 6, D.MINUS_C] == 2.0
    with pytest.raises(ValueError):
        c[0, 0, 5, D.PLUS_R] = 1.0
    with pytest.raises(ValueError):
        c[0, 0, 1, D.MINUS_C] = 1.0
    c[1, 1, 7] = -0.75
    assert c[1, 1, 7] == -0.75
    # a fresh Chimera lists the open-boundary bonds and the field of every site
    assert sorted(G.Chimera(1, 1).adj_nodes(0)) == [0, 4, 5, 6, 7]
    assert sorted(G.Chimera(2, 1).adj_nodes(0)) == [0, 4, 5, 6, 7, 8]


def test_chimera_interaction_matrix_and_energy():
    c = chimera_case()
    M = c.get_interactions().toarray()
    n = c.size()
    assert M.shape == (n + 1, n + 1) and M[n, n] == 1.0
    np.testing.assert_array_equal(M, M.T)
    assert M[c.to_ind(0, 0, 0), n] == 1.0
    assert M[c.to_ind(0, 0, 6), c.to_ind(0, 1, 6)] == 1.0
    assert M[c.to_ind(0, 0, 3), c.to_ind(1, 0, 3)] == -1.0
    assert M[c.to_ind(1, 1, 2), c.to_ind(1, 1, 6)] == 0.25
    s = np.array(chimera_ground(c), float)
    e = 0.5 * s @ M[:n, :n] @ s + M[:n, n] @ s
    assert c.calc_energy(chimera_ground(c)) == pytest.approx(e, abs=1e-12)


def test_square_graph():
    sq = G.Square(3, 4, 1.0)
    assert sq.size() == 12 and sq.to_rc(7) == (1, 3) and sq.to_ind(-1, 4) == 8
    assert sq[1, 2] == 1.0 and sq[1, 2, G.Dir.PLUS_C] == 1.0
    sq[2, 3, G.Dir.PLUS_R] = -2.0  # periodic bond to (0, 3)
    assert sq[0, 3, G.Dir.MINUS_R] == -2.0
    assert sorted(sq.adj_nodes(sq.to_ind(0, 3))) == sorted([2, 7, 3, 11])
    M = sq.get_interactions().toarray()
    np.testing.assert_array_equal(M, M.T)
    assert M[3, 11] == -2.0 and M[0, 12] == 1.0


def test_sparse_graph_and_edge_limit():
    g = G.Sparse(5)
    g[0, 1] = -1.0
    g[1, 0] = -2.0  # the same bond
    g[3] = 0.5
    assert g[0, 1] == -2.0 and g[3] == 0.5 and g.get_num_edges() == 5
    with pytest.raises(IndexError):
        g[2, 4]
    assert g.calc_energy([1, 1, 1, -1, 1]) == pytest.approx(-2.0 - 0.5)
    # a list that is full takes no new neighbour (sparse.hpp:42-60)
    lim = G.Sparse(4, 1)
    lim[0, 1] = 1.0
    lim[0, 2] = 3.0
    assert lim.adj_nodes(0) == [1] and lim.adj_nodes(2) == []
    M = lim.get_interactions().toarray()
    assert M[0, 1] == 1.0 and M[0, 2] == 0.0


def test_chimera_case_reference_anneal_on_cpu():
    """The oracle's restatement of the reference anneal (Xorshift, FP64)
    reaches the reference's stated Chimera ground state on this matrix."""
    c = chimera_case()
    g = O.AugCSR(c.get_interactions())
    init = np.asarray(c.gen_spin(1264), np.int8)
    sched = O.classical_schedule(0.1, 100.0, 100)
    out = O.ref_sa(g, init, sched, np.full(len(sched), 100, np.int64), 12356)
    assert list(out) == chimera_ground(c)


# ---- models (CPU) ------------------------------------------------------------

def test_chimera_model():
    Q = {(0, 4): -1, (4, 12): -1}
    cm = ChimeraModel.from_qubo(Q, unit_num_L=2)
    assert cm.validate_chimera() and cm.coordinate == "index" and cm.variables == [0, 4, 12]
    assert cm.chimera_coordinate(12, 2) == (0, 1, 4) and cm.to_index(0, 1, 4, 2) == 12
    g = cm.get_cxxjij_ising_graph()
    assert g.size() == 32
    assert g[0, 0, 0, D.IN_0or4] == -0.25 and g[0, 0, 4, D.PLUS_C] == -0.25 and g[0, 0, 4] == -0.5
    with pytest.raises(ValueError):
        ChimeraModel({}, {(0, 1): -1}, unit_num_L=2).validate_chimera()
    with pytest.raises(ValueError):
        ChimeraModel({}, {(0, 8): -1}, unit_num_L=2).validate_chimera()  # z 0 couples vertically, not across
    with pytest.raises(ValueError):
        ChimeraModel({}, {(0, 4): -1}, unit_num_L=0)
    cc = ChimeraModel({(0, 0, 1): 0.5}, {((0, 0, 0), (0, 0, 5)): -1, ((0, 0, 5), (0, 1, 5)): 2}, unit_num_L=2)
    assert cc.coordinate == "chimera coordinate" and cc.graph_sites() == [0, 1, 5, 13]
    assert cc.get_cxxjij_ising_graph()[0, 1, 5, D.MINUS_C] == 2.0
    assert chimera_to_ind(1, 1, 3, 2) == 27
    with pytest.raises(ValueError):
        chimera_to_ind(2, 0, 0, 2)


def test_king_graph():
    kg = KingGraph(machine_type="ASIC", linear={}, quadratic={(0, 1): -1.0, (1, 2): -3.0})
    assert kg.get_ising_king_graph() == [[0, 0, 1, 0, -1.0], [1, 0, 2, 0, -3.0]]
    assert kg.king_indices() == [(0, 0), (1, 0), (2, 0)] and kg.convert_to_index(3, 1) == 355
    kl = KingGraph(machine_type="FPGA", king_graph=[[0, 0, 1, 0, -1.0], [1, 0, 2, 1, -3.0], [2, 1, 2, 1, 2.0]])
    assert kl.variables == [(0, 0), (1, 0), (2, 1)] and kl.linear[(2, 1)] == 2.0
    for bad in ({(0, 2): -1.0}, {(0, 1): -5.0}):
        with pytest.raises(ValueError):
            KingGraph(machine_type="ASIC", quadratic=bad)
    with pytest.raises(ValueError):
        KingGraph(quadratic={(0, 1): -1.0})
    kq = KingGraph.from_qubo({(0, 0): -1, (0, 1): 2}, machine_type="FPGA")
    assert kq.vartype == oj.BINARY and kq.get_ising_king_graph() == [[1, 0, 1, 0, 0.5], [0, 0, 1, 0, 0.5]]
    m = np.array([[1.0, 2.0], [0.0, 3.0]])
    qubo_to_ising(m)
    np.testing.assert_array_equal(m, [[1.0, 0.5], [0.0, 1.5]])


# ---- on the GPU ----------------------------------------------------------------

@pytest.mark.gpu
def test_chimera_classical_ground_state():
    """FindTrueGroundState_ChimeraClassicalGPU (tests/cxxtest/sampler/gpu.hpp:67-86)."""
    c = chimera_case()
    system = S.make_classical_ising(c.gen_spin(1264), c)
    A.Algorithm_SingleSpinFlip_run(system, 12356, U.make_classical_schedule_list(0.1, 100.0, 100, 100))
    assert R.get_solution(system) == chimera_ground(c)


@pytest.mark.gpu
def test_chimera_transverse_ground_state():
    """FindTrueGroundState_ChimeraTransverseGPU (gpu.hpp:42-65), with 4 slices."""
    c = chimera_case()
    trotter = [c.gen_spin(1253 + t) for t in range(4)]
    system = S.make_transverse_ising(trotter, c, 1.0)
    A.Algorithm_SingleSpinFlip_run(system, 12356, U.make_transverse_field_schedule_list(10, 100, 100))
    assert R.get_solution(system) == chimera_ground(c)


@pytest.mark.gpu
def test_chimera_system_matches_replay():
    """The Chimera system's anneal equals the colour-class replay on its matrix."""
    c = G.Chimera(4, 4)
    rng = np.random.default_rng(3)
    for ind in range(c.size()):
        r, col, i = c.to_rci(ind)
        for d in (D.IN_0or4, D.IN_1or5, D.IN_2or6, D.IN_3or7):
            c[r, col, i, d] = float(rng.choice([-1.0, 1.0, 0.5]))
        c[r, col, i] = float(rng.normal())
    init = np.asarray([c.gen_spin(s) for s in range(16)], np.int8)
    system = S.make_classical_ising(init, c)
    sched = U.make_classical_schedule_list(0.1, 5.0, 2, 30)
    A.Algorithm_SingleSpinFlip_run(system, 77, sched)
    assert oj.cxxjij.last_run_info()["kernel"] == "colour"
    g = O.AugCSR(c.get_interactions())
    betas = np.array([e.updater_parameter.beta for e in sched])
    ref = O.replay_sa(g, init, np.repeat(betas, 2).astype(np.float32), 77)
    got = np.asarray(R.get_solution(system), np.int8).reshape(16, -1)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
def test_chimera_model_samplers():
    Q = {(0, 4): -1, (4, 12): -1, (0, 0): 0.5, (12, 12): -0.25}
    cm = ChimeraModel.from_qubo(Q, unit_num_L=2)
    best = min(itertools.product((0, 1), repeat=3), key=lambda x: cm.energy(list(x)))
    for sampler in (oj.SASampler(), oj.SQASampler()):
        res = sampler.sample(cm, num_reads=8, seed=5)
        assert res.variables == [0, 4, 12]
        assert list(res.first.sample.values()) == list(best)
        np.testing.assert_allclose(res.energies, [cm.energy(list(s)) for s in res.states], atol=1e-12)
    res = oj.SASampler().sample(cm, num_reads=2, initial_state={0: 1, 4: 1, 12: 0}, num_sweeps=10, seed=1)
    assert res.states.shape == (2, 3)


@pytest.mark.gpu
def test_king_graph_sampler():
    rng = np.random.default_rng(4)
    quad, lin = {}, {}
    W, H = 4, 3
    for x, y in itertools.product(range(W), range(H)):
        lin[(x, y)] = int(rng.integers(-3, 4))
        for dx, dy in ((1, 0), (0, 1), (1, 1), (1, -1)):
            if 0 <= x + dx < W and 0 <= y + dy < H:
                quad[((x, y), (x + dx, y + dy))] = int(rng.integers(-3, 4))
    kg = KingGraph(linear=lin, quadratic=quad, machine_type="ASIC")
    e0 = min(kg.energy(list(s)) for s in itertools.product((-1, 1), repeat=W * H))
    res = oj.SASampler().sample(kg, num_reads=16, num_sweeps=500, seed=2)
    assert res.first.energy == pytest.approx(e0)
    assert res.info["run"]["kernel"] == "colour"
