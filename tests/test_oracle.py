"""The oracle against the reference's own known answers (CPU only)."""
import math

import numpy as np
import pytest

from oracle import oracle as O

# tests/test_cxx.py:32-69 (= tests/cxxtest/testcase.hpp:33-77): J[i,i] is h_i
CASE8 = {(0, 0): -0.1, (0, 1): -0.9, (0, 2): 0.2, (0, 3): 0.1, (0, 4): 1.3, (0, 5): 0.8, (0, 6): 0.9,
         (0, 7): 0.4, (1, 1): -0.7, (1, 2): -1.6, (1, 3): 1.5, (1, 4): 1.5, (1, 5): 1.2, (1, 6): -1.5,
         (1, 7): -1.7, (2, 2): -0.6, (2, 3): 1.2, (2, 4): -1.3, (2, 5): -0.5, (2, 6): -1.9, (2, 7): 1.2,
         (3, 3): 0.8, (3, 4): -0.5, (3, 5): -0.4, (3, 6): -1.8, (3, 7): -2.0, (4, 4): 0.6, (4, 5): -2.0,
         (4, 6): -1.9, (4, 7): 0.5, (5, 5): -1.8, (5, 6): -1.2, (5, 7): 1.8, (6, 6): 0.3, (6, 7): 1.4,
         (7, 7): 1.8}
GROUND8 = [-1, -1, 1, 1, 1, 1, 1, -1]


def case8():
    h = {i: v for (i, j), v in CASE8.items() if i == j}
    J = {(i, j): v for (i, j), v in CASE8.items() if i != j}
    return O.AugCSR.from_ising(h, J, 8)


def test_philox_known_answers():
    # Random123 known-answer vectors for philox4x32-10
    assert list(O.philox4x32_10([0, 0, 0, 0], [0, 0])) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(O.philox4x32_10([0xffffffff] * 4, [0xffffffff] * 2)) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(O.philox4x32_10([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                [0xa4093822, 0x299f31d0])) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_neglog_accuracy():
    rng = np.random.default_rng(0)
    xs = list(rng.integers(0, 2**32, size=20000, dtype=np.uint64)) + [0, 1, 511, 512, 2**31, 2**32 - 1]
    for x in xs:
        u = (2 * (int(x) >> 9) + 1) * 2.0**-24
        want = -math.log(u)
        got = O.neglog(int(x))
        assert got > 0
        assert abs(got - want) <= 4e-7 * max(1.0, want), (x, got, want)


def test_neglog_largest_value():
    """The sweep kernels skip the uniforms of a 128-site chunk when every
    site's beta*dE is at least 0x1.0a2b24p+4: no -ln u reaches past it (the
    largest, at u = 2^-24, is exactly that)."""
    assert O.neglog_max() == float.fromhex("0x1.0a2b24p+4") == O.neglog(0)


def test_neglog_integer_range_reduction():
    """The sweep kernels reduce u by integer steps (1 + k 2^-23 from the bits
    0x3F800000 | k, minus 1 - 2^-24; an offset split of the bits for m and e;
    float(e) through 0x4B400000 + e): for every k = x >> 9 these give the u, m
    and float(e) of the arithmetic definition the oracle follows, so both
    compute the same -ln u."""
    f32 = np.float32
    for lo in range(0, 1 << 23, 1 << 21):
        k = np.arange(lo, lo + (1 << 21), dtype=np.uint32)
        u = (2 * k + 1).astype(f32) * f32(2.0**-24)
        u_int = (np.uint32(0x3F800000) | k).view(f32) + f32(float.fromhex("-0x1.fffffep-1"))
        np.testing.assert_array_equal(u.view(np.uint32), u_int.view(np.uint32))
        b = u.view(np.uint32)
        e = (b >> 23).astype(np.int32) - 127
        m = ((b & np.uint32(0x7FFFFF)) | np.uint32(0x3F800000)).view(f32)
        big = m > f32(float.fromhex("0x1.6a09e6p+0"))
        m = np.where(big, m * f32(0.5), m)
        e = e + big.astype(np.int32)
        bb = b - np.uint32(0x3F3504F4)
        e_int = bb.view(np.int32) >> 23
        m_int = ((bb & np.uint32(0x7FFFFF)) + np.uint32(0x3F3504F4)).view(f32)
        ef = (np.int32(0x4B400000) + e_int).view(f32) - f32(12582912.0)
        np.testing.assert_array_equal(m.view(np.uint32), m_int.view(np.uint32))
        np.testing.assert_array_equal(e, e_int)
        np.testing.assert_array_equal(e.astype(f32), ef)


def test_schedules_match_reference_formula():
    b = O.classical_schedule(0.1, 100.0, 100)
    assert b[0] == 0.1 and abs(b[-1] - 100.0) < 1e-9
    s = O.transverse_schedule(100)
    assert s[0] == 0.0 and abs(s[-1] - 1.0) < 1e-12


@pytest.mark.parametrize("engine,spin_seed,mc_seed", [("xorshift", 1234, 5678), ("mt", 1, 1)])
def test_reference_sa_finds_known_ground_state(engine, spin_seed, mc_seed):
    # tests/test_cxx.py:224-275 (Xorshift) and tests/cxxtest/sampler/quadraitc.hpp:21-73 (mt19937(1))
    g = case8()
    init = O.gen_spin(spin_seed, 8, engine)
    betas = O.classical_schedule(0.1, 100.0, 100)
    out = O.ref_sa(g, init, betas, np.full(100, 100), mc_seed, engine)
    assert list(out) == GROUND8


def test_reference_sqa_finds_known_ground_state():
    # tests/test_cxx.py:419-469: make_transverse_ising(gen_spin(1234), dense, 1.0, 10)
    g = case8()
    init = O.gen_spin(1234, 8)
    ss = O.transverse_schedule(100)
    _, best = O.ref_sqa(g, np.tile(init, (10, 1)), 1.0, np.full(100, 10.0), ss, np.full(100, 100), 5678)
    assert list(best) == GROUND8


def test_reference_sqa_mt_trotter_init():
    # tests/cxxtest/sampler/quadraitc.hpp:75-102: 10 slices drawn from one mt19937(1), MC mt19937(1)
    g = case8()
    init = O.gen_spin_seq(1, 8, 10, "mt")
    ss = O.transverse_schedule(100)
    _, best = O.ref_sqa(g, init, 1.0, np.full(100, 10.0), ss, np.full(100, 100), 1, "mt")
    assert list(best) == GROUND8


def test_energy_layout_and_value():
    g = case8()
    # the ground state energy of the 8-spin instance
    e = O.energy(g, np.array(GROUND8, np.int8))
    assert abs(e - (-21.5)) < 1e-9


def test_five_spin_sampler_case():
    # tests/test_sampler.py:11-20: h={0:-1,1:-1,2:1,3:1}, J={(0,1):-1,(3,4):-1}, ground [1,1,-1,-1,-1], e=-6
    g = O.AugCSR.from_ising({0: -1, 1: -1, 2: 1, 3: 1}, {(0, 1): -1, (3, 4): -1}, 5)
    assert O.energy(g, np.array([1, 1, -1, -1, -1], np.int8)) == -6.0
    betas, mcs = O.classical_schedule(0.1, 50.0, 100), np.full(100, 10)
    out = O.ref_sa(g, O.gen_spin(1, 5), betas, mcs, 1)
    assert O.energy(g, out) == -6.0


def test_greedy_colouring_checkerboard():
    from openjij_b200 import instances as I
    m, _ = I.lattice_pm_j(8)
    g = O.AugCSR(m)
    col = O.greedy_colour(g)
    ij = np.arange(64).reshape(8, 8)
    assert np.array_equal(col.reshape(8, 8), (ij // 8 + ij % 8) % 2)


def _py_replay_sqa_msc(g, init3d, thr, mode, seed):
    """Slice-by-slice Python restatement of the bit-packed SQA replay (tiny sizes)."""
    R, T, n = init3d.shape
    S = init3d.astype(np.int64).copy()
    nb = [[(int(g.indices[p]), g.data[p]) for p in range(g.indptr[i], g.indptr[i + 1])
           if g.indices[p] != i and g.indices[p] != n and g.data[p] != 0] for i in range(n)]
    col = O.kernel_colour(g)
    classes = [[i for i in range(n) if col[i] == c] for c in range(max(col) + 1)]
    upper = T - 1 if T % 2 else T
    groups = [list(range(0, upper, 2)), list(range(1, T, 2)), [T - 1] if T % 2 else []]
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    for r in range(R):
        for k in range(thr.shape[0]):
            always, live = int(mode[k, 0]), int(mode[k, 1])
            for q, grp in enumerate(groups):
                if not grp:
                    continue
                for cl in classes:
                    for i in cl:
                        before = S[r, :, i].copy()
                        W = []
                        for qq in range(8):
                            W += list(O.philox4x32_10([i, k, r, (qq << 16) | (q << 8) | 0xC3], [k0, k1]))
                        for t in grp:
                            si = before[t]
                            u = sum(1 for j, v in nb[i] if v * si * S[r, t, j] > 0)
                            kk = int(before[(t + 1) % T] == si) + int(before[(t - 1) % T] == si)
                            m = 3 * u + kk
                            if (always >> m) & 1:
                                S[r, t, i] = -si
                            elif (live >> m) & 1:
                                U = sum(((int(W[l]) >> t) & 1) << (31 - l) for l in range(32))
                                if U < int(thr[k, m]):
                                    S[r, t, i] = -si
    return S.astype(np.int8)


@pytest.mark.parametrize("T", [2, 3, 6])
def test_bitpacked_sqa_replay_matches_python_restatement(T):
    rng = np.random.default_rng(T)
    n = 8  # ring of 8 with +-1 couplings: 2-regular
    J = {(i, (i + 1) % n): float(rng.choice([-1.0, 1.0])) for i in range(n)}
    g = O.AugCSR.from_ising(np.zeros(n), J, n)
    ss = np.linspace(0.0, 1.0, 5)
    betas = np.full(5, 3.0)
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    thr, mode = O.sqa_msc_thresholds(a, b, 1.0, 2)
    init = rng.choice(np.array([-1, 1], np.int8), size=(2, T, n))
    got = O.replay_sqa_msc(g, init, thr, mode, seed=0x1234_0000_0007)
    want = _py_replay_sqa_msc(g, init, thr, mode, seed=0x1234_0000_0007)
    np.testing.assert_array_equal(got, want)


def test_bitpacked_sqa_thresholds_classes():
    # a = 0.25, B = -0.5: dE = 0.25*2(2-2u) - 0.5*(4-4k) for D = 2
    thr, mode = O.sqa_msc_thresholds(np.array([0.25], np.float32), np.array([-0.5], np.float32), 1.0, 2)
    for u in range(3):
        for k in range(3):
            m = 3 * u + k
            dE = 0.25 * 2 * (2 - 2 * u) - 0.5 * (4 - 4 * k)
            if dE <= 0:
                assert (mode[0, 0] >> m) & 1 and thr[0, m] == 0
            else:
                assert (mode[0, 1] >> m) & 1
                assert thr[0, m] == math.floor(math.exp(-dE) * 2 ** 32)
    # s = 1 -> B = -inf: k = 1 is NaN (never), k = 0 always, k = 2 never
    thr, mode = O.sqa_msc_thresholds(np.array([0.1], np.float32), np.array([-np.inf], np.float32), 1.0, 2)
    for u in range(3):
        assert (mode[0, 0] >> (3 * u)) & 1
        assert not (mode[0, 0] >> (3 * u + 1)) & 1 and not (mode[0, 1] >> (3 * u + 1)) & 1
        assert not (mode[0, 0] >> (3 * u + 2)) & 1 and not (mode[0, 1] >> (3 * u + 2)) & 1


def _py_replay_sqa_split(g, init3d, thr, mode, seed):
    """Python restatement of the slice-split bit-packed SQA replay (tiny sizes)."""
    R, T, n = init3d.shape
    H = T // 2
    P = 1
    while 2 * P * H <= 32:
        P *= 2
    S = init3d.astype(np.int64).copy()
    nb = [[(int(g.indices[p]), g.data[p]) for p in range(g.indptr[i], g.indptr[i + 1])
           if g.indices[p] != i and g.indices[p] != n and g.data[p] != 0] for i in range(n)]
    col = O.kernel_colour(g)
    classes = [[i for i in range(n) if col[i] == c] for c in range(max(col) + 1)]
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    for r in range(R):
        gi, p = divmod(r, P)
        for k in range(thr.shape[0]):
            always, live = int(mode[k, 0]), int(mode[k, 1])
            for q in (0, 1):
                for cl in classes:
                    for i in cl:
                        W = []
                        for qq in range(8):
                            W += list(O.philox4x32_10([i, k, gi, (qq << 16) | (q << 8) | 0x69], [k0, k1]))
                        for t in range(q, T, 2):
                            bit = p * H + t // 2
                            si = S[r, t, i]
                            u = sum(1 for j, v in nb[i] if v * si * S[r, t, j] > 0)
                            kk = int(S[r, (t + 1) % T, i] == si) + int(S[r, (t - 1) % T, i] == si)
                            m = 3 * u + kk
                            if (always >> m) & 1:
                                S[r, t, i] = -si
                            elif (live >> m) & 1:
                                U = sum(((int(W[l]) >> bit) & 1) << (31 - l) for l in range(32))
                                if U < int(thr[k, m]):
                                    S[r, t, i] = -si
    return S.astype(np.int8)


@pytest.mark.parametrize("T,R", [(2, 3), (6, 9), (32, 3)])
def test_slice_split_sqa_replay_matches_python_restatement(T, R):
    rng = np.random.default_rng(10 + T)
    n = 6
    J = {(i, (i + 1) % n): float(rng.choice([-1.0, 1.0])) for i in range(n)}
    g = O.AugCSR.from_ising(np.zeros(n), J, n)
    ss = np.linspace(0.0, 1.0, 3)
    betas = np.full(3, 3.0)
    a, b = O.sqa_coefficients(betas, ss, 1.0, T)
    thr, mode = O.sqa_msc_thresholds(a, b, 1.0, 2)
    init = rng.choice(np.array([-1, 1], np.int8), size=(R, T, n))
    got = O.replay_sqa_split(g, init, thr, mode, seed=0x9_0000_0003)
    want = _py_replay_sqa_split(g, init, thr, mode, seed=0x9_0000_0003)
    np.testing.assert_array_equal(got, want)


def _py_replay_sa_batch(mats, reads, spins, betas, seed, inst0=0, recompute=0):
    """Python restatement of the batched dense SA replay (tiny sizes): fields
    on the grid 2^e (e = E - 26, 2^(E-1) <= max|J| < 2^E, couplings rounded
    half to even), f = fp32(fp64(h) + 2^e sum q s); set anew before every
    sweep k > 0 that is a multiple of `recompute`.  Returns the spins and the
    largest |f - f_new| per replica (recompute points and the end)."""
    import math
    out = np.array(spins, np.int64)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    off = 0
    drifts = []
    for m, A in enumerate(mats):
        n = A.shape[0] - 1
        J = A[:n, :n].astype(np.float32)
        h = A[:n, n].astype(np.float32)
        amax = float(np.abs(J).max()) if n else 0.0
        e = math.frexp(amax)[1] - 26 if amax > 0 else 0
        q = [[int(np.rint(math.ldexp(float(J[j, i]), -e))) for i in range(n)] for j in range(n)]

        def field(s):
            return np.array([np.float32(float(h[j]) + math.ldexp(sum(q[j][i] * int(s[i]) for i in range(n)), e))
                             for j in range(n)], np.float32)

        for r in range(reads[m]):
            s = out[off + r * n: off + (r + 1) * n]
            f = field(s)
            drift = np.float32(0.0)
            for k, beta in enumerate(np.asarray(betas, np.float32)):
                if recompute and k > 0 and k % recompute == 0:
                    fn = field(s)
                    drift = max(drift, np.abs(fn - f).max())
                    f = fn
                for i in range(n):
                    dE = np.float32(-2.0) * f[i] if s[i] > 0 else np.float32(2.0) * f[i]
                    u = O.philox4x32_10([i >> 2, k, r, ((inst0 + m) << 8) | 0x96], [k0, k1])[i & 3]
                    if dE <= 0 or np.float32(beta * dE) < np.float32(O.neglog(int(u))):
                        c = np.float32(-2.0 if s[i] > 0 else 2.0)
                        f = (f + c * J[i]).astype(np.float32)
                        s[i] = -s[i]
            drifts.append(max(drift, np.abs(field(s) - f).max()))
        off += reads[m] * n
    return out.astype(np.int8), np.array(drifts, np.float32)


@pytest.mark.parametrize("recompute", [0, 2])
def test_batched_replay_matches_python_restatement(recompute):
    rng = np.random.default_rng(7)
    mats = []
    for n in (5, 3, 6):
        Q = np.triu(rng.standard_normal((n, n)).astype(np.float32).astype(np.float64))
        A = np.zeros((n + 1, n + 1))
        A[:n, :n] = np.triu(Q, 1) + np.triu(Q, 1).T
        A[:n, n] = A[n, :n] = np.diag(Q)
        A[n, n] = 1.0
        mats.append(A)
    reads = [2, 3, 1]
    spins = rng.choice(np.array([-1, 1], np.int8), size=sum(r * (m.shape[0] - 1) for r, m in zip(reads, mats)))
    betas = np.array([0.3, 1.0, 2.0, 4.0, 6.0])
    got, drift = O.replay_sa_batch(mats, reads, spins, betas, seed=0x55_0000_0011, inst0=4, recompute=recompute,
                                   drift=True)
    want, want_drift = _py_replay_sa_batch(mats, reads, spins, betas, seed=0x55_0000_0011, inst0=4,
                                           recompute=recompute)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(drift, want_drift)


def test_kernel_colouring_is_proper_and_even():
    from openjij_b200 import instances as I
    for m in (I.random_regular_pm_j(4096, 3, seed=4)[0], I.lattice_pm_j(16, seed=1)[0],
              I.random_regular_pm_j(500, 5, seed=2)[0]):
        g = O.AugCSR(m)
        col = O.kernel_colour(g)
        greedy = O.greedy_colour(g)
        rp, ci = O.neighbour_csr(g)[:2]
        for i in range(g.n):
            assert all(col[i] != col[j] for j in ci[rp[i]:rp[i + 1]])
        sizes = np.bincount(col)
        assert len(sizes) == greedy.max() + 1
        assert sizes.max() <= max(np.bincount(greedy).max(), -(-g.n // len(sizes)))
    sizes = np.bincount(O.kernel_colour(O.AugCSR(I.random_regular_pm_j(4096, 3, seed=4)[0])))
    assert sizes.max() == 1024  # four classes of 1024 (greedy gives 1526/1506/968/96)
