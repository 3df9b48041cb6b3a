"""Error paths, made on the host (no device fault): every device allocation of
a call failing in turn (oj_ctx_inject_fault) must give OJ_ERR_OOM with the
context still usable; non-finite couplings and bad shapes are refused before
any device work.  The reference maps its C++ exceptions to Python errors
(include/openjij/graph/dense.hpp:122-137, system/transverse_ising.hpp:78-81);
here each becomes a status code and a message."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _init(shape, seed):
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=shape)


def _each_allocation_fails(run):
    """Runs run(ctx) on a fresh context with the k-th device allocation failing,
    k = 0, 1, ... until a run needs no more allocations than k; every failing
    run must report OJ_ERR_OOM and the same context must then run cleanly.
    Returns the number of allocation points met."""
    for k in range(200):
        ctx = N.Context(0)
        ctx.inject_alloc_failure(k)
        try:
            run(ctx)
            failed = False
        except N.OJError as err:
            assert err.status == N.OJ_ERR_OOM, err
            failed = True
        finally:
            ctx.inject_alloc_failure(None)
        run(ctx)  # the context is still usable and the run completes
        ctx.close()
        if not failed:
            return k
    raise AssertionError("more than 200 allocation points")


def test_sa_runs_survive_every_allocation_failure():
    m, _ = I.dense_qubo_normal(200, seed=3)
    g = O.AugCSR(m)
    lat, _ = I.lattice_pm_j(16, seed=2)
    gl = O.AugCSR(lat)
    betas, mcs = I.geometric_betas(0.1, 5.0, 20)
    per = np.repeat(betas, mcs).astype(np.float32)
    s0 = _init((9, g.n), 1)
    s0l = _init((64, gl.n), 2)
    want = O.replay_sa_batch([m.toarray()], [9], s0.ravel(), per, 4).reshape(9, g.n)
    thr, alw = O.msc_thresholds(per, 1.0, 4)
    want_l = O.replay_sa_msc(gl, s0l, thr, alw, 4)

    def run(ctx):
        dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
        s = s0.copy()
        e = np.zeros(9)
        N.sa_run(dg, s, betas, mcs, seed=4, kernel="dense_jump", energies=e)
        np.testing.assert_array_equal(s, want)
        lg = N.Graph(ctx, gl.n, gl.indptr, gl.indices, gl.data)
        s = s0l.copy()
        N.sa_run(lg, s, betas, mcs, seed=4, kernel="bitpacked")
        np.testing.assert_array_equal(s, want_l)

    assert _each_allocation_fails(run) > 5


def test_batched_and_sqa_runs_survive_every_allocation_failure():
    mats = [I.dense_qubo_normal(n, seed=n)[0].toarray() for n in (50, 140)]
    reads = [3, 5]
    betas, mcs = I.geometric_betas(0.1, 5.0, 20)
    per = np.repeat(betas, mcs).astype(np.float32)
    sb0 = _init(sum(r * (a.shape[0] - 1) for r, a in zip(reads, mats)), 3)
    want_b = O.replay_sa_batch(mats, reads, sb0, per, 6)
    m, _ = I.random_regular_pm_j(96, 3, seed=4)
    g = O.AugCSR(m)
    T = 8
    t0 = np.ascontiguousarray(np.broadcast_to(_init((8, g.n), 4)[:, None, :], (8, T, g.n)))
    ss = np.linspace(0.0, 0.9, 6)
    sb = np.full(6, 4.0)
    sm = np.ones(6, np.int32)

    def run(ctx):
        b = N.Batch(ctx, mats)
        s = sb0.copy()
        N.sa_run_batched(b, reads, s, betas, mcs, seed=6)
        np.testing.assert_array_equal(s, want_b)
        dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
        t = t0.copy()
        e = np.zeros((8, T))
        N.sqa_run(dg, t, 1.0, sb, ss, sm, seed=2, kernel="bitpacked", energies=e)
        assert np.isfinite(e).all()

    assert _each_allocation_fails(run) > 5


def test_non_finite_couplings_and_bad_shapes_are_refused(ctx):
    m, _ = I.dense_ising_uniform(20, seed=1)
    A = m.toarray()
    for bad in (np.nan, np.inf):
        B = A.copy()
        B[2, 5] = B[5, 2] = bad
        g = O.AugCSR(B)
        with pytest.raises(N.OJError) as ei:
            N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
        assert ei.value.status == N.OJ_ERR_ARG
        with pytest.raises(N.OJError) as ei:
            N.Batch(ctx, [A, B])
        assert ei.value.status == N.OJ_ERR_ARG
    g = O.AugCSR(A)
    dg = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    for R, T in ((4, 1), (4, 0)):  # fewer than two Trotter slices
        with pytest.raises(N.OJError) as ei:
            N.sqa_run(dg, np.ones((R, max(T, 1), g.n), np.int8)[:, :T, :], 1.0, [1.0], [0.5], [1], seed=1)
        assert ei.value.status == N.OJ_ERR_ARG
    with pytest.raises(N.OJError) as ei:  # replica_offset not a multiple of 32
        N.sa_run(dg, np.ones((4, g.n), np.int8), [1.0], [1], seed=1, replica_offset=5)
    assert ei.value.status == N.OJ_ERR_ARG
    with pytest.raises(N.OJError) as ei:  # negative beta
        N.sa_run(dg, np.ones((4, g.n), np.int8), [-1.0], [1], seed=1)
    assert ei.value.status == N.OJ_ERR_ARG
