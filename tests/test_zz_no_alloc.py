"""The allocation-free bit-packed entry point (oj_sa_run_bitpacked_noalloc).

It serves callers that cannot call cudaMalloc while they run — an
application whose device memory is already held by another framework's
allocator, or code that cannot take cudaMalloc's implicit device
synchronisation — by keeping its scratch in a fixed device array inside the
library.  It must give exactly the spins of the regular oj_sa_run bit-packed
path, on consecutive calls that reuse (and overwrite) that array, without the
device's free memory moving across a call, and it must refuse what it cannot
run before touching the spins.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    from openjij_b200 import _native as N
    from openjij_b200 import instances as I
    from oracle import oracle as O

    ctx = N.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    m, _ = I.lattice_pm_j(32, seed=12)
    g = O.AugCSR(m)
    graph = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    betas, mcs = I.geometric_betas(0.1, 5.0, 60)
    R = 96
    rng = np.random.default_rng(7)
    init = torch.from_numpy(rng.choice(np.array([-1, 1], np.int8), size=(R, g.n))).cuda()

    for call, seed in enumerate([31, 32]):
        want = init.clone()
        N.sa_run(graph, want, betas, mcs, seed=seed, kernel="bitpacked", device=True)
        got = init.clone()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        N.sa_run_bitpacked_noalloc(graph, got, betas, mcs, seed=seed)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert free_after == free_before, f"call {call}: device free memory moved by {free_before - free_after} B"
        assert torch.equal(got, want), f"call {call}: allocation-free run differs from oj_sa_run"
        assert not torch.equal(got, init)

    # a schedule whose thresholds exceed the fixed scratch is rejected before any work
    spins = init.clone()
    with pytest.raises(N.OJError) as ei:
        N.sa_run_bitpacked_noalloc(graph, spins, [1.0], [900000], seed=1)
    assert ei.value.status == N.OJ_ERR_ARG
    torch.cuda.synchronize()
    assert torch.equal(spins, init)

    # host memory is refused
    host = init.cpu().numpy().copy()
    with pytest.raises(N.OJError) as ei:
        N.sa_run_bitpacked_noalloc(graph, host, betas, mcs, seed=1)
    assert ei.value.status == N.OJ_ERR_ARG
    np.testing.assert_array_equal(host, init.cpu().numpy())

    # a graph that has not run oj_sa_run yet has no site partition
    fresh = N.Graph(ctx, g.n, g.indptr, g.indices, g.data)
    with pytest.raises(N.OJError) as ei:
        N.sa_run_bitpacked_noalloc(fresh, spins, betas, mcs, seed=1)
    assert ei.value.status == N.OJ_ERR_UNSUPPORTED

    # couplings of two magnitudes are not the bit-packed kernel's +-c
    A = m.toarray()
    i, j = 0, int(np.flatnonzero(A[0, :g.n])[0])
    A[i, j] *= 2.0
    A[j, i] *= 2.0
    mixed = O.AugCSR(A)
    gm = N.Graph(ctx, mixed.n, mixed.indptr, mixed.indices, mixed.data)
    with pytest.raises(N.OJError) as ei:
        N.sa_run_bitpacked_noalloc(gm, spins, betas, mcs, seed=1)
    assert ei.value.status == N.OJ_ERR_UNSUPPORTED
    torch.cuda.synchronize()
    assert torch.equal(spins, init)

    # a stream under capture is refused (the thresholds pass through a buffer
    # that is gone when a graph would replay the copy)
    side = torch.cuda.Stream()
    ctx.set_stream(side.cuda_stream)
    cg = torch.cuda.CUDAGraph()
    with torch.cuda.graph(cg, stream=side):
        spins.add_(0)
        with pytest.raises(N.OJError) as ei:
            N.sa_run_bitpacked_noalloc(graph, spins, betas, mcs, seed=1)
    assert ei.value.status == N.OJ_ERR_UNSUPPORTED
    ctx.set_stream(stream.cuda_stream)
    del cg
    torch.cuda.synchronize()
    assert torch.equal(spins, init)
    for x in (gm, fresh, graph):
        x.close()
    ctx.close()
