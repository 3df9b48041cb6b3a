"""The allocation-free bit-packed entry point (oj_sa_run_bitpacked_noalloc).

It serves callers that cannot call cudaMalloc while they run — an
application whose device memory is already held by another framework's
allocator, or code that cannot take cudaMalloc's implicit device
synchronisation — by keeping its scratch in a fixed device array inside the
library.  It must give exactly the spins of the regular oj_sa_run bit-packed
path, on consecutive calls that reuse (and overwrite) that array.
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
        N.sa_run_bitpacked_noalloc(graph, got, betas, mcs, seed=seed)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: allocation-free run differs from oj_sa_run"
        assert not torch.equal(got, init)

    # a schedule whose thresholds exceed the fixed scratch is rejected before any work
    spins = init.clone()
    with pytest.raises(N.OJError) as ei:
        N.sa_run_bitpacked_noalloc(graph, spins, [1.0], [900000], seed=1)
    assert ei.value.status == N.OJ_ERR_ARG
    torch.cuda.synchronize()
    assert torch.equal(spins, init)
    graph.close()
    ctx.close()
