"""Batched uneven-size dense SA (oj_sa_run_batched) against its CPU replay,
spin for spin, through the C ABI."""
import numpy as np
import pytest

from openjij_b200 import _native as N
from openjij_b200 import instances as I
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _int_batch(sizes, seed):
    return [I.dense_qubo_int(int(n), seed=seed + k)[0].toarray() for k, n in enumerate(sizes)]


def _normal_batch(sizes, seed):
    return [I.dense_qubo_normal(int(n), seed=seed + k)[0].toarray() for k, n in enumerate(sizes)]


def _spins(mats, reads, seed):
    total = sum(r * (m.shape[0] - 1) for r, m in zip(reads, mats))
    return np.random.default_rng(seed).choice(np.array([-1, 1], np.int8), size=total)


def _per_sweep(betas, mcs):
    return np.repeat(np.asarray(betas, np.float64), mcs).astype(np.float32)


def _energies(mats, reads, spins):
    out, off = [], 0
    for m, r in zip(mats, reads):
        n = m.shape[0] - 1
        g = O.AugCSR(m)
        for q in range(r):
            out.append(O.energy(g, spins[off + q * n: off + (q + 1) * n]))
        off += r * n
    return np.array(out)


def _wide_int_batch(sizes, seed):
    """Integer couplings up to 225 in magnitude: exact FP32 fields and FP16 flip
    rows, but past the int8 range of the dp4a initial fields."""
    return [I.dense_qubo_int(int(n), lo=-900, hi=900, seed=seed + k)[0].toarray() for k, n in enumerate(sizes)]


@pytest.mark.parametrize("kind", ["integer", "normal", "wide"])
def test_batched_bit_exact(ctx, kind):
    """Spins and energies against the replay: integer couplings (int8 initial
    fields, FP16 rows), wide integers (FP32 initial fields, FP16 rows) and
    N(0, 1) couplings (FP32 throughout)."""
    sizes = [1, 7, 64, 130, 300, 1024, 255, 129]
    reads = [1, 3, 8, 9, 17, 2, 0, 33]
    make = {"integer": (_int_batch, 40), "normal": (_normal_batch, 50), "wide": (_wide_int_batch, 45)}[kind]
    mats = make[0](sizes, make[1])
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 10.0, 30)
    s0 = _spins(mats, reads, 1)
    s = s0.copy()
    e = np.zeros(sum(reads))
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=77, energies=e)
    assert st["launches"] >= 2 and st["attempts"] == sum(r * n for r, n in zip(reads, sizes)) * 30
    ref = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 77)
    np.testing.assert_array_equal(s, ref)
    want = _energies(mats, reads, ref)
    np.testing.assert_allclose(e, want, rtol=1e-12, atol=1e-9)


def test_batched_split_over_calls_and_instances(ctx):
    """Sweeps split over two calls (first_sweep) and instances split over two
    batches (instance_offset) reproduce the single run."""
    sizes = [90, 200, 33, 140]
    reads = [5, 3, 8, 2]
    mats = _int_batch(sizes, 60)
    betas, mcs = I.geometric_betas(0.2, 5.0, 20)
    s0 = _spins(mats, reads, 2)
    whole = s0.copy()
    N.sa_run_batched(N.Batch(ctx, mats), reads, whole, betas, mcs, seed=5)
    cut = reads[0] * sizes[0] + reads[1] * sizes[1]
    a, b = s0[:cut].copy(), s0[cut:].copy()
    ba, bb = N.Batch(ctx, mats[:2]), N.Batch(ctx, mats[2:])
    for part, bt, off, rd in ((a, ba, 0, reads[:2]), (b, bb, 2, reads[2:])):
        N.sa_run_batched(bt, rd, part, betas[:7], mcs[:7], seed=5, instance_offset=off)
        N.sa_run_batched(bt, rd, part, betas[7:], mcs[7:], seed=5, instance_offset=off,
                         first_sweep=int(np.sum(mcs[:7])))
    np.testing.assert_array_equal(np.concatenate([a, b]), whole)


def test_batched_device_pointers(ctx):
    import torch
    sizes, reads = [100, 260], [4, 6]
    mats = _normal_batch(sizes, 70)
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 3.0, 10)
    s0 = _spins(mats, reads, 3)
    sd = torch.from_numpy(s0.copy()).cuda()
    ed = torch.zeros(sum(reads), dtype=torch.float64, device="cuda")
    N.sa_run_batched(b, reads, sd, betas, mcs, seed=9, energies=ed, device=True)
    ctx.synchronize()
    ref = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 9)
    np.testing.assert_array_equal(sd.cpu().numpy(), ref)
    np.testing.assert_allclose(ed.cpu().numpy(), _energies(mats, reads, ref), rtol=1e-12, atol=1e-9)


def test_batched_rejects_bad_input(ctx):
    big = np.zeros((4098, 4098))  # n = 4097 > 4096
    big[-1, -1] = 1.0
    with pytest.raises(N.OJError) as ei:
        N.Batch(ctx, [big])
    assert ei.value.status == N.OJ_ERR_ARG
    asym = _int_batch([5], 1)[0]
    asym[0, 1] += 1.0
    with pytest.raises(N.OJError) as ei:
        N.Batch(ctx, [asym])
    assert ei.value.status == N.OJ_ERR_ARG
    b = N.Batch(ctx, _int_batch([5], 1))
    with pytest.raises(N.OJError):
        N.sa_run_batched(b, [-1], np.zeros(5, np.int8), [1.0], [1], seed=1)
    # no replicas at all: nothing runs
    N.sa_run_batched(b, [0], np.zeros(0, np.int8), [1.0], [1], seed=1)


@pytest.mark.parametrize("n,R,kind", [(50, 3, "integer"), (300, 17, "normal"), (2048, 8, "integer"),
                                      (4096, 2, "normal")])
def test_dense_jump_kernel_bit_exact(ctx, n, R, kind):
    """oj_sa_run with OJ_KERNEL_DENSE_JUMP (the batched kernel on one graph)
    against the batched replay of that single instance."""
    A = (I.dense_qubo_int(n, seed=n) if kind == "integer" else I.dense_qubo_normal(n, seed=n))[0].toarray()
    g = N.Graph(ctx, *I.augmented_csr(A))
    betas, mcs = I.geometric_betas(0.1, 5.0, 4 if n >= 2048 else 20)
    s0 = np.random.default_rng(n).choice(np.array([-1, 1], np.int8), size=(R, n))
    s = s0.copy()
    e = np.zeros(R)
    st = N.sa_run(g, s, betas, mcs, seed=31, kernel="dense_jump", energies=e)
    assert st["kernel"] == "dense_jump"
    ref = O.replay_sa_batch([A], [R], s0.ravel(), _per_sweep(betas, mcs), 31).reshape(R, n)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_allclose(e, _energies([A], [R], ref.ravel()), rtol=1e-12, atol=1e-9)


def test_dense_jump_replica_shards(ctx):
    A = I.dense_qubo_normal(200, seed=5)[0].toarray()
    g = N.Graph(ctx, *I.augmented_csr(A))
    betas, mcs = I.geometric_betas(0.1, 5.0, 15)
    s0 = np.random.default_rng(9).choice(np.array([-1, 1], np.int8), size=(64, 200))
    whole = s0.copy()
    N.sa_run(g, whole, betas, mcs, seed=3, kernel="dense_jump")
    part = s0[32:].copy()
    N.sa_run(g, part, betas, mcs, seed=3, kernel="dense_jump", replica_offset=32)
    np.testing.assert_array_equal(part, whole[32:])


_VARIANT_MAX_N = {45: 4096, 82: 4096, 83: 4096, 84: 4096, 162: 3456, 321: 1664}


@pytest.mark.parametrize("variant", sorted(_VARIANT_MAX_N))
@pytest.mark.parametrize("kind", ["integer", "normal"])
def test_batched_launch_variants_same_bits(ctx, monkeypatch, variant, kind):
    """Every launch variant, with FP16 rows (integer couplings) or FP32 rows,
    gives the replay's spins and energies; the batch's largest instance is the
    variant's shared-memory limit (up to 2048 sites)."""
    monkeypatch.setenv("OJ_BATCH_VARIANT", str(variant))
    top = min(_VARIANT_MAX_N[variant], 2048)
    sizes = [top, 1, 7, 130, 300, 255, 129]
    reads = [3, 1, 8, 9, 2, 0, 33]
    mats = _int_batch(sizes, 60) if kind == "integer" else _normal_batch(sizes, 70)
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.05, 5.0, 6)
    s0 = _spins(mats, reads, 5)
    s = s0.copy()
    e = np.zeros(sum(reads))
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=91, energies=e)
    assert st["variant"] == variant
    ref = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 91)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_allclose(e, _energies(mats, reads, ref), rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("variant", [45, 82, 83, 162, 321])
@pytest.mark.parametrize("kind,sizes", [("normal", [1, 7, 64, 100, 128]), ("integer", [1, 7, 64, 100, 128]),
                                        ("integer", [150, 192, 5])])
def test_batched_small_instances_staged_couplings(ctx, monkeypatch, variant, kind, sizes):
    """Batches whose largest block of couplings fits the shared-memory budget
    (FP32 rows up to n = 128, FP16 rows up to n = 192): every work item copies
    its instance's couplings to shared memory and the flips read them there;
    up to 128 sites the one-chunk kernel keeps fields and spins in registers."""
    monkeypatch.setenv("OJ_BATCH_VARIANT", str(variant))
    reads = [5, 3, 9, 2, 33][:len(sizes)]
    mats = _int_batch(sizes, 80) if kind == "integer" else _normal_batch(sizes, 90)
    b = N.Batch(ctx, mats)
    betas, mcs = I.geometric_betas(0.1, 10.0, 40)
    s0 = _spins(mats, reads, 9)
    s = s0.copy()
    e = np.zeros(sum(reads))
    st = N.sa_run_batched(b, reads, s, betas, mcs, seed=23, energies=e)
    assert st["variant"] == variant
    ref = O.replay_sa_batch(mats, reads, s0, _per_sweep(betas, mcs), 23)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_allclose(e, _energies(mats, reads, ref), rtol=1e-12, atol=1e-9)


def test_dense_jump_small_dense_ising(ctx):
    """The dense jump path on a 100-spin dense Ising instance (staged FP32
    couplings), as the 100-spin benchmark case runs it."""
    A = I.dense_ising_uniform(100, seed=1)[0].toarray()
    g = N.Graph(ctx, *I.augmented_csr(A))
    betas, mcs = I.geometric_betas(0.1, 10.0, 50)
    R = 20
    s0 = np.random.default_rng(4).choice(np.array([-1, 1], np.int8), size=(R, 100))
    s = s0.copy()
    e = np.zeros(R)
    st = N.sa_run(g, s, betas, mcs, seed=5, kernel="dense_jump", energies=e)
    assert st["kernel"] == "dense_jump"
    ref = O.replay_sa_batch([A], [R], s0.ravel(), _per_sweep(betas, mcs), 5).reshape(R, 100)
    np.testing.assert_array_equal(s, ref)
    np.testing.assert_allclose(e, _energies([A], [R], ref.ravel()), rtol=1e-12, atol=1e-9)
