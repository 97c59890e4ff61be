"""Batched SPD factor + solve in one persistent launch, its CUDA-graph replay
and its adjoint (finite differences in Float64x4 and an mpmath reference
gradient)."""
import numpy as np
import pytest
import torch

from conftest import assert_bitwise
from test_oracle import syn

pytestmark = pytest.mark.gpu


def _spd_blocks(ref, rng, N, sizes):
    out = []
    for n in sizes:
        S = syn.spd_matrix(rng, N, int(n), ref.gemm)
        out.append(np.tril(S) + np.transpose(np.tril(S, -1), (0, 2, 1)))
    return out


@pytest.mark.parametrize("N", [2, 3, 4])
def test_batched_matches_single_block_oracle(mf, ref, rng, N):
    sizes = rng.integers(1, 70, 23)
    sizes[3] = 300  # one block larger than the CTA (two rows per thread)
    blocks = _spd_blocks(ref, rng, N, sizes)
    rhs = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    batch = mf.batched.SPDBatch(N, sizes)
    for i, (S, b) in enumerate(zip(blocks, rhs)):
        batch.set_block(i, S)
        batch.set_rhs(i, b)
    info = mf.batched.potrf_potrs_batched_(batch)
    assert np.all(info == 0)
    for i, (S, b) in enumerate(zip(blocks, rhs)):
        L, inf = ref.potrf(S)
        assert inf == 0
        assert_bitwise(np.tril(batch.block(i)), np.tril(L), f"factor {i}")
        assert_bitwise(batch.rhs(i), ref.potrs(L, b[:, :, None])[:, :, 0], f"solve {i}")


def test_batched_failure_is_per_block(mf, ref, rng):
    N = 2
    sizes = np.array([5, 6, 7])
    blocks = _spd_blocks(ref, rng, N, sizes)
    blocks[1][0, 2, 2] = -50.0  # not positive definite at column 3
    batch = mf.batched.SPDBatch(N, sizes)
    for i, S in enumerate(blocks):
        batch.set_block(i, S)
        batch.set_rhs(i, np.ones((N, sizes[i])))
    info = mf.batched.potrf_potrs_batched_(batch, check=False)
    assert info[0] == 0 and info[2] == 0 and info[1] > 0
    _, want = ref.potrf(blocks[1])
    assert info[1] == want
    with pytest.raises(mf.PosDefException):
        b2 = mf.batched.SPDBatch(N, sizes)
        for i, S in enumerate(blocks):
            b2.set_block(i, S)
        mf.batched.potrf_potrs_batched_(b2)


def test_batched_graph_replay(mf, ref, rng):
    N = 2
    sizes = rng.integers(8, 40, 50)
    blocks = _spd_blocks(ref, rng, N, sizes)
    rhs = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    batch = mf.batched.SPDBatch(N, sizes)

    def load():
        for i, (S, b) in enumerate(zip(blocks, rhs)):
            batch.set_block(i, S)
            batch.set_rhs(i, b)

    load()
    torch.cuda.synchronize()
    g = mf.batched.BatchedSPDGraph(batch)
    load()  # capture does not run the kernel; refresh and replay twice
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    first = batch.X.clone()
    load()
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(first, batch.X)
    for i in (0, 17, 49):
        L, _ = ref.potrf(blocks[i])
        assert_bitwise(batch.rhs(i), ref.potrs(L, rhs[i][:, :, None])[:, :, 0])


def _loss_x4(ref, S, b, w):
    """sum_j x_j w_j accumulated in Float64x4 (returned as 4 limbs)"""
    L, info = ref.potrf(S)
    assert info == 0
    x = ref.potrs(L, b[:, :, None])[:, :, 0]
    acc = np.zeros(4)
    for j in range(x.shape[1]):
        acc = ref.add(acc, ref.mul(np.ascontiguousarray(x[:, j]), np.ascontiguousarray(w[:, j])))
    return acc


def _fd(ref, lp, lm, h):
    """central difference (lp - lm) / (2h) in Float64x4 (4 limbs)"""
    return ref.div(ref.add(lp, -lm), np.array([2 * h, 0.0, 0.0, 0.0]))


def _close_x4(ref, got, want, rel):
    d = abs(float(ref.to_double(ref.add(got, -want)[:, None])[0]))
    return d <= rel * max(1.0, abs(float(want[0])))


def test_batched_adjoint_vs_finite_differences_x4(mf, ref, rng):
    """central differences of loss = sum_i <w_i, x_i> in Float64x4"""
    N = 4
    sizes = np.array([4, 6, 5])
    blocks = _spd_blocks(ref, rng, N, sizes)
    rhs = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    ws = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    batch = mf.batched.SPDBatch(N, sizes)
    for i, (S, b) in enumerate(zip(blocks, rhs)):
        batch.set_block(i, S)
        batch.set_rhs(i, b)
    x, pullback = mf.batched.solve_spd_batched_rrule(batch)
    wbuf = torch.zeros_like(x)
    for i, w in enumerate(ws):
        o = int(batch.boffsets_host[i])
        wbuf[:, o:o + sizes[i]] = torch.from_numpy(w).cuda()
    sb, bb = pullback(wbuf)
    h = 1e-24
    for i in range(len(sizes)):
        S, b, w = blocks[i], rhs[i], ws[i]
        n = sizes[i]
        Sbar = batch.block(i, sb)
        bbar = batch.rhs(i, bb)
        # d/db_j
        for j in range(n):
            bp, bm = b.copy(), b.copy()
            bp[:, j] = ref.add(b[:, j], np.array([h, 0, 0, 0]))
            bm[:, j] = ref.add(b[:, j], np.array([-h, 0, 0, 0]))
            fd = _fd(ref, _loss_x4(ref, S, bp, w), _loss_x4(ref, S, bm, w), h)
            assert _close_x4(ref, fd, np.ascontiguousarray(bbar[:, j]), 1e-30)
        # symmetric perturbation of S_jk and S_kj
        for (j, k) in [(0, 0), (1, 0), (n - 1, 2), (n - 1, n - 1)]:
            E = np.zeros((N, n, n))
            E[0, j, k] = h
            E[0, k, j] = h
            Sp, Sm = ref.add_n(S, E), ref.add_n(S, -E)
            fd = _fd(ref, _loss_x4(ref, Sp, b, w), _loss_x4(ref, Sm, b, w), h)
            sjk = np.ascontiguousarray(Sbar[:, j, k])
            want = sjk if j == k else ref.add(sjk, np.ascontiguousarray(Sbar[:, k, j]))
            assert _close_x4(ref, fd, want, 1e-30)


def test_batched_adjoint_vs_mpmath_gradient(mf, ref, rng):
    """Float64x2 gradient against a 300-digit mpmath gradient"""
    import mpmath
    N = 2
    sizes = np.array([5, 8])
    blocks = _spd_blocks(ref, rng, N, sizes)
    rhs = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    ws = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    batch = mf.batched.SPDBatch(N, sizes)
    for i, (S, b) in enumerate(zip(blocks, rhs)):
        batch.set_block(i, S)
        batch.set_rhs(i, b)
    x, pullback = mf.batched.solve_spd_batched_rrule(batch)
    wbuf = torch.zeros_like(x)
    for i, w in enumerate(ws):
        o = int(batch.boffsets_host[i])
        wbuf[:, o:o + sizes[i]] = torch.from_numpy(w).cuda()
    sb, bb = pullback(wbuf)
    mpmath.mp.dps = 300
    mpv = lambda limbs: sum(mpmath.mpf(float(v)) for v in limbs)
    for i, n in enumerate(sizes):
        S = mpmath.matrix([[mpv(blocks[i][:, r, c]) for c in range(n)] for r in range(n)])
        b = mpmath.matrix([mpv(rhs[i][:, r]) for r in range(n)])
        w = mpmath.matrix([mpv(ws[i][:, r]) for r in range(n)])
        xs = mpmath.lu_solve(S, b)
        bbar = mpmath.lu_solve(S, w)
        got_b = batch.rhs(i, bb)
        got_S = batch.block(i, sb)
        for r in range(n):
            assert abs(mpv(got_b[:, r]) - bbar[r]) <= 1e-28 * (1 + abs(bbar[r]))
            for c in range(n):
                want = -(bbar[r] * xs[c] + xs[r] * bbar[c]) / 2
                assert abs(mpv(got_S[:, r, c]) - want) <= 1e-28 * (1 + abs(want))


@pytest.mark.parametrize("threads", [64, 512])
def test_batched_block_above_max_size_is_refused(mf, ref, rng, threads):
    """max_size sizes each CTA's shared row buffer: a block larger than the
    declared max_size is skipped with info = -1 and left untouched, the
    others are factored and solved as usual"""
    N = 2
    sizes = np.array([12, 40, 9])
    blocks = _spd_blocks(ref, rng, N, sizes)
    batch = mf.batched.SPDBatch(N, sizes)
    for i, S in enumerate(blocks):
        batch.set_block(i, S)
        batch.set_rhs(i, np.ones((N, sizes[i])))
    S_before = batch.block(1)
    lib = mf._native.load()
    rc = lib.mflab_spd_batched_ex(
        mf._handle(batch.device), torch.cuda.current_stream().cuda_stream, N, batch.nblocks, 12,
        batch.sizes.data_ptr(), batch.offsets.data_ptr(), batch.boffsets.data_ptr(),
        batch.order.data_ptr(), batch.S.data_ptr(), batch.S.shape[1], batch.X.data_ptr(),
        batch.X.shape[1], 16, 1, batch.info.data_ptr(), batch.counter.data_ptr(), 2, threads)
    assert rc == 0
    info = batch.info[:3].cpu().numpy()
    assert info[0] == 0 and info[1] == -1 and info[2] == 0
    assert_bitwise(batch.block(1), S_before, "refused block untouched")
    for i in (0, 2):
        L, _ = ref.potrf(blocks[i])
        assert_bitwise(np.tril(batch.block(i)), np.tril(L), f"factor {i}")
        assert_bitwise(batch.rhs(i), ref.potrs(L, np.ones((N, sizes[i], 1)))[:, :, 0],
                       f"solve {i}")


@pytest.mark.parametrize("N", [2, 4])
def test_batched_launch_shapes_bitwise(mf, ref, rng, N):
    """every CTA size and persistent-CTA count the autotuner may pick gives the
    same factors, solutions and adjoint bit for bit (blocks up to 500, so the
    64-thread CTA holds eight rows per thread); the tuner returns one of them"""
    sizes = rng.integers(1, 90, 30)
    sizes[5], sizes[11] = 500, 260
    blocks = _spd_blocks(ref, rng, N, sizes)
    rhs = [syn.randn_mf(rng, N, int(n), 1)[:, :, 0] for n in sizes]
    outs = []
    for threads, grid in [(256, 0), (128, 7), (512, 3), (128, 0), (512, 148), (64, 5),
                          (64, 148 * 32)]:
        batch = mf.batched.SPDBatch(N, sizes)
        for i, (S, b) in enumerate(zip(blocks, rhs)):
            batch.set_block(i, S)
            batch.set_rhs(i, b)
        x, pullback = mf.batched.solve_spd_batched_rrule(
            batch, tuning={"threads": threads, "grid": grid})
        w = torch.ones_like(x)
        sb, bb = pullback(w)
        outs.append((batch.S.cpu().numpy(), x.cpu().numpy(), sb.cpu().numpy(),
                     bb.cpu().numpy()))
    for o in outs[1:]:
        for a, b in zip(outs[0], o):
            assert_bitwise(a, b, "launch shape")
    batch = mf.batched.SPDBatch(N, sizes)
    for i, (S, b) in enumerate(zip(blocks, rhs)):
        batch.set_block(i, S)
        batch.set_rhs(i, b)
    S_before = batch.S.clone()
    t = mf.batched.autotune(batch, reps=1)
    # 30 blocks: every persistent-CTA count clamps to 30, one shape per CTA size
    assert t["threads"] in (64, 128, 256, 512) and t["grid"] == 30 and len(t["timings"]) == 4
    assert torch.equal(batch.S, S_before), "autotune must restore the batch"
    info = mf.batched.potrf_potrs_batched_(batch, tuning="auto")
    assert np.all(info == 0)
    assert_bitwise(batch.S.cpu().numpy(), outs[0][0], "tuned launch")
