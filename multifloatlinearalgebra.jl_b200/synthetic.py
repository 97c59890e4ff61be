"""Seeded synthetic multi-double workloads (the benchmark shapes).

All generators return limb-major arrays (N, m, n) or device MFMatrix objects
whose values are renormalised with exact FastTwoSum passes, so every input
satisfies the MultiFloats normalisation assumption
(docs/MULACC_X3_PROOF_CONTRACT.md:31-33 of the reference).

Lower limbs follow the workload description: limb l = randn * 2^-53 * |limb
l-1|, a fully populated low part.
"""
from __future__ import annotations

import numpy as np
import torch


def _renorm_np(X: np.ndarray) -> np.ndarray:
    """bottom-up FastTwoSum passes until none changes a limb: every adjacent
    pair then satisfies |x[l]| <= ulp(x[l-1]) / 2 (a pass can move a limb
    down and leave it overlapping the one below, so a fixed number of passes
    is not enough for four limbs)"""
    N = X.shape[0]
    for _ in range(4 * N):
        changed = False
        for lvl in range(N - 1, 0, -1):
            s = X[lvl - 1] + X[lvl]
            e = X[lvl] - (s - X[lvl - 1])
            changed = changed or not (np.array_equal(s, X[lvl - 1]) and np.array_equal(e, X[lvl]))
            X[lvl - 1], X[lvl] = s, e
        if not changed:
            break
    return X


def randn_mf(rng: np.random.Generator, N: int, m: int, n: int, spread: float = 0.0,
             scale: float = 1.0) -> np.ndarray:
    """limb0 ~ N(0,1) * 2^U(-spread, spread); lower limbs as described above."""
    X = np.zeros((N, m, n))
    X[0] = rng.standard_normal((m, n)) * scale
    if spread:
        X[0] *= np.exp2(rng.uniform(-spread, spread, (m, n)))
    for lvl in range(1, N):
        X[lvl] = rng.standard_normal((m, n)) * 2.0 ** -53 * np.abs(X[lvl - 1])
    return _renorm_np(X)


def _renorm_torch(X: torch.Tensor) -> torch.Tensor:
    N = X.shape[0]
    for _ in range(4 * N):
        changed = False
        for lvl in range(N - 1, 0, -1):
            a, b = X[lvl - 1].clone(), X[lvl].clone()
            s = a + b
            e = b - (s - a)
            changed = changed or not (torch.equal(s, a) and torch.equal(e, b))
            X[lvl - 1], X[lvl] = s, e
        if not changed:
            break
    return X


def randn_mf_device(seed: int, N: int, m: int, n: int, spread: float = 0.0,
                    device: int = 0) -> torch.Tensor:
    """Device-generated (N, n, m) limb planes (column-major) of the same
    distribution as randn_mf; used for benchmark-size inputs."""
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed)
    X = torch.empty((N, n, m), dtype=torch.float64, device=f"cuda:{device}")
    X[0].normal_(generator=g)
    if spread:
        u = torch.empty((n, m), dtype=torch.float64, device=f"cuda:{device}")
        u.uniform_(-spread, spread, generator=g)
        X[0] *= torch.exp2(u)
        del u
    for lvl in range(1, N):
        X[lvl].normal_(generator=g)
        X[lvl] *= 2.0 ** -53
        X[lvl] *= X[lvl - 1].abs()
    return _renorm_torch(X)


def spd_matrix(rng: np.random.Generator, N: int, n: int, gemm) -> np.ndarray:
    """S = R R^T + n I with R randn multi-double (config 2 / config 5 shape).
    `gemm` computes the multi-double product (oracle or device)."""
    R = randn_mf(rng, N, n, n)
    S = gemm(R, np.ascontiguousarray(R.transpose(0, 2, 1)))
    S[0] += n * np.eye(n)
    return _renorm_np(S)


def _two_prod_torch(a: torch.Tensor, b: torch.Tensor):
    """exact a*b = p + e with Veltkamp splitting (elementwise IEEE operations)"""
    c = 134217729.0
    p = a * b
    ta = c * a
    ah = ta - (ta - a)
    al = a - ah
    tb = c * b
    bh = tb - (tb - b)
    bl = b - bh
    e = ((ah * bh - p) + ah * bl + al * bh) + al * bl
    return p, e


def mixed_lu_problem(mf, n: int, nrhs: int, seed: int = 4, N: int = 4, device: int = 0):
    """A = U diag(sigma) V^T with U, V orthogonal (QR of randn), sigma geometric
    from 1 to 1e-12, lifted to Float64xN: W = diag(sigma) V^T exactly (two
    limbs, exact products), A = U W with the multi-double GEMM.  B = randn.
    Returns device MFMatrix objects (A, B)."""
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed)
    dev = f"cuda:{device}"
    U, _ = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))
    V, _ = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))
    sigma = torch.logspace(0.0, -12.0, n, dtype=torch.float64, device=dev)
    # W = diag(sigma) V^T, column-major planes (N, n, n): W[i, j] = sigma_i V[j, i]
    p, e = _two_prod_torch(sigma[:, None], V.t().contiguous())
    Wp = torch.zeros((N, n, n), dtype=torch.float64, device=dev)
    Wp[0] = p.t()
    Wp[1] = e.t()
    Up = torch.zeros((N, n, n), dtype=torch.float64, device=dev)
    Up[0] = U.t()
    A = mf.MFMatrix.zeros(N, n, n, device=device)
    mf.gemm_(A, mf.MFMatrix.from_tensor(Up), mf.MFMatrix.from_tensor(Wp))
    Bp = torch.zeros((N, nrhs, n), dtype=torch.float64, device=dev)
    Bp[0].normal_(generator=g)
    return A, mf.MFMatrix.from_tensor(Bp)


def _symmetric_from_lower_(P: torch.Tensor) -> torch.Tensor:
    """(N, n, n) column-major planes made symmetric from their lower triangle"""
    for lvl in range(P.shape[0]):
        S = P[lvl].t()  # S[r, c]
        P[lvl].copy_(torch.tril(S) + torch.tril(S, -1).t())
    return P


def spd_matrix_device(mf, seed: int, N: int, n: int, device: int = 0):
    """S = R R^T + n I in Float64xN with R as randn_mf_device (the Cholesky
    workload's matrix), formed with the device GEMM, made symmetric from its
    lower triangle and renormalised.  Returns a device MFMatrix."""
    Rp = randn_mf_device(seed, N, n, n, device=device)
    S = mf.MFMatrix.zeros(N, n, n, device=device)
    mf.gemm_(S, mf.MFMatrix.from_tensor(Rp),
             mf.MFMatrix.from_tensor(Rp.transpose(1, 2).contiguous()))
    del Rp
    P = _symmetric_from_lower_(S.storage)
    P[0].diagonal().add_(float(n))
    _renorm_torch(P)
    return S


def randn_planes_device(seed: int, N: int, length: int, device: int = 0) -> torch.Tensor:
    """(N, length) planes: limb 0 ~ N(0,1), limb l = randn 2^-53 |limb l-1|,
    renormalised"""
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed)
    X = torch.empty((N, max(length, 1)), dtype=torch.float64, device=f"cuda:{device}")
    X[0].normal_(generator=g)
    for lvl in range(1, N):
        X[lvl].normal_(generator=g)
        X[lvl] *= 2.0 ** -53
        X[lvl] *= X[lvl - 1].abs()
    return _renorm_torch(X)


def spd_batch_fill(mf, batch, seed: int = 5) -> None:
    """Fill an SPDBatch with the batched workload: S_i = R_i R_i^T + n_i I in
    Float64xN, R_i n_i x n_i randn with populated lower limbs (product by the
    device GEMM, symmetric from its lower triangle, renormalised), and one
    randn right-hand side b_i with populated lower limbs per block."""
    N, dev = batch.N, batch.device
    R = randn_planes_device(seed, N, batch.total_s, device=dev)
    sizes, offs = batch.sizes_host, batch.offsets_host
    for i in range(batch.nblocks):
        ni, o = int(sizes[i]), int(offs[i])
        if ni == 0:
            continue
        Rb = R[:, o:o + ni * ni].view(N, ni, ni)
        mf.gemm_(mf.MFMatrix.from_tensor(batch.S[:, o:o + ni * ni].view(N, ni, ni)),
                 mf.MFMatrix.from_tensor(Rb), mf.MFMatrix.from_tensor(Rb.transpose(1, 2).contiguous()))
    del R
    # symmetric from the lower triangle and n_i on the diagonal, per size class
    for s in np.unique(sizes):
        s = int(s)
        if s == 0:
            continue
        idx = np.flatnonzero(sizes == s)
        cols = torch.as_tensor(offs[idx][:, None] + np.arange(s * s)[None, :], device=batch.S.device)
        blk = batch.S[:, cols].view(N, len(idx), s, s)  # [l, b, c, r]
        for lvl in range(N):
            Sb = blk[lvl].transpose(1, 2)  # [b, r, c]
            blk[lvl] = torch.tril(Sb) + torch.tril(Sb, -1).transpose(1, 2)
        blk[0].diagonal(dim1=1, dim2=2).add_(float(s))
        batch.S[:, cols] = blk.view(N, len(idx), s * s)
    _renorm_torch(batch.S)
    batch.X.copy_(randn_planes_device(seed + 1, N, batch.total_b, device=dev)[:, :batch.X.shape[1]])
