"""Batched SPD factor + solve of many uneven blocks and its adjoint.

No reference counterpart: MultiFloatLinearAlgebra.jl factors one matrix per
call.  Every block here follows cholesky!(S_i) / ldiv!(x_i, F_i) of the
reference exactly (one persistent CTA per block for the factor and the
forward substitution, a group of four lanes per block for the backward
substitution), so per block the results equal the single-matrix routines.

    batch = SPDBatch(N, sizes)              # packed device storage
    batch.set_block(i, S_i); batch.set_rhs(i, b_i)
    x, pullback = solve_spd_batched_rrule(batch)
    Sbar, bbar = pullback(xbar)             # ChainRulesCore-style pullback

`BatchedSPDGraph` captures the whole solve (counter reset, the persistent
factor kernel, the backward-substitution kernel) in a CUDA graph and
replays it.  `autotune` picks the launch shape (CTA size, number of
persistent CTAs) by timing the batch itself.
"""
from __future__ import annotations

from typing import Dict, Optional, Sequence

import numpy as np
import torch

from . import _native


class SPDBatch:
    """Packed storage of nblocks SPD blocks (column-major, ld = n_i) and their
    right-hand sides, as limb planes on one device."""

    def __init__(self, N: int, sizes: Sequence[int], device: Optional[int] = None):
        from . import _same_type  # noqa: F401  (validates the package is loaded)
        if not 2 <= N <= 4:
            raise ValueError("limb count must be 2, 3 or 4")
        sizes = np.asarray(sizes, dtype=np.int64)
        if np.any(sizes < 0) or (len(sizes) and sizes.max() > 512):
            raise ValueError("block sizes must be in [0, 512]")
        self.N = N
        self.sizes_host = sizes
        self.device = torch.cuda.current_device() if device is None else device
        dev = torch.device("cuda", self.device)
        sq = sizes * sizes
        self.offsets_host = np.concatenate([[0], np.cumsum(sq)[:-1]]).astype(np.int64) if len(sizes) else sizes
        self.boffsets_host = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if len(sizes) else sizes
        self.total_s = int(sq.sum())
        self.total_b = int(sizes.sum())
        # largest blocks first: the persistent CTAs take them in this order
        self.order_host = np.argsort(-sizes, kind="stable").astype(np.int64)
        t = lambda a: torch.tensor(a, dtype=torch.int64, device=dev)
        self.sizes, self.offsets, self.boffsets, self.order = (
            t(sizes), t(self.offsets_host), t(self.boffsets_host), t(self.order_host))
        self.S = torch.zeros((N, max(self.total_s, 1)), dtype=torch.float64, device=dev)
        self.X = torch.zeros((N, max(self.total_b, 1)), dtype=torch.float64, device=dev)
        self.info = torch.zeros(max(len(sizes), 1), dtype=torch.int32, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)

    @property
    def nblocks(self) -> int:
        return len(self.sizes_host)

    def set_block(self, i: int, S: np.ndarray) -> None:
        """S shaped (N, n_i, n_i), limb-major"""
        n, o = int(self.sizes_host[i]), int(self.offsets_host[i])
        cm = np.ascontiguousarray(np.asarray(S, dtype=np.float64).transpose(0, 2, 1)).reshape(self.N, n * n)
        self.S[:, o:o + n * n] = torch.from_numpy(cm).to(self.S.device)

    def set_rhs(self, i: int, b: np.ndarray) -> None:
        n, o = int(self.sizes_host[i]), int(self.boffsets_host[i])
        self.X[:, o:o + n] = torch.from_numpy(np.asarray(b, dtype=np.float64).reshape(self.N, n)).to(self.X.device)

    def block(self, i: int, buf: Optional[torch.Tensor] = None) -> np.ndarray:
        n, o = int(self.sizes_host[i]), int(self.offsets_host[i])
        src = self.S if buf is None else buf
        return src[:, o:o + n * n].cpu().numpy().reshape(self.N, n, n).transpose(0, 2, 1).copy()

    def rhs(self, i: int, buf: Optional[torch.Tensor] = None) -> np.ndarray:
        n, o = int(self.sizes_host[i]), int(self.boffsets_host[i])
        src = self.X if buf is None else buf
        return src[:, o:o + n].cpu().numpy().copy()

    def flops(self) -> float:
        """multi-double operations: sum n^3/3 (factor) + 2 n^2 (two solves)"""
        n = self.sizes_host.astype(np.float64)
        return float(np.sum(n ** 3 / 3.0 + 2.0 * n * n))


def _launch(batch: SPDBatch, solve: bool, block: int, stream: Optional[int] = None,
            grid: int = 0, threads: int = 256) -> None:
    from . import _check, _handle
    lib = _native.load()
    s = torch.cuda.current_stream(batch.device).cuda_stream if stream is None else stream
    rc = lib.mflab_spd_batched_ex(_handle(batch.device), s, batch.N, batch.nblocks,
                                  int(batch.sizes_host.max()) if batch.nblocks else 0,
                                  batch.sizes.data_ptr(), batch.offsets.data_ptr(),
                                  batch.boffsets.data_ptr(), batch.order.data_ptr(),
                                  batch.S.data_ptr(), batch.S.shape[1], batch.X.data_ptr(),
                                  batch.X.shape[1], block, int(solve), batch.info.data_ptr(),
                                  batch.counter.data_ptr(), grid, threads)
    _check(rc, "spd_batched")


_TUNED: Dict[tuple, dict] = {}


def _signature(batch: SPDBatch, block: int) -> tuple:
    n = batch.sizes_host.astype(np.int64)
    return (batch.N, block, batch.nblocks, int(n.max()) if len(n) else 0, int(n.sum()),
            int((n * n).sum()))


def autotune(batch: SPDBatch, block: int = 16, candidates: Optional[Sequence] = None,
             reps: int = 2, profile=None) -> dict:
    """Launch shape of the batched factor + solve for this batch: the CTA size
    (64, 128, 256 or 512 threads) and the number of persistent CTAs (1 to 32
    per SM, at most 2048 threads per SM), picked by timing the real launch on
    the batch's own blocks (restored afterwards).  Neither knob changes any result (each block's
    arithmetic is per element in the reference order), so the choice is free.
    Cached per (limbs, block, size signature of the batch); a tuning
    profile (tuning.TuneProfile, fingerprint checked) that holds this
    signature supplies the shape without any timing.
    Returns {"threads", "grid", "ms", "timings"}."""
    if profile is not None:
        from .tuning import stored_batched_shape
        got = stored_batched_shape(profile, batch.N, block, batch.sizes_host)
        if got is not None:
            return {"threads": got["threads"], "grid": got["grid"], "ms": got["ms"],
                    "timings": {}, "source": "profile"}
    key = _signature(batch, block)
    if key in _TUNED:
        return _TUNED[key]
    if batch.nblocks == 0:
        return {"threads": 256, "grid": 0, "ms": 0.0, "timings": {}}
    sms = torch.cuda.get_device_properties(batch.device).multi_processor_count
    cands = list(candidates) if candidates is not None else [
        (nt, cps) for nt in (64, 128, 256, 512) for cps in (1, 2, 4, 8, 16, 32)
        if nt * cps <= 2048]
    S0, X0 = batch.S.clone(), batch.X.clone()
    timings = {}
    best = None
    for nt, cps in cands:
        grid = int(min(sms * cps, batch.nblocks))
        if f"{nt}x{grid}" in timings:  # the same shape (few blocks)
            continue
        times = []
        for r in range(reps + 1):
            batch.S.copy_(S0)
            batch.X.copy_(X0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _launch(batch, True, block, grid=grid, threads=nt)
            e1.record()
            e1.synchronize()
            if r > 0:
                times.append(e0.elapsed_time(e1))
        t = min(times)
        timings[f"{nt}x{grid}"] = t
        if best is None or t < best[0]:
            best = (t, nt, grid)
    batch.S.copy_(S0)
    batch.X.copy_(X0)
    del S0, X0
    res = {"threads": best[1], "grid": best[2], "ms": best[0], "timings": timings}
    _TUNED[key] = res
    return res


def _shape(batch: SPDBatch, block: int, tuning) -> tuple:
    """(threads, grid) from tuning: None = defaults, "auto" = autotune, or a
    dict as autotune returns"""
    if tuning is None:
        return 256, 0
    if tuning == "auto":
        tuning = autotune(batch, block)
    return int(tuning["threads"]), int(tuning["grid"])


def potrf_potrs_batched_(batch: SPDBatch, block: int = 16, check: bool = True,
                         tuning=None) -> np.ndarray:
    """Factor every block in place (S_i <- L_i) and overwrite every right-hand
    side with its solution.  Returns the per-block status (0 or the failing
    column, as cholesky!'s info).  tuning: None (default launch shape),
    "auto" (autotune) or an autotune result."""
    from . import PosDefException
    threads, grid = _shape(batch, block, tuning)
    _launch(batch, True, block, grid=grid, threads=threads)
    info = batch.info[:batch.nblocks].cpu().numpy().copy()
    if check and np.any(info != 0):
        bad = int(np.flatnonzero(info)[0])
        raise PosDefException(int(info[bad]))
    return info


class BatchedSPDGraph:
    """The batched factor + solve captured once in a CUDA graph and replayed
    (inputs are refreshed in place between replays).  tuning as in
    potrf_potrs_batched_ (an autotune runs before the capture)."""

    def __init__(self, batch: SPDBatch, block: int = 16, tuning=None):
        self.batch = batch
        self.threads, self.grid = _shape(batch, block, tuning)
        self.graph = torch.cuda.CUDAGraph()
        self.stream = torch.cuda.Stream(device=batch.device)
        _native.load()
        from . import _handle
        _handle(batch.device)  # create the handle before capture
        with torch.cuda.stream(self.stream):
            with torch.cuda.graph(self.graph, stream=self.stream):
                _launch(batch, True, block, stream=self.stream.cuda_stream, grid=self.grid,
                        threads=self.threads)

    def replay(self) -> None:
        self.graph.replay()


def solve_spd_batched_rrule(batch: SPDBatch, block: int = 16, tuning=None):
    """x_i = S_i^{-1} b_i for every block, with a pullback.

    Mirrors a ChainRulesCore rrule: returns (x, pullback) where x is the packed
    solution (N, total) tensor and pullback(xbar) -> (Sbar, bbar) gives, per
    block, bbar = S^{-1} xbar and Sbar = -(bbar x^T + x bbar^T)/2 (symmetric
    parametrisation), reusing the factors."""
    from . import _check, _handle
    threads, grid = _shape(batch, block, tuning)
    potrf_potrs_batched_(batch, block, tuning={"threads": threads, "grid": grid})
    x = batch.X.clone()

    def pullback(xbar: torch.Tensor):
        lib = _native.load()
        xb = xbar.clone()
        sb = torch.zeros_like(batch.S)
        rc = lib.mflab_spd_batched_adjoint_ex(
            _handle(batch.device), torch.cuda.current_stream(batch.device).cuda_stream, batch.N,
            batch.nblocks, int(batch.sizes_host.max()) if batch.nblocks else 0,
            batch.sizes.data_ptr(), batch.offsets.data_ptr(), batch.boffsets.data_ptr(),
            batch.order.data_ptr(), batch.S.data_ptr(), batch.S.shape[1], x.data_ptr(),
            xb.data_ptr(), x.shape[1], sb.data_ptr(), batch.info.data_ptr(),
            batch.counter.data_ptr(), grid, threads)
        _check(rc, "spd_batched adjoint")
        return sb, xb

    return x, pullback
