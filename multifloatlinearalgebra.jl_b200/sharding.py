"""Multi-rank plumbing for the paths that shard (one process per GPU).

No reference counterpart: MultiFloatLinearAlgebra.jl runs in one process.
Two paths split into independent work:

* GEMM: C = A*B splits into 2-D output tiles; rank r multiplies its row panel
  of A by its column panel of B (matched order is preserved: no k split, so
  every entry is the same ascending-k chain as on one GPU).  With the
  operands on one rank (gemm_sharded_), the panels are scattered from it and
  the tiles gathered back to it; independent problems (one per rank, the
  weak-scaling benchmark) need no split and no collective at all.
* batched SPD solve: the blocks are dealt to ranks by cost (n^3/3 + 2 n^2,
  longest first onto the least loaded rank).

Factorizations of one matrix stay on one GPU (replicas only).  The host-side
agreement (the tuned modulus count, the max-over-ranks time) and the optional
gather of results use torch.distributed; the functions here take the compute
step as a callable, so the same partition and gather logic runs under the
gloo backend on CPUs and under NCCL on GPUs.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist


def _world(group=None) -> Tuple[int, int]:
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def _device(group=None) -> torch.device:
    """device for the small agreement tensors: CUDA under NCCL, else CPU"""
    if dist.is_initialized() and dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def spd_block_costs(sizes: Sequence[int]) -> np.ndarray:
    """multi-double flops of one factor + solve per block: n^3/3 + 2 n^2"""
    n = np.asarray(sizes, dtype=np.float64)
    return n ** 3 / 3.0 + 2.0 * n ** 2


def partition_by_cost(costs: Sequence[float], world: int) -> List[np.ndarray]:
    """Deal items to `world` ranks, largest cost first onto the least loaded
    rank (ties: the lower rank).  Deterministic, so every rank computes the
    same partition without communication.  Returns the item indices of each
    rank in ascending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return [np.flatnonzero(owner == r) for r in range(world)]


def tile_grid(world: int) -> Tuple[int, int]:
    """rows x columns of ranks for a 2-D split of C (as square as possible)"""
    pr = int(np.floor(np.sqrt(world)))
    while world % pr:
        pr -= 1
    return pr, world // pr


def gemm_tile(m: int, n: int, world: int, rank: int) -> Tuple[slice, slice]:
    """row and column ranges of C that `rank` computes (balanced blocks)"""
    pr, pc = tile_grid(world)
    i, j = divmod(rank, pc)
    rb = np.linspace(0, m, pr + 1).round().astype(int)
    cb = np.linspace(0, n, pc + 1).round().astype(int)
    return slice(int(rb[i]), int(rb[i + 1])), slice(int(cb[j]), int(cb[j + 1]))


def agree(value: int, group=None, src: int = 0) -> int:
    """the value of rank `src` on every rank (e.g. the tuned modulus count,
    so that every rank runs the same route)"""
    world, _ = _world(group)
    if world == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=_device(group))
    dist.broadcast(t, src, group=group)
    return int(t.item())


def max_over_ranks(t: float, group=None) -> float:
    """the largest of the ranks' values (device times of one timed region)"""
    world, _ = _world(group)
    if world == 1:
        return float(t)
    x = torch.tensor([float(t)], dtype=torch.float64, device=_device(group))
    dist.all_reduce(x, op=dist.ReduceOp.MAX, group=group)
    return float(x.item())


def gemm_sharded(A: np.ndarray, B: np.ndarray,
                 multiply: Callable[[np.ndarray, np.ndarray], np.ndarray],
                 group=None, gather: bool = True) -> np.ndarray:
    """C = A*B split into 2-D output tiles over the ranks of `group`.

    A (N, m, k) and B (N, k, n) are limb-major arrays every rank holds (or can
    slice); `multiply(A_rows, B_cols)` computes one tile on this rank's device
    (the device GEMM, or the oracle in CPU tests).  Returns the full C on
    every rank when `gather`, else this rank's tile."""
    world, rank = _world(group)
    m, n = A.shape[1], B.shape[2]
    rs, cs = gemm_tile(m, n, world, rank)
    tile = np.ascontiguousarray(multiply(np.ascontiguousarray(A[:, rs, :]),
                                         np.ascontiguousarray(B[:, :, cs])))
    if not gather or world == 1:
        return tile
    return _gather_tiles(tile, A.shape[0], m, n, world, group)


def _gather_tiles(tile: np.ndarray, N: int, m: int, n: int, world: int, group) -> np.ndarray:
    pr, pc = tile_grid(world)
    mr = -(-m // pr) + 1
    nc = -(-n // pc) + 1
    buf = np.zeros((N, mr, nc))
    buf[:, :tile.shape[1], :tile.shape[2]] = tile
    dev = _device(group)
    parts = [torch.zeros((N, mr, nc), dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(parts, torch.from_numpy(buf).to(dev), group=group)
    C = np.zeros((N, m, n))
    for r in range(world):
        rs, cs = gemm_tile(m, n, world, r)
        C[:, rs, cs] = parts[r].cpu().numpy()[:, :rs.stop - rs.start, :cs.stop - cs.start]
    return C


def solve_spd_sharded(sizes: Sequence[int], solve_blocks: Callable[[np.ndarray], List[np.ndarray]],
                      group=None, gather: bool = True) -> Optional[List[np.ndarray]]:
    """Batched SPD solve with the blocks dealt to ranks by cost.

    `solve_blocks(indices)` solves the blocks `indices` on this rank (the
    batched device kernel, or the oracle in CPU tests) and returns their
    solutions (N, n_i) in the same order.  With `gather`, every rank gets
    the list of all solutions in block order; otherwise None on every rank
    and each keeps its own results."""
    world, rank = _world(group)
    parts = partition_by_cost(spd_block_costs(sizes), world)
    mine = parts[rank]
    local = solve_blocks(mine)
    if not gather:
        return None
    if world == 1:
        return list(local)
    N = local[0].shape[0] if len(local) else 0
    N = agree(max(N, 0), group, src=int(np.argmax([len(p) for p in parts])))
    lens = [int(np.sum(np.asarray(sizes)[p])) for p in parts]
    width = max(lens) if lens else 0
    buf = np.zeros((N, max(width, 1)))
    o = 0
    for x in local:
        buf[:, o:o + x.shape[1]] = x
        o += x.shape[1]
    dev = _device(group)
    got = [torch.zeros_like(torch.from_numpy(buf)).to(dev) for _ in range(world)]
    dist.all_gather(got, torch.from_numpy(buf).to(dev), group=group)
    out: List[Optional[np.ndarray]] = [None] * len(sizes)
    for r in range(world):
        flat = got[r].cpu().numpy()
        o = 0
        for i in parts[r]:
            ni = int(sizes[i])
            out[i] = flat[:, o:o + ni].copy()
            o += ni
    return out


def gemm_sharded_(C, A, B, alpha=1.0, beta=0.0, config=None, group=None, root: int = 0,
                  multiply: Optional[Callable] = None):
    """C = alpha A B + beta C over the ranks of `group`, with the operands
    resident on `root` as limb-plane tensors (the storage of an MFMatrix:
    A (N, k, m), B (N, n, k), C (N, n, m), column-major planes); the other
    ranks pass None for A, B and C.

    1. The shapes are broadcast from root; the row panel of A and the column
       panel of B of every rank's 2-D output tile (gemm_tile) are scattered
       from root, zero-padded to one size (one scatter collective each, over
       NCCL on GPUs: the transfers are plain device buffers, no kernel reads
       another GPU's memory); with beta != 0 the C tiles are scattered too.
    2. Every rank multiplies its tile: multiply(Ap, Bp, Ct) with the panels
       and the tile as views of the padded buffers (MFMatrix objects on a
       GPU; by default gemm_(Ct, Ap, Bp, alpha, beta, config), so each entry
       is the same ascending-k chain as on one GPU: no k split, the matched
       order is kept).  CPU tests pass the oracle instead.
    3. The tiles are gathered to root and written into C.

    Returns C on root, None on the other ranks."""
    world, rank = _world(group)
    # the collectives' device (CUDA under NCCL, the CPU under gloo); one rank
    # without a process group keeps the operands where they are
    dev = _device(group) if world > 1 else A.device
    if rank == root:
        N, k, m = (int(x) for x in A.shape)
        n = int(B.shape[1])
        if B.shape[0] != N or B.shape[2] != k or tuple(C.shape) != (N, n, m):
            raise ValueError("gemm_sharded_: operand shapes differ")
        hdr = torch.tensor([N, m, k, n, int(beta != 0)], dtype=torch.int64, device=dev)
    else:
        hdr = torch.zeros(5, dtype=torch.int64, device=dev)
    if world > 1:
        dist.broadcast(hdr, root, group=group)
    N, m, k, n, use_beta = (int(x) for x in hdr.tolist())
    pr, pc = tile_grid(world)
    rmax, cmax = max(-(-m // pr), 1), max(-(-n // pc), 1)
    tiles = [gemm_tile(m, n, world, r) for r in range(world)]
    f64 = torch.float64

    def scatter(make_part, shape):
        mine = torch.zeros(shape, dtype=f64, device=dev)
        parts = None
        if rank == root:
            parts = []
            for r in range(world):
                buf = torch.zeros(shape, dtype=f64, device=dev)
                make_part(buf, *tiles[r])
                parts.append(buf)
        if world > 1:
            dist.scatter(mine, parts, src=root, group=group)
        else:
            mine.copy_(parts[0])
        return mine

    def a_part(buf, rs, cs):
        buf[:, :, :rs.stop - rs.start] = A[:, :, rs]

    def b_part(buf, rs, cs):
        buf[:, :cs.stop - cs.start, :] = B[:, cs, :]

    def c_part(buf, rs, cs):
        buf[:, :cs.stop - cs.start, :rs.stop - rs.start] = C[:, cs, rs]

    a_mine = scatter(a_part, (N, max(k, 1), rmax))
    b_mine = scatter(b_part, (N, cmax, max(k, 1)))
    c_mine = scatter(c_part, (N, cmax, rmax)) if use_beta else \
        torch.zeros((N, cmax, rmax), dtype=f64, device=dev)
    rs, cs = tiles[rank]
    rows, cols = rs.stop - rs.start, cs.stop - cs.start
    if multiply is None:
        from . import KernelConfig, MFMatrix, gemm_
        Ap = MFMatrix(a_mine, 0, 0, rows, k)
        Bp = MFMatrix(b_mine, 0, 0, k, cols)
        Ct = MFMatrix(c_mine, 0, 0, rows, cols)
        gemm_(Ct, Ap, Bp, alpha, beta, config=config if config is not None else KernelConfig())
    else:
        multiply(a_mine[:, :k, :rows], b_mine[:, :cols, :k], c_mine[:, :cols, :rows])
    parts = [torch.zeros_like(c_mine) for _ in range(world)] if rank == root else None
    if world > 1:
        dist.gather(c_mine, parts, dst=root, group=group)
    else:
        parts[0].copy_(c_mine)
    if rank != root:
        return None
    for r, (rs_r, cs_r) in enumerate(tiles):
        C[:, cs_r, rs_r] = parts[r][:, :cs_r.stop - cs_r.start, :rs_r.stop - rs_r.start]
    return C
