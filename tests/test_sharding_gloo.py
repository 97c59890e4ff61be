"""Multi-rank host logic on CPUs: two gloo ranks (spawned processes) run the
partition, agreement, max-over-ranks and gather steps of the sharded GEMM and
batched SPD paths, with the oracle as the per-rank compute step, and compare
with the single-process results bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import __graft_entry__
        mf = __graft_entry__.load_package()
        from oracle import mfref
        from mflab200 import sharding, synthetic as syn
        res = {}
        # agreement and max over ranks
        res["agreed"] = sharding.agree(31 if rank == 0 else 5)
        res["tmax"] = sharding.max_over_ranks(1.0 + rank)
        # sharded GEMM (same seeded operands on every rank)
        rng = np.random.default_rng(3)
        A, B = syn.randn_mf(rng, 2, 37, 29, spread=6), syn.randn_mf(rng, 2, 29, 23, spread=6)
        res["gemm"] = sharding.gemm_sharded(A, B, lambda a, b: mfref.gemm(a, b, nthreads=1))
        # batched SPD blocks dealt by cost
        sizes = [5, 17, 3, 12, 9, 1, 14, 6]
        rng = np.random.default_rng(4)
        blocks = [syn.spd_matrix(rng, 2, n, lambda x, y: mfref.gemm(x, y, nthreads=1))
                  for n in sizes]
        rhs = [syn.randn_mf(rng, 2, n, 1) for n in sizes]
        seen = []

        def solve(idx):
            out = []
            for i in idx:
                seen.append(int(i))
                L, info = mfref.potrf(blocks[i], nthreads=1)
                assert info == 0
                out.append(mfref.potrs(L, rhs[i], nthreads=1)[:, :, 0])
            return out

        res["spd"] = sharding.solve_spd_sharded(sizes, solve)
        res["mine"] = seen
        # the device data path of the GEMM split: operands on rank 0 as limb
        # planes, panels scattered, tiles gathered back (oracle as multiply)
        planes = lambda X: torch.from_numpy(np.ascontiguousarray(X.transpose(0, 2, 1)))
        rng = np.random.default_rng(5)
        A2, B2 = syn.randn_mf(rng, 2, 41, 30, spread=6), syn.randn_mf(rng, 2, 30, 26, spread=6)
        C0 = syn.randn_mf(rng, 2, 41, 26)
        for beta in (0.0, 1.0):
            def mult(a, b, c, beta=beta):
                lm = lambda t: np.ascontiguousarray(t.permute(0, 2, 1).numpy())
                got = mfref.gemm(lm(a), lm(b), lm(c), 1.0, beta, nthreads=1)
                c.copy_(torch.from_numpy(np.ascontiguousarray(got.transpose(0, 2, 1))))
            Cp = planes(C0).clone() if rank == 0 else None
            out = sharding.gemm_sharded_(Cp, planes(A2) if rank == 0 else None,
                                         planes(B2) if rank == 0 else None, 1.0, beta,
                                         multiply=mult)
            res[f"gemm_dev_beta{int(beta)}"] = None if out is None else \
                np.ascontiguousarray(out.numpy().transpose(0, 2, 1))
        np.save(os.path.join(outdir, f"rank{rank}.npy"), np.array(res, dtype=object),
                allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_partition_is_deterministic_disjoint_and_balanced(mf):
    from mflab200 import sharding
    rng = np.random.default_rng(0)
    sizes = rng.integers(8, 257, 1000)
    costs = sharding.spd_block_costs(sizes)
    for world in (1, 2, 3, 8):
        parts = sharding.partition_by_cost(costs, world)
        again = sharding.partition_by_cost(costs, world)
        assert all(np.array_equal(a, b) for a, b in zip(parts, again))
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) <= 1.02 * (sum(loads) / world) + costs.max()


def test_gemm_tiles_cover_c_once(mf):
    from mflab200 import sharding
    for world in (1, 2, 3, 4, 6, 8):
        cover = np.zeros((50, 37), dtype=int)
        for r in range(world):
            rs, cs = sharding.gemm_tile(50, 37, world, r)
            cover[rs, cs] += 1
        assert np.all(cover == 1)


def test_two_gloo_ranks_match_one_process(mf, ref, tmp_path):
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = [np.load(tmp_path / f"rank{r}.npy", allow_pickle=True).item() for r in range(world)]
    # single-process references
    from mflab200 import synthetic as syn
    rng = np.random.default_rng(3)
    A, B = syn.randn_mf(rng, 2, 37, 29, spread=6), syn.randn_mf(rng, 2, 29, 23, spread=6)
    C = ref.gemm(A, B, nthreads=1)
    sizes = [5, 17, 3, 12, 9, 1, 14, 6]
    rng = np.random.default_rng(4)
    blocks = [syn.spd_matrix(rng, 2, n, lambda x, y: ref.gemm(x, y, nthreads=1)) for n in sizes]
    rhs = [syn.randn_mf(rng, 2, n, 1) for n in sizes]
    xs = [ref.potrs(ref.potrf(b, nthreads=1)[0], r, nthreads=1)[:, :, 0]
          for b, r in zip(blocks, rhs)]
    for r in range(world):
        assert res[r]["agreed"] == 31
        assert res[r]["tmax"] == 2.0
        assert np.array_equal(res[r]["gemm"].view(np.uint64), C.view(np.uint64))
        for i in range(len(sizes)):
            assert np.array_equal(res[r]["spd"][i].view(np.uint64), xs[i].view(np.uint64))
    rng = np.random.default_rng(5)
    A2, B2 = syn.randn_mf(rng, 2, 41, 30, spread=6), syn.randn_mf(rng, 2, 30, 26, spread=6)
    C0 = syn.randn_mf(rng, 2, 41, 26)
    for beta in (0, 1):
        want = ref.gemm(A2, B2, C0.copy(), 1.0, float(beta), nthreads=1)
        assert np.array_equal(res[0][f"gemm_dev_beta{beta}"].view(np.uint64), want.view(np.uint64))
        assert res[1][f"gemm_dev_beta{beta}"] is None
    # every block was solved by exactly one rank
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(len(sizes)))
