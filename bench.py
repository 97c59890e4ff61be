"""Benchmark: Float64xN GEMM at m = n = k = 8192 on B200.

One step is one C = A*B over the full synthetic n = 8192 workload (entries
randn * 2^U(-20,20), lower limbs randn * 2^-53 * |previous limb|; seeded).
The headline path is the INT8 tensor-core GEMM for Float64x2 (modular residue
scheme; the digit-slice scheme is timed beside it at its own equal-error S);
the plain FP64 matched-order kernel is timed beside it, with the componentwise
error of both against the exact superaccumulator oracle on sampled entries.

    python bench.py [--gpus N --steps K --warmup W] [--impl mflab|reference]

Multi-GPU (torchrun): every rank multiplies its own independent n = 8192
problem (weak scaling, no data-path collective); the time is the max over
ranks.  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Float64x2/x4 GEMM GFLOP/s at n=8192, INT8-slice vs plain FP64, equal oracle error"
UNIT = "multi-double GFLOP/s (2mnk/t)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="mflab", choices=["mflab", "reference"])
    p.add_argument("--n", type=int, default=8192)
    p.add_argument("--limbs", type=int, default=2)
    p.add_argument("--route", default="auto", help="headline route: auto (ozaki if built), plain, ozaki")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--scheme", default="modular", choices=["modular", "slices"],
                   help="INT8 scheme of the headline route (modular falls back to slices when "
                        "the modulus table cannot reach the accuracy)")
    p.add_argument("--knob", type=int, default=0,
                   help="fixed modulus (modular) or slice (slices) count instead of the "
                        "equal-error search (the error at that count is still reported)")
    p.add_argument("--no-slices", action="store_true",
                   help="skip the digit-slice companion of the modular headline")
    p.add_argument("--no-x4", action="store_true", help="skip the Float64x4 companion run")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the factorization / mixed-LU / batched-SPD workloads")
    p.add_argument("--config-reps", type=int, default=3,
                   help="timed repeats (after one warm-up) of each of those workloads")
    p.add_argument("--case", default=None,
                   choices=["crt_gemm", "getrf64", "lu64_solve", "mixed_lu", "potrf", "getrf",
                            "batched"],
                   help="run one small workload (one warm-up call, then --steps calls) and "
                        "exit: the cases the ncu summaries under profiles/ are taken on "
                        "(crt_gemm: modular x2 GEMM at --n with --knob moduli; getrf64: "
                        "binary64 LU at --n; lu64_solve: its 16-RHS prepared solve; "
                        "mixed_lu: the mixed-precision solve at --n; potrf: Cholesky "
                        "Float64x--limbs at --n; getrf: LU Float64x--limbs at --n; batched: "
                        "--n Float64x--limbs SPD blocks of sizes U{8..256}, factor + solve "
                        "with --knob threads per CTA and 8 CTAs per SM)")
    p.add_argument("--split", default="replicas", choices=["replicas", "tiles"],
                   help="replicas: one independent problem per rank (weak scaling); tiles: "
                        "one problem held by rank 0, its 2-D output tiles computed by all "
                        "ranks (panels scattered, tiles gathered; strong scaling)")
    return p.parse_args()


# ------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


_NVML_CHILD = r"""
import sys, time
import pynvml as nv
nv.nvmlInit()
bus = sys.argv[1]
try:
    h = nv.nvmlDeviceGetHandleByPciBusId(bus)
except Exception:
    h = nv.nvmlDeviceGetHandleByIndex(int(sys.argv[2]))
fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
    nv.nvmlDeviceGetCurrentClocksThrottleReasons
print("max", nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM), flush=True)
while True:
    print(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), int(fn(h)), flush=True)
    time.sleep(0.005)
"""


class NvmlClockSampler:
    """Clock / throttle-reason sampling through NVML (read-only queries) every
    5 ms in a child process, so that short timed regions still get many
    samples whatever the benchmark thread holds; falls back to the
    nvidia-smi sampler when NVML is unavailable."""

    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.proc, self.fallback, self.lines = None, None, []

    def start(self):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            self.proc = subprocess.Popen([sys.executable, "-c", _NVML_CHILD, bus, str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            first = self.proc.stdout.readline().split()
            if len(first) != 2 or first[0] != "max":
                raise OSError("nvml child did not start")
            self.max_mhz = float(first[1])
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            if self.proc is not None:
                self.proc.kill()
            self.proc = None
            self.fallback = ClockSampler(self.index)
            self.fallback.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line)

    def stop(self) -> dict:
        if self.fallback is not None:
            return self.fallback.stop()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, reasons = [], set()
        for line in self.lines:
            f = line.split()
            if len(f) != 2:
                continue
            sm.append(float(f[0]))
            for name, b in self.BITS.items():
                if int(f[1]) & b:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 5 ms"}


# ------------------------------------------------------------ helpers ----
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def fp64_peak(mf, torch) -> float:
    """Measured FP64 pipe instruction rate (instr/s), DFMA probe, burst."""
    lib = mf._native.load()
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    out = torch.empty(sms * 4 * 256, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    ins = C.c_double()
    best = 0.0
    for it in (2000, 40000, 40000):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = lib.mflab_probe_fp64(s, 0, sms * 4, 256, it, out.data_ptr(), C.byref(ins))
        e1.record()
        torch.cuda.synchronize()
        assert rc == 0
        best = max(best, ins.value / (e0.elapsed_time(e1) / 1e3))
    return best


def read_traffic(kernel_key: str, scale_from_smaller: bool = False):
    """dram bytes per launch from the committed ncu summary, if present.  With
    scale_from_smaller, a key "<prefix>_n<N>" missing at this N is taken from
    the largest captured smaller N, times (N / N0)^2: for the residue GEMMs
    at a fixed modulus count the operand and result bytes grow as n^2 (the
    captures at n = 2048 and 4096 differ by 4.27x)."""
    p = os.path.join(REPO, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    found = {}
    for line in open(p):
        if line.startswith("#") or "=" not in line:
            continue
        kv = dict(x.split("=", 1) for x in line.split())
        found[kv.get("key")] = float(kv["dram_bytes_per_launch"])
    if kernel_key in found:
        return found[kernel_key]
    if not scale_from_smaller or "_n" not in kernel_key:
        return None
    prefix, n = kernel_key.rsplit("_n", 1)
    smaller = [(int(k.rsplit("_n", 1)[1]), v) for k, v in found.items()
               if k and k.rsplit("_n", 1)[0] == prefix and int(k.rsplit("_n", 1)[1]) < int(n)]
    if not smaller:
        return None
    n0, v0 = max(smaller)
    return v0 * (int(n) / n0) ** 2


def ops_per_term(N: int) -> int:
    """FP64 instructions of one acc + a*b in the matched networks
    (x2: 8 mul + 20 add; x3 fused: 99; x4: 103 mul + 124 add)."""
    return {2: 28, 3: 99, 4: 227}[N]


def cpu_sample(mfref, N, n, threads, target_s=15.0):
    """Time the oracle GEMM on a row sample of the same workload: C[:r, :] =
    A[:r, :] * B with the full k = n reduction, r chosen for ~target_s of CPU
    work.  All column panels run in parallel over `threads` host threads."""
    import numpy as np
    from importlib import import_module
    syn = import_module("mflab200.synthetic")
    rng = np.random.default_rng(11)
    B = syn.randn_mf(rng, N, n, n, spread=20)
    r, dt = 4, 0.0
    while True:
        A = syn.randn_mf(rng, N, r, n, spread=20)
        t0 = time.perf_counter()
        mfref.gemm(A, B, nthreads=threads)
        dt = time.perf_counter() - t0
        if dt >= 0.6 * target_s or r >= n:
            break
        # grow the sample towards target_s of CPU work (at least doubling)
        r = int(min(n, max(2 * r, r * target_s / max(dt, 1e-3))))
    gf = 2.0 * r * n * n / dt / 1e9
    return gf, (f"C[:{r}, :] of the n={n} x{N} GEMM (k={n}) on {threads} host threads, "
                f"{dt:.1f} s")


# -------------------------------------------------------- reference arm --
def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    from oracle import mfref
    import __graft_entry__
    __graft_entry__.load_package()
    threads = mfref.threads()
    vals = []
    sample = ""
    for step in range(args.warmup + args.steps):
        v, sample = cpu_sample(mfref, args.limbs, args.n, threads, target_s=6.0)
        if step >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded randn * 2^U(-20,20))",
        "config": {"workload": f"Float64x{args.limbs} GEMM m=n=k={args.n}", "limbs": args.limbs,
                   "n": args.n, "parallelism": f"replicas{world}"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Julia and MultiFloats.jl are not available here: the reference arm times the "
                "oracle's C++ restatement of the reference GEMM loop order (4-row SIMD x 2-column "
                "micro-tile, column panels over all host threads).",
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- main arm ----
def _check_entries(mfref, An, Bn, Cm, rows, cols):
    """exact check of entries (rows[j], cols[j]) of a device result: returns the
    componentwise relative errors |C - C_exact| / sum_k |a_ik||b_kj|"""
    import numpy as np
    Cs = Cm.planes()[:, cols, :].cpu().numpy()  # (N, s, m): column cols[j] at index j
    Csub = np.ascontiguousarray(Cs.transpose(0, 2, 1))
    Bsub = np.ascontiguousarray(Bn[:, :, cols])
    err, scale, _ = mfref.exact_gemm_check(An, Bsub, Csub, rows, np.arange(len(rows)))
    return err / scale


class Runner:
    def __init__(self, args, torch, dist, world, rank, local):
        self.args, self.torch, self.dist = args, torch, dist
        self.world, self.rank, self.local = world, rank, local
        import __graft_entry__
        self.mf = __graft_entry__.load_package()
        from importlib import import_module
        self.syn = import_module("mflab200.synthetic")
        self.sharding = import_module("mflab200.sharding")
        self.stream = torch.cuda.current_stream()

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()
        self.torch.cuda.synchronize()

    def timed(self, fn, steps, warmup):
        torch = self.torch
        for _ in range(warmup):
            fn()
        self.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        for _ in range(steps):
            fn()
        e1.record(self.stream)
        self.barrier()
        return self.sharding.max_over_ranks(e0.elapsed_time(e1) / 1e3)

    def operands(self, N, n):
        mf, syn = self.mf, self.syn
        A = mf.MFMatrix.from_tensor(syn.randn_mf_device(1000 + self.rank, N, n, n, spread=20))
        B = mf.MFMatrix.from_tensor(syn.randn_mf_device(2000 + self.rank, N, n, n, spread=20))
        return A, B

    def cfg(self, scheme, knob):
        """KernelConfig of the INT8 route: scheme "modular" (knob = moduli) or
        "slices" (knob = digit slices); knob 0 = the tuner's choice"""
        mf = self.mf
        if scheme == "modular":
            return mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular",
                                   ozaki_moduli=knob)
        return mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="slices", ozaki_slices=knob)

    def checker(self, n, A, B, Cm):
        """exact oracle check of 256 sampled entries of Cm: returns a function
        giving the max componentwise relative error of the current Cm"""
        import numpy as np
        from oracle import mfref
        rs = np.random.default_rng(5)
        rows, cols = rs.integers(0, n, 256), rs.integers(0, n, 256)
        An, Bn = A.to_numpy(), B.to_numpy()
        return lambda: float(np.max(_check_entries(mfref, An, Bn, Cm, rows, cols)))

    def accuracy_search(self, N, n, A, B, Cm, scheme, e_plain, check):
        """INT8 route errors against the exact oracle on the sampled entries:
        the knob (moduli or slices) starts at the tuner's choice, is raised
        until the route's error is no worse than the plain kernel's, then
        lowered to the smallest value that still is."""
        mf = self.mf
        last = mf.ozaki_last_moduli if scheme == "modular" else mf.ozaki_last_slices
        top = 49 if scheme == "modular" else 64
        mf.gemm_(Cm, A, B, config=self.cfg(scheme, 0))
        K0 = last()
        K = K0
        e = check()
        e_tuner = e

        def err_at(K):
            mf.gemm_(Cm, A, B, config=self.cfg(scheme, K))
            return check()

        while e > e_plain and K < min(K0 + 6, top):
            K += 1
            e = err_at(K)
        while K > 1:
            try:
                e_lo = err_at(K - 1)
            except mf.ArgumentError:  # fewer moduli than the digit width needs
                break
            if e_lo > e_plain:
                break
            K, e = K - 1, e_lo
        knob = "moduli" if scheme == "modular" else "slices"
        return {"scheme": scheme, knob: K, "plain_max_rel_err": e_plain, "ozaki_max_rel_err": e,
                f"tuner_{knob}": K0, "tuner_max_rel_err": e_tuner, "samples": 256,
                "rule": f"smallest {knob} count with INT8-route error <= plain error on the "
                        "sampled entries"}

    def phases(self, N, n, A, B, Cm, scheme, K):
        import ctypes as C
        mf = self.mf
        lib = mf._native.load()
        h = mf._handle(self.local)
        ms = (C.c_float * 4)()
        ops = C.c_double()
        one = (C.c_double * 4)(1.0)
        zero = (C.c_double * 4)()
        fn = lib.mflab_gemm_ozaki_crt_phases if scheme == "modular" else lib.mflab_gemm_ozaki_phases
        rc = fn(h, self.stream.cuda_stream, N, K, n, n, n, A.ptr(), A.ld, A.ls, B.ptr(), B.ld, B.ls,
                Cm.ptr(), Cm.ld, Cm.ls, one, zero, ms, C.byref(ops))
        assert rc == 0, rc
        return [ms[i] for i in range(4)], ops.value

    def int8_peak(self, fill=1):
        """library int8 GEMM throughput, the measured denominator of the
        tensor roofline (the route itself runs the tcgen05 kernel): fill 1 on
        uniformly distributed bytes like the route's residues, fill 0 on
        constant bytes (less switching power, so a higher clock under the
        power cap)"""
        import ctypes as C
        mf = self.mf
        lib = mf._native.load()
        ms = C.c_float()
        n, k = 8192, 16384
        rc = lib.mflab_probe_int8_gemm(mf._handle(self.local), self.stream.cuda_stream, n, n, k, 3,
                                       fill, C.byref(ms))
        assert rc == 0, rc
        return 2.0 * n * n * k / (ms.value / 1e3)


def _time_median(torch, fn, setup=None, reps=3, warmup=1):
    """median device time (CUDA events on the current stream) of fn over
    `reps` calls after `warmup` untimed ones; setup() restores the inputs
    before every call, outside the timed region.  Returns (median s, all
    times in ms, last result)."""
    times, out = [], None
    for r in range(warmup + reps):
        if setup is not None:
            setup()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        if r >= warmup:
            times.append(e0.elapsed_time(e1))
    return statistics.median(times) / 1e3, [round(t, 3) for t in times], out


def _fp64_roof(instr: float, seconds: float, peak: float) -> dict:
    """FP64-pipe roofline of a multi-double kernel sequence: FP64
    instructions of its multiply-add networks over the DFMA probe rate"""
    a = instr / seconds
    return {"bound": "fp64", "achieved": a / 1e12, "peak": peak / 1e12, "unit": "T FP64 instr/s",
            "frac": a / peak, "peak_source": "measured in this run (DFMA probe, burst)"}


def _cpu_timed(fn):
    t0 = time.perf_counter()
    out = fn()
    return time.perf_counter() - t0, out


def config_cholesky(R, torch, peak, reps):
    """Cholesky + 64-RHS solve, n = 2048, Float64x2/x3/x4 (S = R R^T + n I)"""
    import numpy as np
    mf, syn = R.mf, R.syn
    from oracle import mfref
    threads = mfref.threads()
    n, nrhs = 2048, 64
    out = {}
    for N in (2, 3, 4):
        S = syn.spd_matrix_device(mf, 70 + N, N, n)
        Bn = syn.randn_mf(np.random.default_rng(80 + N), N, n, nrhs)
        Bm = mf.MFMatrix.from_numpy(Bn)
        Sw = S.copy()
        t_f, ts_f, F = _time_median(torch, lambda: mf.cholesky_(Sw), lambda: Sw.copy_(S), reps)
        t_s, ts_s, X = _time_median(torch, lambda: mf.solve(F, Bm), None, reps)
        fast = mf.KernelConfig(solve_order="fast")
        t_sf, _, _ = _time_median(torch, lambda: mf.solve(F, Bm, config=fast), None, reps)
        # the same factorization with INT8 (modular) trailing updates between
        # 256-column panels, solved with the matched-order solves
        Sw2 = S.copy()
        ocfg = mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular", ozaki_block=256)
        t_fo, ts_fo, Fo = _time_median(torch, lambda: mf.cholesky_(Sw2, config=ocfg),
                                       lambda: Sw2.copy_(S), reps)
        Xo = mf.solve(Fo, Bm)
        # parity: exact (superaccumulator) backward errors of four columns, and
        # for Float64x2 the full factor and solve bitwise against the oracle
        Sn, Xn, Xon = S.to_numpy(), X.to_numpy(), Xo.to_numpy()
        cols = [0, 21, 42, 63]
        be = mfref.backward_error(Sn, Xn[:, :, cols], Bn[:, :, cols])
        beo = mfref.backward_error(Sn, Xon[:, :, cols], Bn[:, :, cols])
        parity = {"exact_backward_error_max": float(be.max()),
                  "int8_trailing_exact_backward_error_max": float(beo.max()),
                  "columns_checked": cols, "bound": 4096 * n * 2.0 ** (-52 * N),
                  "oracle": "superaccumulator residual ||b - S x||_inf / (||S|| ||x|| + ||b||)"}
        cpu = {}
        if N == 2:
            t_cf, (L, info) = _cpu_timed(lambda: mfref.potrf(Sn, nthreads=threads))
            t_cs, Xr = _cpu_timed(lambda: mfref.potrs(L, Bn, nthreads=threads))
            parity["bitwise_factor_and_solve_vs_oracle"] = bool(
                info == 0 and np.array_equal(np.tril(Sw.to_numpy()).view(np.uint64),
                                             np.tril(L).view(np.uint64))
                and np.array_equal(Xn.view(np.uint64), Xr.view(np.uint64)))
            cpu["all_cores"] = {"md_gflops": (n ** 3 / 3.0 + 2.0 * n * n * nrhs) / (t_cf + t_cs)
                                / 1e9, "cores": threads, "factor_s": t_cf, "solve_s": t_cs,
                                "sample": f"full n={n}, {nrhs} RHS"}
        else:
            nc = 1024
            Sc = syn.spd_matrix(np.random.default_rng(3), N, nc,
                                lambda a, b: mfref.gemm(a, b, nthreads=threads))
            Bc = syn.randn_mf(np.random.default_rng(4), N, nc, nrhs)
            t_cf, (L, _) = _cpu_timed(lambda: mfref.potrf(Sc, nthreads=threads))
            t_cs, _ = _cpu_timed(lambda: mfref.potrs(L, Bc, nthreads=threads))
            cpu["all_cores"] = {"md_gflops": (nc ** 3 / 3.0 + 2.0 * nc * nc * nrhs) / (t_cf + t_cs)
                                / 1e9, "cores": threads, "factor_s": t_cf, "solve_s": t_cs,
                                "sample": f"n={nc}, {nrhs} RHS (rate; the n={n} time scales "
                                          "as n^3 for the factor, n^2 for the solves)"}
        n1 = 512
        S1 = syn.spd_matrix(np.random.default_rng(5), N, n1,
                            lambda a, b: mfref.gemm(a, b, nthreads=threads))
        B1 = syn.randn_mf(np.random.default_rng(6), N, n1, nrhs)
        t1f, (L1, _) = _cpu_timed(lambda: mfref.potrf(S1, nthreads=1))
        t1s, _ = _cpu_timed(lambda: mfref.potrs(L1, B1, nthreads=1))
        cpu["one_core"] = {"md_gflops": (n1 ** 3 / 3.0 + 2.0 * n1 * n1 * nrhs) / (t1f + t1s) / 1e9,
                           "cores": 1, "factor_s": t1f, "solve_s": t1s,
                           "sample": f"n={n1}, {nrhs} RHS (rate)"}
        cpu["kind"] = "port"
        work = n ** 3 / 3.0 + 2.0 * n * n * nrhs
        ops = ops_per_term(N)
        out[f"x{N}"] = {
            "factor_ms": t_f * 1e3, "solve_ms": t_s * 1e3, "solve_fast_order_ms": t_sf * 1e3,
            "repeats_ms": {"factor": ts_f, "solve": ts_s, "int8_trailing_factor": ts_fo},
            "md_gflops": work / (t_f + t_s) / 1e9,
            "roofline_factor": _fp64_roof(n ** 3 / 6.0 * ops, t_f, peak),
            "roofline_solve": _fp64_roof(float(n) * n * nrhs * ops, t_s, peak),
            "int8_trailing": {"factor_ms": t_fo * 1e3, "factor_speedup_vs_matched": t_f / t_fo,
                              "panel": 256},
            "parity": parity, "cpu_baseline": cpu}
        del S, Sw, Sw2, F, Fo, X, Xo, Bm
        torch.cuda.empty_cache()
    return out


def config_mixed_lu(R, torch, peak, reps):
    """mixed-precision LU solve (binary64 factor, Float64x4 refinement), n =
    4096, 16 RHS, against the plain Float64x4 LU"""
    import numpy as np
    mf, syn = R.mf, R.syn
    from oracle import mfref
    threads = mfref.threads()
    n, nrhs = 4096, 16
    A, B = syn.mixed_lu_problem(mf, n, nrhs, seed=4)
    t_m, ts_m, (X, rep) = _time_median(
        torch, lambda: mf.solve_mixed_lu(A, B, tol=1e-60, timing=True), None, reps)
    Aw = A.copy()
    t_p, ts_p, Xp = _time_median(torch, lambda: mf.solve(mf.lu_(Aw), B), lambda: Aw.copy_(A),
                                 reps)
    # the plain x4 factor and its solve timed apart: the solve's backward
    # substitution in the reference order (each row's chain starts at the
    # unknown solved last) is n(n-1)/2 dependent subtractions per column
    t_pf, ts_pf, Fp = _time_median(torch, lambda: mf.lu_(Aw), lambda: Aw.copy_(A), reps)
    t_ps, ts_ps, _ = _time_median(torch, lambda: mf.solve(Fp, B), None, reps)
    Aw2 = A.copy()
    ocfg = mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular", ozaki_block=256)
    t_o, ts_o, Xo = _time_median(torch, lambda: mf.solve(mf.lu_(Aw2, config=ocfg), B),
                                 lambda: Aw2.copy_(A), reps)
    # parity: exact backward errors of four columns of every solution
    An, Bn = A.to_numpy(), B.to_numpy()
    cols = [0, 5, 10, 15]
    be = lambda Xm: float(mfref.backward_error(An, Xm.to_numpy()[:, :, cols], Bn[:, :, cols]).max())
    parity = {"mixed_exact_backward_error_max": be(X), "plain_x4_exact_backward_error_max": be(Xp),
              "int8_trailing_x4_exact_backward_error_max": be(Xo), "columns_checked": cols,
              "target": 1e-60,
              "oracle": "superaccumulator residual ||b - A x||_inf / (||A|| ||x|| + ||b||)"}
    # CPU: the reference's route for a Float64x4 system (lu! + ldiv! in x4)
    cpu = {"kind": "port"}
    for key, nc, th in (("all_cores", 512, threads), ("one_core", 256, 1)):
        Ac = syn.randn_mf(np.random.default_rng(7), 4, nc, nc)
        Bc = syn.randn_mf(np.random.default_rng(8), 4, nc, nrhs)
        t_cf, (LU, piv, _) = _cpu_timed(lambda: mfref.getrf(Ac, nthreads=th))
        t_cs, _ = _cpu_timed(lambda: mfref.getrs(LU, piv, Bc, nthreads=th))
        w = 2.0 * nc ** 3 / 3.0 + 2.0 * nc * nc * nrhs
        cpu[key] = {"md_gflops": w / (t_cf + t_cs) / 1e9, "cores": th,
                    "extrapolated_n4096_s": (t_cf * (n / nc) ** 3 + t_cs * (n / nc) ** 2),
                    "sample": f"Float64x4 LU + {nrhs}-RHS solve at n={nc}, scaled as n^3 (factor) "
                              "and n^2 (solves) to n=4096"}
    flops64 = 2.0 * n ** 3 / 3.0
    out = {
        "mixed_ms": t_m * 1e3, "repeats_ms": {"mixed": ts_m, "plain_x4": ts_p, "int8_x4": ts_o,
                                              "plain_x4_factor": ts_pf, "plain_x4_solve": ts_ps},
        "binary64_factor_ms": rep["factor_ms"], "refinement_ms": rep["refine_ms"],
        "iterations": rep["iterations"], "mixed_backward_error": rep["backward_error"],
        "plain_x4_ms": t_p * 1e3, "speedup_vs_plain_x4": t_p / t_m,
        "plain_x4_factor_ms": t_pf * 1e3, "plain_x4_solve_ms": t_ps * 1e3,
        "plain_x4_factor_md_gflops": 2.0 * n ** 3 / 3.0 / t_pf / 1e9,
        "plain_x4_solve_chain": {"dependent_subtractions_per_column": n * (n - 1) // 2,
                                 "ns_per_subtraction": t_ps / (n * (n - 1) / 2) * 1e9,
                                 "note": "reference order (solve.jl / trsm.jl): row r's chain "
                                         "starts at the unknown solved last, so the backward "
                                         "substitution is one serial chain per column"},
        "int8_trailing_x4_ms": t_o * 1e3,
        "roofline_binary64_factor": {"bound": "fp64", "unit": "TFLOP/s",
                                     "achieved": flops64 / (rep["factor_ms"] / 1e3) / 1e12,
                                     "peak": 2 * peak / 1e12,
                                     "frac": flops64 / (rep["factor_ms"] / 1e3) / (2 * peak),
                                     "peak_source": "2 x DFMA probe instruction rate"},
        "roofline_plain_x4": _fp64_roof(n ** 3 / 3.0 * ops_per_term(4) + float(n) * n * nrhs
                                        * ops_per_term(4), t_p, peak),
        "roofline_plain_x4_factor": _fp64_roof(n ** 3 / 3.0 * ops_per_term(4), t_pf, peak),
        "parity": parity, "cpu_baseline": cpu,
        "matrix": "U diag(sigma) V^T, sigma geometric 1 -> 1e-12, lifted to Float64x4"}
    del A, B, X, Aw, Aw2, Xp, Xo, Fp
    torch.cuda.empty_cache()
    return out


def config_batched(R, torch, peak, reps):
    """10,000 batched Float64x2 SPD blocks, sizes U{8..256}, factor + solve in
    one graph-captured persistent launch, and the adjoint"""
    import numpy as np
    from concurrent.futures import ThreadPoolExecutor
    mf, syn = R.mf, R.syn
    from oracle import mfref
    threads = mfref.threads()
    rng = np.random.default_rng(5)
    sizes = rng.integers(8, 257, 10000)
    batch = mf.batched.SPDBatch(2, sizes)
    syn.spd_batch_fill(mf, batch, seed=5)
    S0, X0 = batch.S.clone(), batch.X.clone()
    tuned = mf.batched.autotune(batch)  # launch shape timed on the batch itself
    graph = mf.batched.BatchedSPDGraph(batch, tuning=tuned)

    def restore():
        batch.S.copy_(S0)
        batch.X.copy_(X0)

    t_b, ts_b, _ = _time_median(torch, graph.replay, restore, reps)
    info = batch.info[:batch.nblocks].cpu().numpy()
    restore()
    x, pullback = mf.batched.solve_spd_batched_rrule(batch, tuning=tuned)
    w = syn.randn_planes_device(17, 2, x.shape[1])
    t_a, ts_a, _ = _time_median(torch, lambda: pullback(w), None, reps)
    # parity: 16 blocks (the 4 largest, the 4 smallest, 8 random) bitwise
    # against the oracle's per-block Cholesky and solve
    picks = np.concatenate([np.argsort(-sizes)[:4], np.argsort(sizes)[:4],
                            np.random.default_rng(9).choice(len(sizes), 8, replace=False)])
    ok, bes = True, []
    for i in picks:
        Si, bi = batch.block(i, S0), batch.rhs(i, X0)
        L, inf = mfref.potrf(Si)
        xr = mfref.potrs(L, bi[:, :, None])
        ok = ok and inf == 0 and np.array_equal(np.tril(batch.block(i)).view(np.uint64),
                                                np.tril(L).view(np.uint64)) \
            and np.array_equal(batch.rhs(i).view(np.uint64), xr[:, :, 0].view(np.uint64))
        Ss = np.tril(Si) + np.transpose(np.tril(Si, -1), (0, 2, 1))
        bes.append(float(mfref.backward_error(Ss, xr, bi[:, :, None]).max()))
    parity = {"blocks_checked": [int(i) for i in picks], "bitwise_vs_oracle": bool(ok),
              "exact_backward_error_max": max(bes)}
    # CPU: the oracle's Cholesky + solve per block on a 300-block sample,
    # blocks spread over the host threads (all cores) and one after another
    samp = np.random.default_rng(11).choice(len(sizes), 300, replace=False)
    blocks = [(batch.block(i, S0), batch.rhs(i, X0)[:, :, None]) for i in samp]

    def one(b):
        L, _ = mfref.potrf(b[0], nthreads=1)
        return mfref.potrs(L, b[1], nthreads=1)

    wsamp = float(np.sum(sizes[samp].astype(float) ** 3 / 3 + 2.0 * sizes[samp].astype(float) ** 2))
    t_all, _ = _cpu_timed(lambda: list(ThreadPoolExecutor(threads).map(one, blocks)))
    t_one, _ = _cpu_timed(lambda: [one(b) for b in blocks])
    cpu = {"kind": "port",
           "all_cores": {"md_gflops": wsamp / t_all / 1e9, "cores": threads,
                         "sample": "300 random blocks, one block per host thread at a time"},
           "one_core": {"md_gflops": wsamp / t_one / 1e9, "cores": 1, "sample": "the same blocks"}}
    nn = sizes.astype(np.float64)
    instr = float(np.sum(nn ** 3 / 6.0 + nn * nn)) * ops_per_term(2)
    out = {
        "factor_solve_ms": t_b * 1e3, "repeats_ms": {"factor_solve": ts_b, "adjoint": ts_a},
        "md_gflops": batch.flops() / t_b / 1e9, "adjoint_ms": t_a * 1e3,
        "failed_blocks": int(np.count_nonzero(info)),
        "roofline": _fp64_roof(instr, t_b, peak),
        "launch": "counter memset, the persistent factor + forward-substitution kernel and the "
                  "backward-substitution kernel, replayed from a CUDA graph",
        "autotuned": {"threads": tuned["threads"], "grid": tuned["grid"],
                      "default_256x592_ms": tuned["timings"].get("256x592")},
        "parity": parity, "cpu_baseline": cpu,
        "data": "S_i = R_i R_i^T + n_i I, R_i randn Float64x2 with a populated low limb, one "
                "randn Float64x2 right-hand side per block (seeded)"}
    del graph, batch, S0, X0, x
    torch.cuda.empty_cache()
    return out


def run_configs(R, torch, peak, reps=3):
    """The other benchmark workloads beside the GEMM headline: device times
    (median of `reps` after a warm-up), FP64-pipe rooflines, oracle parity
    and CPU-oracle rates on all host cores and on one core."""
    return {"cholesky_n2048_rhs64": config_cholesky(R, torch, peak, reps),
            "mixed_lu_n4096_rhs16": config_mixed_lu(R, torch, peak, reps),
            "batched_spd_10000_x2": config_batched(R, torch, peak, reps)}


def run_tiles(args, R, torch, dist, world, rank):
    """One n x n x n Float64xN GEMM whose operands live on rank 0, split into
    2-D output tiles over all ranks (sharding.gemm_sharded_: panels scattered
    from rank 0, tiles gathered back): the timed step includes both
    transfers.  Strong scaling: the total work is fixed."""
    mf = R.mf
    N, n = args.limbs, args.n
    cfg = R.cfg("modular", args.knob or 30) if args.route != "plain" else mf.KernelConfig()
    A = B = C = None
    if rank == 0:
        A, B = R.operands(N, n)
        C = mf.MFMatrix.zeros(N, n, n)
    step = lambda: R.sharding.gemm_sharded_(C.storage if rank == 0 else None,
                                            A.storage if rank == 0 else None,
                                            B.storage if rank == 0 else None, config=cfg)
    clocks = NvmlClockSampler(R.local)
    clocks.start()
    t = R.timed(step, args.steps, args.warmup) / args.steps
    clk = clocks.stop()
    line = {
        "metric": METRIC, "value": 2.0 * n ** 3 / t / 1e9, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded randn * 2^U(-20,20), lower limbs randn*2^-53*|prev|)",
        "config": {"workload": f"Float64x{N} GEMM m=n=k={n}", "limbs": N, "n": n,
                   "route": "plain" if args.route == "plain" else "ozaki",
                   "moduli": None if args.route == "plain" else (args.knob or 30),
                   "parallelism": f"tiles{world}",
                   "l2": "inputs larger than L2 (each operand >= 1 GiB)"},
        "clocks": clk,
        "note": "rank 0 holds A, B and C; each step scatters the row panels of A and column "
                "panels of B, multiplies one 2-D tile per rank and gathers the tiles to rank 0",
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_case(args):
    """One small workload for a profiler capture: a warm-up call, then
    args.steps calls, timed with CUDA events (printed, not a bench value)."""
    import ctypes as C
    import torch
    import __graft_entry__
    mf = __graft_entry__.load_package()
    from mflab200 import synthetic as syn
    lib, n, N = mf._native.load(), args.n, args.limbs
    h, s = mf._handle(0), torch.cuda.current_stream().cuda_stream
    calls = []
    if args.case == "crt_gemm":
        A = mf.MFMatrix.zeros(N, n, n)
        B = mf.MFMatrix.zeros(N, n, n)
        Cm = mf.MFMatrix.zeros(N, n, n)
        A.planes()[0].normal_()
        B.planes()[0].normal_()
        cfg = mf.KernelConfig(gemm_strategy="ozaki", ozaki_scheme="modular",
                              ozaki_moduli=args.knob or 30)
        calls.append(lambda: mf.gemm_(Cm, A, B, config=cfg))
    elif args.case in ("getrf64", "lu64_solve", "mixed_lu"):
        A, B = syn.mixed_lu_problem(mf, n, 16, seed=4)
        LU = mf._leading_limb(A)
        LU0 = LU.storage.clone()
        ipiv = torch.arange(1, n + 1, dtype=torch.int64, device="cuda")
        info = torch.zeros(1, dtype=torch.int32, device="cuda")

        def factor():
            LU.storage.copy_(LU0)
            lib.mflab_getrf(h, s, 1, n, n, LU.ptr(), LU.ld, LU.ls, ipiv.data_ptr(), 32,
                            info.data_ptr())
        if args.case == "getrf64":
            calls.append(factor)
        elif args.case == "lu64_solve":
            factor()
            wb = C.c_size_t()
            lib.mflab_lu64_work_bytes(n, C.byref(wb))
            work = torch.empty(wb.value, dtype=torch.uint8, device="cuda")
            lib.mflab_lu64_prepare(h, s, n, LU.ptr(), LU.ld, ipiv.data_ptr(), work.data_ptr())
            D = mf._leading_limb(B)
            calls.append(lambda: lib.mflab_lu64_solve(h, s, n, D.n, LU.ptr(), LU.ld,
                                                      work.data_ptr(), D.ptr(), D.ld))
        else:
            calls.append(lambda: mf.solve_mixed_lu(A, B, tol=1e-60))
    elif args.case == "potrf":
        S = syn.spd_matrix_device(mf, 3, N, n)
        Aw = S.copy()
        calls.append(lambda: (Aw.copy_(S), mf.cholesky_(Aw)))
    elif args.case == "batched":
        import numpy as np
        sizes = np.random.default_rng(5).integers(8, 257, n)
        batch = mf.batched.SPDBatch(N, sizes)
        syn.spd_batch_fill(mf, batch, seed=5)
        S0, X0 = batch.S.clone(), batch.X.clone()
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        shape = {"threads": args.knob or 128, "grid": sms * 8}
        calls.append(lambda: (batch.S.copy_(S0), batch.X.copy_(X0),
                              mf.batched.potrf_potrs_batched_(batch, tuning=shape)))
    elif args.case == "getrf":
        A, _ = syn.mixed_lu_problem(mf, n, 1, seed=4)
        A = mf.MFMatrix(A.storage[:N].clone())
        Aw = A.copy()
        calls.append(lambda: (Aw.copy_(A), mf.lu_(Aw)))
    fn = calls[0]
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(max(args.steps, 1)):
        fn()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"case": args.case, "n": n, "limbs": N,
                      "ms_per_call": e0.elapsed_time(e1) / max(args.steps, 1)}))


def main():
    args = parse()
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    import numpy as np
    import torch
    import torch.distributed as dist

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    R = Runner(args, torch, dist, world, rank, local)
    mf = R.mf
    if args.split == "tiles":
        run_tiles(args, R, torch, dist, world, rank)
        if world > 1:
            dist.destroy_process_group()
        return
    N, n = args.limbs, args.n
    route = args.route
    if route == "auto":
        route = "ozaki" if mf.ozaki_available() else "plain"
    flops = 2.0 * n * n * n
    plain_cfg = mf.KernelConfig(gemm_strategy="auto")

    peak_fp64 = fp64_peak(mf, torch)  # before the power-capped tensor work
    A, B = R.operands(N, n)
    Cm = mf.MFMatrix.zeros(N, n, n)
    scheme = args.scheme
    acc, e_plain, check = {}, None, None
    if rank == 0:
        check = R.checker(n, A, B, Cm)
        mf.gemm_(Cm, A, B)
        e_plain = check()
        if route != "ozaki":
            acc = {"plain_max_rel_err": e_plain, "samples": 256}
        elif args.knob > 0:
            mf.gemm_(Cm, A, B, config=R.cfg(scheme, args.knob))
            knob_name = "moduli" if scheme == "modular" else "slices"
            acc = {"scheme": scheme, knob_name: args.knob, "plain_max_rel_err": e_plain,
                   "ozaki_max_rel_err": check(), "samples": 256,
                   "rule": f"{knob_name} count fixed on the command line"}
        else:
            try:
                acc = R.accuracy_search(N, n, A, B, Cm, scheme, e_plain, check)
            except mf.ArgumentError:
                if scheme != "modular":
                    raise
                scheme = "slices"  # the modulus table cannot reach the requirement
                acc = R.accuracy_search(N, n, A, B, Cm, scheme, e_plain, check)
    knob = acc.get("moduli", acc.get("slices", 0))
    # every rank runs the route rank 0 tuned
    knob = R.sharding.agree(knob)
    scheme = "modular" if R.sharding.agree(1 if scheme == "modular" else 0) else "slices"
    oz_cfg = R.cfg(scheme, knob)
    head_cfg = oz_cfg if route == "ozaki" else plain_cfg

    clocks = NvmlClockSampler(local)
    clocks.start()
    t_head = R.timed(lambda: mf.gemm_(Cm, A, B, config=head_cfg), args.steps, args.warmup)
    clk = clocks.stop()
    t_head /= args.steps
    t_plain = R.timed(lambda: mf.gemm_(Cm, A, B, config=plain_cfg), 1, 1) if route == "ozaki" \
        else t_head

    # end to end through the public API with host buffers in the reference's
    # own storage order (a Julia Matrix{Float64xN} keeps the N limbs of an
    # element together): every step uploads A and B from pinned interleaved
    # host memory into limb planes (mflab_h2d_interleaved), multiplies, and
    # downloads C back to interleaved host memory (mflab_d2h_interleaved);
    # the uploads of step i+1 (A and B each on a stream and handle of its
    # own, so that B's copy does not wait for A's permutation kernel) and the
    # download of step i-1 run while step i multiplies (two device buffer
    # sets); the staging of one handle takes a whole 1 GiB matrix per copy
    hA = torch.empty((n, n, N), dtype=torch.float64, pin_memory=True)
    hB = torch.empty((n, n, N), dtype=torch.float64, pin_memory=True)
    hC = torch.empty((n, n, N), dtype=torch.float64, pin_memory=True)
    A.copy_to_interleaved_(hA)
    B.copy_to_interleaved_(hB)
    torch.cuda.synchronize()
    bufs = [tuple(mf.MFMatrix.empty(N, n, n) for _ in range(3)) for _ in range(2)]
    h_upA, h_upB, h_down = (mf.create_handle(local) for _ in range(3))

    def e2e_run(steps):
        cs = torch.cuda.current_stream()
        hsA, hsB, ds = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
        upA = [torch.cuda.Event() for _ in range(2)]
        upB = [torch.cuda.Event() for _ in range(2)]
        done = [torch.cuda.Event() for _ in range(2)]
        down = [torch.cuda.Event() for _ in range(2)]
        R.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(cs)
        for st in (hsA, hsB, ds):
            st.wait_event(e0)
        for i in range(steps):
            b = i % 2
            dA, dB, dC = bufs[b]
            if i >= 2:  # step i-2 no longer reads this set
                hsA.wait_event(done[b])
                hsB.wait_event(done[b])
            dA.copy_from_interleaved_(hA, stream=hsA, handle=h_upA)
            upA[b].record(hsA)
            dB.copy_from_interleaved_(hB, stream=hsB, handle=h_upB)
            upB[b].record(hsB)
            cs.wait_event(upA[b])
            cs.wait_event(upB[b])
            if i >= 2:
                cs.wait_event(down[b])  # step i-2's result has left dC
            mf.gemm_(dC, dA, dB, config=head_cfg)
            done[b].record(cs)
            ds.wait_event(done[b])
            dC.copy_to_interleaved_(hC, stream=ds, handle=h_down)
            down[b].record(ds)
        for st in (hsA, hsB, ds):
            cs.wait_stream(st)
        e1.record(cs)
        R.barrier()
        return R.sharding.max_over_ranks(e0.elapsed_time(e1) / 1e3)

    e2e_run(2)  # warm-up (scratch, staging, host page mappings)
    e2e_steps = max(2, args.steps)
    t_e2e = e2e_run(e2e_steps) / e2e_steps
    # the downloaded result equals the device-resident call on the same operands
    mf.gemm_(Cm, A, B, config=head_cfg)
    e2e_ok = bool(torch.equal(torch.from_numpy(Cm.to_interleaved()), hC))
    torch.cuda.synchronize()
    for hh in (h_upA, h_upB, h_down):
        mf.destroy_handle(hh)
    del bufs, hA, hB, hC
    instr = float(n) ** 3 * ops_per_term(N)
    plain_roof = {"bound": "fp64", "achieved": instr / t_plain / 1e12, "peak": peak_fp64 / 1e12,
                  "unit": "T FP64 instr/s", "frac": instr / t_plain / peak_fp64,
                  "traffic": read_traffic(f"mm_x{N}_n{n}"),
                  "peak_source": "measured in this run (DFMA probe, burst)"}
    if route == "ozaki":
        ph, ops = R.phases(N, n, A, B, Cm, scheme, knob)
        peak8 = R.int8_peak(fill=1)
        peak8c = R.int8_peak(fill=0)
        achieved = ops / (ph[2] / 1e3)
        roof = {"bound": "tensor", "achieved": achieved / 1e12, "peak": peak8 / 1e12,
                "unit": "INT8 TOP/s", "frac": achieved / peak8,
                "frac_of_constant_data_peak": achieved / peak8c,
                "peak_constant_data": peak8c / 1e12,
                "frac_of_nominal_4500": achieved / 4.5e15,
                "traffic": read_traffic(f"int8_tc_{scheme}_x{N}_n{n}", scale_from_smaller=True),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                                  "(profiles/ncu_traffic.txt); sizes above the largest capture "
                                  "scaled by (n / n_capture)^2",
                "kernel": "mfl::int8_tc_gemm_kernel (tcgen05.mma kind::i8, TMA, TMEM): the int8 "
                          + ("residue GEMMs, all moduli of a digit level in one launch"
                             if scheme == "modular" else "level GEMMs (K = (L-1) k)"),
                "peak_source": "measured in this run: cuBLASLt int8 TN GEMM 8192x8192x16384 "
                               "(burst) on uniformly distributed bytes, like the residues; "
                               "peak_constant_data is the same GEMM on constant bytes, which "
                               "draws less power and runs faster under the power cap; nominal "
                               "dense INT8 is 4500 TOP/s",
                "phases_ms": {"exponents_tune": ph[0], "split": ph[1], "int8_gemms": ph[2],
                              "reconstruct_accumulate": ph[3]}}
    else:
        roof = plain_roof

    if route != "ozaki":
        launches = 1
    elif scheme == "modular":
        launches = 5 + (1 if N == 2 else 2)  # scales 2, split 2, one GEMM launch per digit level, 1
    else:
        launches = 5 + knob                  # scales 2, split 2, one GEMM per level, accumulate
    value = world * flops / t_head / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_head * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded randn * 2^U(-20,20), lower limbs randn*2^-53*|prev|)",
        "config": {"workload": f"Float64x{N} GEMM m=n=k={n}", "limbs": N, "n": n,
                   "route": route, "scheme": scheme if route == "ozaki" else None,
                   "moduli": knob if route == "ozaki" and scheme == "modular" else None,
                   "slices": knob if route == "ozaki" and scheme == "slices" else None,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (each operand >= 1 GiB)"},
        "accuracy": acc,
        "plain_fp64": {"value": world * flops / t_plain / 1e9, "ms_per_step": t_plain * 1e3,
                       "roofline": plain_roof},
        "speedup_vs_plain": t_plain / t_head,
        "e2e": {"value": world * flops / t_e2e / 1e9, "unit": UNIT,
                "h2d_bytes_per_step": 2 * N * n * n * 8, "d2h_bytes_per_step": N * n * n * 8,
                "host_layout": "interleaved (n, n, N) pinned host arrays, as a Julia "
                               "Matrix{Float64xN}; converted to and from limb planes by "
                               "mflab_h2d_interleaved / mflab_d2h_interleaved inside the step",
                "result_equals_device_resident_call": e2e_ok},
        "roofline": roof,
        "clocks": clk,
        "gpu_launches": args.steps * launches,
        "library_launches": 0,
    }
    if rank == 0 and world == 1 and route == "ozaki" and scheme == "modular" \
            and not args.no_slices:
        # the digit-slice scheme on the same operands, at its own equal-error S
        sacc = R.accuracy_search(N, n, A, B, Cm, "slices", e_plain, check)
        ts = R.timed(lambda: mf.gemm_(Cm, A, B, config=R.cfg("slices", sacc["slices"])), 2, 1) / 2
        line["slices_scheme"] = {"value": flops / ts / 1e9, "ms_per_step": ts * 1e3,
                                 "speedup_vs_plain": t_plain / ts, "accuracy": sacc}
    if N == 2 and route == "ozaki" and not args.no_x4 and world == 1:
        del A, B, Cm
        torch.cuda.empty_cache()
        A4, B4 = R.operands(4, n)
        C4 = mf.MFMatrix.zeros(4, n, n)
        chk4 = R.checker(n, A4, B4, C4)
        t4p = R.timed(lambda: mf.gemm_(C4, A4, B4), 1, 0)
        e4p = chk4()
        x4 = {"workload": f"Float64x4 GEMM m=n=k={n}", "plain_value": flops / t4p / 1e9,
              "plain_ms": t4p * 1e3}
        for sch in (("modular", "slices") if scheme == "modular" else ("slices",)):
            try:
                a4 = R.accuracy_search(4, n, A4, B4, C4, sch, e4p, chk4)
            except mf.ArgumentError:
                continue
            k4 = a4.get("moduli", a4.get("slices"))
            t4 = R.timed(lambda: mf.gemm_(C4, A4, B4, config=R.cfg(sch, k4)), 2, 1) / 2
            x4[sch] = {"value": flops / t4 / 1e9, "ms": t4 * 1e3, "speedup_vs_plain": t4p / t4,
                       "accuracy": a4}
        line["x4"] = x4
    if rank == 0 and world == 1 and not args.no_configs:
        line["configs"] = run_configs(R, torch, peak_fp64, args.config_reps)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import mfref
        threads = mfref.threads()
        v, sample = cpu_sample(mfref, N, n, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
