"""Persisted device tuning profiles.

The reference keeps CPU tuning explicit and reproducible: `calibrate_gemm`
measures, a `GemmProfile` tagged with `machine_fingerprint()` stores the
result, `profile_compatible` checks the fingerprint and `with_gemm_profile`
copies it into a `KernelConfig` (src/calibration.jl:15-115); nothing
calibrates behind the caller's back.  This module does the same for the
device choices that otherwise need a measurement on every run:

* the launch shape (CTA size, persistent CTA count) of the batched SPD
  solve, per batch size signature (batched.autotune);
* the modulus count of the modular INT8 GEMM that reaches the plain
  kernel's accuracy, per (limbs, k, operand exponent spread);
* the int8 engine.

    prof = calibrate(batches=[batch], moduli={(2, 8192, 20): 30})
    save_profile(prof, "b200.json")
    prof = load_profile("b200.json")            # later, on the same device kind
    cfg = with_tune_profile(KernelConfig(gemm_strategy="ozaki"), prof, N=2, k=8192)
    batched.autotune(batch, profile=prof)       # the stored shape, no timing
"""
from __future__ import annotations

import dataclasses
import json
from typing import Dict, Optional, Sequence

import torch

PROFILE_VERSION = 1


def device_fingerprint(device: Optional[int] = None) -> dict:
    """Stable identity of a device and the software that tuned on it (the
    GPU model, SM count, compute capability and memory, the CUDA runtime and
    library versions); clocks are not part of it (they vary under load)."""
    from . import _native
    dev = torch.cuda.current_device() if device is None else device
    p = torch.cuda.get_device_properties(dev)
    return {
        "name": p.name, "sms": int(p.multi_processor_count),
        "capability": f"{p.major}.{p.minor}", "memory_gib": int(p.total_memory >> 30),
        "cuda": torch.version.cuda, "library": int(_native.load().mflab_version()),
    }


@dataclasses.dataclass
class TuneProfile:
    """Measured device choices and the fingerprint they were measured on."""
    fingerprint: dict
    batched: Dict[str, dict] = dataclasses.field(default_factory=dict)
    moduli: Dict[str, int] = dataclasses.field(default_factory=dict)
    engine: str = "tcgen05"
    source: str = "measured"
    version: int = PROFILE_VERSION


def batch_key(limbs: int, block: int, sizes) -> str:
    """signature of a batch for the launch-shape table: limbs, inner block,
    block count, largest size, sum of sizes and of squared sizes"""
    import numpy as np
    n = np.asarray(sizes, dtype=np.int64)
    return (f"x{limbs}-b{block}-n{len(n)}-max{int(n.max()) if len(n) else 0}-"
            f"s{int(n.sum())}-q{int((n * n).sum())}")


def moduli_key(limbs: int, k: int, spread_bits: float) -> str:
    return f"x{limbs}-k{int(k)}-spread{float(spread_bits):g}"


def profile_compatible(profile: TuneProfile, device: Optional[int] = None) -> bool:
    """Whether `profile` was measured on this kind of device with this
    software (every fingerprint field must match)."""
    return profile.version == PROFILE_VERSION and profile.fingerprint == device_fingerprint(device)


def save_profile(profile: TuneProfile, path: str) -> None:
    with open(path, "w") as f:
        json.dump(dataclasses.asdict(profile), f, indent=1, sort_keys=True)


def load_profile(path: str) -> TuneProfile:
    with open(path) as f:
        d = json.load(f)
    if d.get("version") != PROFILE_VERSION:
        raise ValueError(f"tuning profile {path} has version {d.get('version')}, "
                         f"expected {PROFILE_VERSION}")
    return TuneProfile(**d)


def _check(profile: TuneProfile, strict: bool, device: Optional[int]) -> None:
    from . import ArgumentError
    if strict and not profile_compatible(profile, device):
        raise ArgumentError("TuneProfile fingerprint does not match this device; pass "
                            "strict=False to apply it anyway")


def with_tune_profile(config, profile: TuneProfile, N: int, k: int, spread_bits: float = 0.0,
                      strict: bool = True, device: Optional[int] = None):
    """A copy of `config` with the profile's modulus count for (N, k,
    spread) and its int8 engine (the other fields are kept; no stored count:
    the route's own tuner decides)."""
    _check(profile, strict, device)
    T = profile.moduli.get(moduli_key(N, k, spread_bits), 0)
    return dataclasses.replace(config, ozaki_moduli=int(T), ozaki_engine=profile.engine)


def stored_batched_shape(profile: TuneProfile, limbs: int, block: int, sizes,
                         strict: bool = True, device: Optional[int] = None) -> Optional[dict]:
    """The profile's launch shape for a batch of this signature, or None."""
    _check(profile, strict, device)
    return profile.batched.get(batch_key(limbs, block, sizes))


def calibrate(batches: Sequence = (), block: int = 16, moduli: Optional[Dict] = None,
              engine: str = "tcgen05", device: Optional[int] = None) -> TuneProfile:
    """Measure a profile on this device: the batched launch shape of each
    given SPDBatch (batched.autotune, timed on the batch itself) and the
    modulus counts passed in `moduli` ({(N, k, spread_bits): T} found by an
    accuracy search such as bench.py's); `engine` is recorded as given."""
    from . import batched as _batched
    prof = TuneProfile(fingerprint=device_fingerprint(device), engine=engine)
    for b in batches:
        t = _batched.autotune(b, block)
        prof.batched[batch_key(b.N, block, b.sizes_host)] = {
            "threads": int(t["threads"]), "grid": int(t["grid"]), "ms": float(t["ms"])}
    for (N, k, spread), T in (moduli or {}).items():
        prof.moduli[moduli_key(N, k, spread)] = int(T)
    return prof
