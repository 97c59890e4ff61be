"""Persisted tuning profiles (the device counterpart of the reference's
GemmProfile / profile_compatible / with_gemm_profile, calibration.jl:15-115):
JSON round trip, fingerprint check, application to a KernelConfig, and the
batched launch shape taken from a profile without timing."""
import dataclasses

import numpy as np
import pytest


def _fake_fp(monkeypatch, mf, fp):
    monkeypatch.setattr(mf.tuning, "device_fingerprint", lambda device=None: dict(fp))


FP = {"name": "NVIDIA B200", "sms": 148, "capability": "10.0", "memory_gib": 178,
      "cuda": "12.8", "library": 100}


def test_profile_round_trip_and_application(mf, monkeypatch, tmp_path):
    _fake_fp(monkeypatch, mf, FP)
    t = mf.tuning
    prof = t.TuneProfile(fingerprint=dict(FP), engine="tcgen05_1sm")
    prof.moduli[t.moduli_key(2, 8192, 20)] = 30
    prof.batched[t.batch_key(2, 16, [8, 9, 10])] = {"threads": 128, "grid": 1184, "ms": 1.0}
    path = tmp_path / "prof.json"
    t.save_profile(prof, str(path))
    back = t.load_profile(str(path))
    assert back == prof
    assert t.profile_compatible(back)
    cfg = t.with_tune_profile(mf.KernelConfig(gemm_strategy="ozaki"), back, N=2, k=8192,
                              spread_bits=20)
    assert cfg.ozaki_moduli == 30 and cfg.ozaki_engine == "tcgen05_1sm"
    assert cfg.gemm_strategy == "ozaki"
    # an unknown shape leaves the route's own tuner in charge
    assert t.with_tune_profile(mf.KernelConfig(), back, N=4, k=100).ozaki_moduli == 0
    assert t.stored_batched_shape(back, 2, 16, [10, 9, 8])["grid"] == 1184
    assert t.stored_batched_shape(back, 2, 16, [8, 9]) is None


def test_profile_fingerprint_mismatch(mf, monkeypatch):
    _fake_fp(monkeypatch, mf, FP)
    t = mf.tuning
    other = dict(FP, sms=132)
    prof = t.TuneProfile(fingerprint=other)
    assert not t.profile_compatible(prof)
    with pytest.raises(mf.ArgumentError):
        t.with_tune_profile(mf.KernelConfig(), prof, N=2, k=64)
    assert t.with_tune_profile(mf.KernelConfig(), prof, N=2, k=64, strict=False).ozaki_moduli == 0


def test_profile_version_is_checked(mf, tmp_path):
    p = tmp_path / "old.json"
    p.write_text('{"version": 0, "fingerprint": {}}')
    with pytest.raises(ValueError):
        mf.tuning.load_profile(str(p))


@pytest.mark.gpu
def test_batched_autotune_uses_a_profile_without_timing(mf, tmp_path):
    t = mf.tuning
    sizes = np.random.default_rng(2).integers(8, 64, 300)
    batch = mf.batched.SPDBatch(2, sizes)
    prof = t.calibrate(batches=[batch], moduli={(2, 1024, 10): 25})
    assert t.profile_compatible(prof)
    path = tmp_path / "p.json"
    t.save_profile(prof, str(path))
    loaded = t.load_profile(str(path))
    got = mf.batched.autotune(batch, profile=loaded)
    assert got["source"] == "profile" and got["timings"] == {}
    key = t.batch_key(2, 16, sizes)
    assert (got["threads"], got["grid"]) == (loaded.batched[key]["threads"],
                                             loaded.batched[key]["grid"])
    cfg = t.with_tune_profile(mf.KernelConfig(gemm_strategy="ozaki"), loaded, 2, 1024, 10)
    assert cfg.ozaki_moduli == 25
