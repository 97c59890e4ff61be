"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes

import pytest


def test_library_exports_declared_symbols(mf):
    lib = mf._native.load()
    names = mf._native.declared_symbols()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_status_strings(mf):
    lib = mf._native.load()
    assert lib.mflab_version() >= 100
    assert lib.mflab_status_string(0) == b"ok"
    assert b"dimension" in lib.mflab_status_string(-1)
    assert b"option" in lib.mflab_status_string(-7)


def test_status_codes_map_to_reference_exceptions(mf):
    """shape errors are DimensionMismatch, option codes / aliasing /
    unsupported options ArgumentError (trsv.jl:28-34 raises both kinds)"""
    nat = mf._native
    with pytest.raises(mf.DimensionMismatch):
        mf._check(nat.MFLAB_ERR_ARG, "x")
    for rc in (nat.MFLAB_ERR_FLAG, nat.MFLAB_ERR_ALIAS, nat.MFLAB_ERR_UNSUPPORTED):
        with pytest.raises(mf.ArgumentError):
            mf._check(rc, "x")
    with pytest.raises(mf.MFLABError):
        mf._check(nat.MFLAB_ERR_TIMEOUT, "x")


def test_binding_covers_header(mf):
    """every declared entry point has a ctypes signature in the binding"""
    assert set(mf._native.declared_symbols()) <= set(mf._native.SIGNATURES)


def test_gemm_plan_routes(mf):
    assert mf.gemm_plan(3, 8, 8, 8)["strategy"] == "fused"
    assert mf.gemm_plan(2, 8, 8, 8)["strategy"] == "direct"
    with pytest.raises(mf.ArgumentError):
        mf.gemm_plan(2, 8, 8, 8, mf.KernelConfig(gemm_strategy="fused"))
    with pytest.raises(mf.ArgumentError):
        mf.gemm_plan(2, 8, 8, 8, mf.KernelConfig(gemm_strategy="bogus"))


def test_capabilities(mf):
    c = mf.capabilities(2)
    assert c["supported"] and c["limb_count"] == 2 and c["syrk_authoritative_triangle"] == "lower"
    assert not mf.capabilities(7)["supported"]


def test_debug_library_matches_release_exports(mf):
    """the index-checking debug build (libmflab200_debug.so) exports the same
    entry points; it reports itself as a debug build, the release as not"""
    import os
    nat = mf._native
    if not os.path.exists(nat.DEBUG_LIB_PATH):
        pytest.skip("debug library not built")
    dbg = nat.load_library(nat.DEBUG_LIB_PATH)
    missing = [n for n in nat.declared_symbols() if not hasattr(dbg, n)]
    assert not missing, missing
    assert dbg.mflab_debug_build() == 1
    assert nat.load().mflab_debug_build() == 0
