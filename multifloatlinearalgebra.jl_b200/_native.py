"""Binding of the mflab200 C ABI (include/mflab200.h) and its in-tree build.

The product path is the CUDA library built here for sm_100a.  Loading fails
loudly when the library is missing or no CUDA device is present: there is no
CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(PKG_DIR, "libmflab200.so")
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(REPO_DIR, "include")

# -fno-gnu-unique: the function-local statics of templates (the "attribute
# already set" flags of the launchers) stay private to each library, so the
# release and the debug build can be loaded into one process side by side
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-gnu-unique", "-shared",
]

MFLAB_OK = 0
MFLAB_ERR_ARG = -1
MFLAB_ERR_CUDA = -2
MFLAB_ERR_UNSUPPORTED = -3
MFLAB_ERR_TIMEOUT = -4
MFLAB_ERR_ALLOC = -5
MFLAB_ERR_ALIAS = -6
MFLAB_ERR_FLAG = -7


OBJ_DIR = os.path.join(PKG_DIR, "_build")
# the debug build: the same sources with -DMFLAB_DEBUG (device index checks
# that record violations instead of trapping), loaded when MFLAB_DEBUG=1
DEBUG_LIB_PATH = os.path.join(PKG_DIR, "libmflab200_debug.so")
DEBUG_OBJ_DIR = os.path.join(PKG_DIR, "_build_debug")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers() -> list[str]:
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _run(cmd: list[str]) -> str:
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out.stdout + out.stderr)
    return out.stdout + out.stderr


def build(verbose: bool = False, jobs: int | None = None, debug: bool = True) -> str:
    """Compile every CUDA source (sm_100a) into libmflab200.so in the package
    and, with `debug`, into libmflab200_debug.so with -DMFLAB_DEBUG: one nvcc
    per translation unit and variant in parallel (objects under _build/ and
    _build_debug/, rebuilt when the source or any header is newer), then one
    link per library.  Returns the release library's path."""
    from concurrent.futures import ThreadPoolExecutor

    nvcc = os.environ.get("NVCC", "nvcc")
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    variants = [(OBJ_DIR, LIB_PATH, [])]
    if debug:
        variants.append((DEBUG_OBJ_DIR, DEBUG_LIB_PATH, ["-DMFLAB_DEBUG"]))
    todo, links = [], []
    for obj_dir, lib_path, extra in variants:
        os.makedirs(obj_dir, exist_ok=True)
        objs, stale = [], False
        for src in sources():
            obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
            objs.append(obj)
            if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src),
                                                                        newest_header):
                todo.append([nvcc, *compile_flags, *extra, "-I", INCLUDE, "-c", "-o", obj, src])
                stale = True
        if stale or not os.path.exists(lib_path):
            links.append([nvcc, *NVCC_FLAGS, "-o", lib_path, *objs, "-lcublasLt"])
    logs = []
    if todo:
        with ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            logs = list(ex.map(_run, todo))
    for cmd in links:
        logs.append(_run(cmd))
    if verbose:
        print("".join(logs))
    return LIB_PATH


_d = C.POINTER(C.c_double)
_i64 = C.c_int64
_vp = C.c_void_p
_int = C.c_int

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "mflab_version": [],
    "mflab_status_string": [_int],
    "mflab_last_error": [],
    "mflab_create": [C.POINTER(_vp), _int],
    "mflab_destroy": [_vp],
    "mflab_set_solve_order": [_vp, _int],
    "mflab_gemm": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _vp,
                   _i64, _i64, _d, _d],
    "mflab_syrk_lower": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _d, _d],
    "mflab_syrk_packed": [_vp, _vp, _int, _i64, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _d,
                          _d],
    "mflab_trmm": [_vp, _vp, _int, _int, _int, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                   _i64, _d],
    "mflab_gemmt_lower": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                          _i64, _d, _d],
    "mflab_trsm": [_vp, _vp, _int, _int, _int, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                   _i64, _d],
    "mflab_potrf": [_vp, _vp, _int, _i64, _vp, _i64, _i64, _i64, _vp],
    "mflab_pstrf": [_vp, _vp, _int, _i64, _vp, _i64, _i64, _d, _vp, _vp],
    "mflab_qr": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp],
    "mflab_apply_q": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _i64,
                      _i64, _i64],
    "mflab_qr_numerical_rank": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _d, _d, _vp],
    "mflab_potrs": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64],
    "mflab_getrf": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp],
    "mflab_getrs": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _vp, _i64, _i64],
    "mflab_max_abs": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _int, _vp],
    "mflab_residual": [_vp, _vp, _int, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                       _i64, _vp, _i64, _i64, _vp, _i64, _i64],
    "mflab_residual_mixed": [_vp, _vp, _int, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp,
                             _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64],
    "mflab_backward_error": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                             _i64, _vp, _i64, _i64, _vp, _i64, _i64, _vp],
    "mflab_add_widened": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64],
    "mflab_spd_batched": [_vp, _vp, _int, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _i64,
                          _i64, _int, _vp, _vp, _int],
    "mflab_spd_batched_adjoint": [_vp, _vp, _int, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _vp,
                                  _vp, _i64, _vp, _vp, _vp, _int],
    "mflab_spd_batched_ex": [_vp, _vp, _int, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _i64,
                             _i64, _int, _vp, _vp, _int, _int],
    "mflab_spd_batched_adjoint_ex": [_vp, _vp, _int, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64,
                                     _vp, _vp, _i64, _vp, _vp, _vp, _int, _int],
    "mflab_sytrf": [_vp, _vp, _int, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp, _int, _i64, _vp],
    "mflab_sytrs": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i64,
                    _i64, _vp],
    "mflab_ldlt_diagnostics": [_vp, _vp, _int, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp],
    "mflab_max_abs_noalloc": [_vp, _int, _i64, _i64, _vp, _i64, _i64, _int, _vp],
    "mflab_diag_summary": [_vp, _vp, _int, _vp, _i64, _i64, _i64, _vp, _vp, _vp],
    "mflab_probe_fp64": [_vp, _int, _int, _int, _i64, _vp, _d],
    "mflab_gemm_ozaki": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64,
                         _vp, _i64, _i64, _d, _d],
    "mflab_ozaki_default_slices": [_int, _i64],
    "mflab_gemv": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _i64, _d,
                   _d],
    "mflab_symv": [_vp, _vp, _int, _int, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _i64, _d, _d],
    "mflab_dot": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _vp],
    "mflab_gemm_ozaki_crt": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                             _i64, _vp, _i64, _i64, _d, _d],
    "mflab_ozaki_last_moduli": [_vp],
    "mflab_ozaki_crt_tune": [_vp, _vp, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64,
                             C.POINTER(_int)],
    "mflab_syrk_lower_ozaki": [_vp, _vp, _int, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                               _i64, _d, _d],
    "mflab_potrf_ozaki": [_vp, _vp, _int, _int, _i64, _vp, _i64, _i64, _i64, _i64, _vp],
    "mflab_getrf_ozaki": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64,
                          _vp],
    "mflab_opnorm_inf": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp, _vp],
    "mflab_backward_error_norm": [_vp, _vp, _int, _i64, _i64, _i64, _vp, _vp, _vp, _i64, _i64,
                                  _vp, _i64, _i64, _vp, _i64, _i64, _vp],
    "mflab_ozaki_crt_plan": [_int, _i64, _int, _int, C.POINTER(_int), C.POINTER(_int),
                             C.POINTER(_int)],
    "mflab_ozaki_crt_modulus": [_int],
    "mflab_ozaki_crt_reduce_host": [_int, _int, _vp, _vp, _vp],
    "mflab_gemm_ozaki_crt_phases": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp,
                                    _i64, _i64, _vp, _i64, _i64, _d, _d, C.POINTER(C.c_float),
                                    _d],
    "mflab_ozaki_last_slices": [_vp],
    "mflab_set_int8_engine": [_vp, _int],
    "mflab_device_status": [_vp, C.POINTER(_int)],
    "mflab_int8_gemm_tn": [_vp, _vp, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64,
                           _i64, _vp, _i64, _vp],
    "mflab_gemm_ozaki_phases": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _i64, _i64, _vp, _i64,
                                _i64, _vp, _i64, _i64, _d, _d, C.POINTER(C.c_float), _d],
    "mflab_probe_int8_gemm": [_vp, _vp, _i64, _i64, _i64, _int, _int, C.POINTER(C.c_float)],
    "mflab_set_tc_debug": [_vp, _i64, _int],
    "mflab_ozaki_crt_prepare_bytes": [_int, _int, _i64, _i64, C.POINTER(C.c_size_t)],
    "mflab_ozaki_crt_prepare": [_vp, _vp, _int, _int, _i64, _i64, _vp, _i64, _i64, _vp],
    "mflab_gemm_ozaki_crt_prepared": [_vp, _vp, _int, _int, _i64, _i64, _i64, _vp, _vp, _i64,
                                      _i64, _vp, _i64, _i64, _d, _d],
    "mflab_lu64_work_bytes": [_i64, C.POINTER(C.c_size_t)],
    "mflab_lu64_prepare": [_vp, _vp, _i64, _vp, _i64, _vp, _vp],
    "mflab_lu64_solve": [_vp, _vp, _i64, _i64, _vp, _i64, _vp, _vp, _i64],
    "mflab_malloc": [_int, C.c_size_t, C.POINTER(_vp)],
    "mflab_free": [_vp],
    "mflab_memcpy": [_vp, _vp, C.c_size_t, _int, _vp],
    "mflab_memset": [_vp, _int, C.c_size_t, _vp],
    "mflab_stream_synchronize": [_vp],
    "mflab_h2d_interleaved": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _vp, _i64, _i64],
    "mflab_d2h_interleaved": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64],
    "mflab_interleaved_to_planes": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _vp, _i64, _i64],
    "mflab_planes_to_interleaved": [_vp, _vp, _int, _i64, _i64, _vp, _i64, _i64, _vp, _i64],
    "mflab_debug_violations": [C.POINTER(C.c_longlong), _int],
    "mflab_debug_build": [],
}
_RESTYPE = {"mflab_status_string": C.c_char_p, "mflab_last_error": C.c_char_p}

_lib = None


def load(path: str | None = None):
    """Load the built library (no build, no fallback): libmflab200.so, or the
    debug build when the environment sets MFLAB_DEBUG=1."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = DEBUG_LIB_PATH if os.environ.get("MFLAB_DEBUG") == "1" else LIB_PATH
    lib = load_library(path)
    _lib = lib
    return lib


def load_library(path: str):
    """A separately loaded copy of a built library (its own handles and
    device state), with the ctypes signatures set."""
    if not os.path.exists(path):
        raise RuntimeError(
            f"mflab200 CUDA library not found at {path}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, _int)
    return lib


def declared_symbols() -> list[str]:
    """Every function the public headers declare (parsed from include/*.h)."""
    import re
    names = []
    for h in sorted(glob.glob(os.path.join(INCLUDE, "*.h"))):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(mflab_\w+)\s*\(", text)
    return sorted(set(names))
