"""The Julia ccall layer (multifloatlinearalgebra.jl_b200/julia/MFLAB200.jl)
against the C header: every ccall names a declared entry point, with the
declared number of arguments and matching argument and return types, and the
binding covers the hot-path entry points.  Julia is not installed here, so
the file is checked as text (no GPU)."""
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(REPO, "multifloatlinearalgebra.jl_b200", "julia", "MFLAB200.jl")
HEADERS = [os.path.join(REPO, "include", "mflab200.h")]

# C parameter type -> the Julia ccall type that passes it
C2JL = {
    "int": "Cint", "int64_t": "Int64", "size_t": "Csize_t",
    "double*": "Ptr{Float64}", "const double*": "Ptr{Float64}",
    "int*": "Ptr{Cint}", "const int*": "Ptr{Cint}",
    "int64_t*": "Ptr{Int64}", "const int64_t*": "Ptr{Int64}", "size_t*": "Ptr{Csize_t}",
    "uint8_t*": "Ptr{UInt8}", "const uint8_t*": "Ptr{UInt8}",
    "void*": "Ptr{Cvoid}", "const void*": "Ptr{Cvoid}", "mflab_handle*": "Ptr{Cvoid}",
    "mflab_handle**": "Ptr{Ptr{Cvoid}}", "void**": "Ptr{Ptr{Cvoid}}",
}
RET = {"int": "Cint", "constchar*": "Cstring"}


def _prototypes():
    protos = {}
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"\n(int|const char \*)\s*(mflab_\w+)\s*\(([^;]*?)\);", text, re.S):
            params = []
            body = " ".join(m.group(3).split())
            if body != "void":
                for p in body.split(","):
                    p = p.strip()
                    name = re.match(r"(.*?)(\w+)$", p)
                    typ = name.group(1).replace(" ", "").replace("const", "const ")
                    params.append(typ.strip())
            protos[m.group(2)] = (m.group(1).replace(" ", ""), params)
    return protos


def _split_top(s):
    """split a comma list at nesting depth 0"""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _ccalls():
    text = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(", text):
        i, depth = m.end(), 1
        while depth:
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        parts = _split_top(text[m.end():i - 1])
        sym = re.match(r"\(:(\w+),\s*libmflab\)", parts[0])
        assert sym, parts[0]
        tup = parts[2]
        assert tup.startswith("(") and tup.endswith(")"), tup
        types = [t for t in _split_top(tup[1:-1]) if t]
        calls.append((sym.group(1), parts[1], types, parts[3:]))
    return calls


def _norm(c_type):
    t = c_type.replace("const ", "const ")
    t = re.sub(r"\s+", "", t).replace("const", "const ")
    return t


def test_every_ccall_matches_the_header():
    protos = _prototypes()
    calls = _ccalls()
    assert len(calls) > 40
    for name, ret, types, args in calls:
        assert name in protos, f"{name} is not declared in include/mflab200.h"
        cret, cparams = protos[name]
        assert RET[cret] == ret, (name, cret, ret)
        assert len(types) == len(cparams), (name, types, cparams)
        assert len(args) == len(cparams), (name, "argument count", len(args), len(cparams))
        for jt, ct in zip(types, cparams):
            key = _norm(ct)
            assert key in C2JL, (name, ct)
            assert C2JL[key] == jt, (name, ct, jt)


@pytest.mark.parametrize("entry", [
    "mflab_gemm", "mflab_gemm_ozaki_crt", "mflab_gemm_ozaki", "mflab_syrk_lower",
    "mflab_syrk_lower_ozaki", "mflab_gemmt_lower", "mflab_trsm", "mflab_trmm", "mflab_gemv",
    "mflab_symv", "mflab_dot", "mflab_potrf", "mflab_potrf_ozaki", "mflab_potrs", "mflab_getrf",
    "mflab_getrf_ozaki", "mflab_getrs", "mflab_sytrf", "mflab_sytrs", "mflab_pstrf", "mflab_qr",
    "mflab_apply_q", "mflab_residual", "mflab_residual_mixed", "mflab_backward_error",
    "mflab_h2d_interleaved", "mflab_d2h_interleaved", "mflab_max_abs", "mflab_add_widened",
    "mflab_device_status", "mflab_create", "mflab_destroy", "mflab_malloc", "mflab_free"])
def test_binding_covers_the_hot_path(entry):
    assert entry in {c[0] for c in _ccalls()}


def test_reference_generics_are_extended():
    """the binding adds methods to MultiFloatLinearAlgebra's own functions
    (src/MultiFloatLinearAlgebra.jl:34-49) rather than defining new names"""
    text = open(JL).read()
    imported = re.search(r"import MultiFloatLinearAlgebra:(.*?)\n\n", text, re.S).group(1)
    for fn in ("gemm!", "syrk!", "gemmt!", "trsm!", "trsv!", "cholesky!", "lu!", "ldlt!",
               "ldiv!", "solve", "residual!", "normwise_backward_error"):
        assert fn in imported
        assert re.search(r"^" + re.escape(fn) + r"\(|^function " + re.escape(fn) + r"\(", text,
                         re.M), fn
