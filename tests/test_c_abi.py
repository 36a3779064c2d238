"""The C ABI of libwsr.so, checked without a GPU: include/wsr.h declares exactly the entry points the Python
binding binds, with the same number of parameters; the built library exports every one of them; the header's
constants are the binding's; and creating a context on a machine without a usable CUDA device fails with a
status and a message saying why (there is no CPU fallback)."""
import ctypes as C
import re
from pathlib import Path

import pytest
import torch

from weno_sr_publishing_b200 import _native as N
from weno_sr_publishing_b200 import adv1d

HEADER = Path(__file__).resolve().parents[1] / "include" / "wsr.h"


def _header_code() -> str:
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _defines() -> dict[str, int]:
    return {k: int(v) for k, v in re.findall(r"^#define (WSR_[A-Z0-9_]+) ([0-9]+)\s*$", _header_code(), flags=re.M)}


def _declarations() -> dict[str, int]:
    """entry point -> number of parameters, from the prototypes of the header"""
    out = {}
    for name, params in re.findall(r"\b(wsr_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", _header_code()):
        parts = [p.strip() for p in params.split(",")]
        out[name] = 0 if parts == ["void"] or parts == [""] else len(parts)
    return out


def _library():
    if not N.LIB_PATH.exists():
        from weno_sr_publishing_b200 import build
        build.build()
    return N.lib()


def test_header_declares_exactly_the_bound_entry_points():
    assert set(_declarations()) == set(N.exported_symbols())


def test_library_exports_every_declared_entry_point_with_matching_arity():
    lib = _library()
    missing = [s for s in N.exported_symbols() if not hasattr(lib, s)]
    assert not missing
    arity = _declarations()
    bound = {s: len(getattr(lib, s).argtypes) for s in N.exported_symbols() if getattr(lib, s).argtypes is not None}
    assert len(bound) == len(arity)  # every entry point has its argument types declared in the binding
    assert {s: arity[s] for s in bound} == bound


def test_header_constants_match_the_binding():
    d = _defines()
    assert {k: d["WSR_METHOD_" + k.upper()] for k in N.METHOD} == N.METHOD
    assert {k: d["WSR_BC_" + k.upper().replace("-", "_")] for k in N.BC} == N.BC
    assert {k: d["WSR_FLUX_" + k.upper()] for k in N.FLUX} == N.FLUX
    assert {k: d["WSR_FLUX3_" + k.upper()] for k in N.FLUX3} == N.FLUX3
    assert {k: d["WSR_INTEG_" + k.upper()] for k in adv1d.INTEG} == adv1d.INTEG
    assert [d["WSR_PROF_" + k.upper()] for k in N.PROF_KINDS] == list(range(len(N.PROF_KINDS)))
    assert d["WSR_PROF_KINDS"] == len(N.PROF_KINDS)
    pairs = {"WSR_OK": N.WSR_OK, "WSR_ERR_ARG": N.WSR_ERR_ARG, "WSR_ERR_CUDA": N.WSR_ERR_CUDA,
             "WSR_ERR_NO_CLOSURE": N.WSR_ERR_NO_CLOSURE, "WSR_BC_Y_HALO": N.BC_Y_HALO, "WSR_HOST_ASYNC": N.HOST_ASYNC,
             "WSR_OPT_ENO_CUTOFF": N.OPT_ENO_CUTOFF, "WSR_OPT_JS_FALLBACK": N.OPT_JS_FALLBACK,
             "WSR_OPT_COUNT": N.OPT_COUNT, "WSR_OPT_Z_HALO": N.OPT_Z_HALO,
             "WSR_OPT_FACE_THREADS_8": N.OPT_FACE_THREADS_8, "WSR_OPT_FACE_THREADS_1": N.OPT_FACE_THREADS_1,
             "WSR_OPT_FACE_THREADS_4": N.OPT_FACE_THREADS_4}
    assert {k: d[k] for k in pairs} == pairs
    # the option flags are distinct bits
    opts = [v for k, v in d.items() if k.startswith("WSR_OPT_")]
    assert all(v & (v - 1) == 0 for v in opts) and len(set(opts)) == len(opts)


def test_context_creation_rejects_a_null_output_pointer():
    lib = _library()
    assert lib.wsr_ctx_create(0, None) == N.WSR_ERR_ARG
    assert lib.wsr_last_error(None) == b"wsr_ctx_create: null output pointer"


@pytest.mark.skipif(torch.cuda.is_available(), reason="a CUDA device is present")
def test_context_creation_without_a_device_fails_and_says_why():
    lib = _library()
    h = C.c_void_p()
    assert lib.wsr_ctx_create(0, C.byref(h)) == N.WSR_ERR_CUDA
    assert not h.value
    assert lib.wsr_last_error(None).decode().startswith("wsr_ctx_create(device 0): cudaSetDevice: ")
    with pytest.raises(RuntimeError, match="wsr_ctx_create failed with status 2: wsr_ctx_create"):
        N.Context(0)
