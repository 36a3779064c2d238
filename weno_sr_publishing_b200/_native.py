"""ctypes binding of libwsr.so (the C ABI declared in include/wsr.h).

The CUDA library is the only compute path: importing this module fails loudly when libwsr.so is
missing, and every call raises on a non-zero status. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwsr.so"

WSR_OK, WSR_ERR_ARG, WSR_ERR_CUDA, WSR_ERR_NO_CLOSURE = 0, 1, 2, 3
METHOD = {"js": 0, "sr_f64": 1, "sr_f32": 2, "sr_bf16": 3, "z": 4, "sr_bf16_tc": 5}
# methods whose weights come from an uploaded MLP closure
SR_METHODS = ("sr_f64", "sr_f32", "sr_bf16", "sr_bf16_tc")
BC = {"transmissive": 0, "periodic": 1, "double-mach": 2}
BC_Y_HALO = 16  # flag: y ghost rows read as stored (slabs of a y-decomposed grid)
FLUX = {"hllc": 0, "force": 1}
HOST_ASYNC = 1  # wsr_euler2d_advance_host: return once queued
FLUX3 = {"evilin": 0, "hllc": 1}
OPT_ENO_CUTOFF, OPT_JS_FALLBACK, OPT_COUNT, OPT_Z_HALO = 1, 2, 4, 8
OPT_FACE_THREADS_8, OPT_FACE_THREADS_1, OPT_FACE_THREADS_4 = 32, 64, 128  # 2D reconstruction kernels: threads per face
PROF_KINDS = ("normal_x", "normal_y", "flux_x", "flux_y", "update", "control")
N_PARAMS5 = 189
PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")

_lib = None
_lock = threading.Lock()


class NativeLibraryMissing(ImportError):
    pass


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise NativeLibraryMissing(
                    f"{LIB_PATH} is not built; run `python -m weno_sr_publishing_b200.build` (needs nvcc)")
            L = C.CDLL(str(LIB_PATH))
            vp, i, d, sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
            L.wsr_ctx_create.argtypes = [i, C.POINTER(vp)]
            L.wsr_ctx_destroy.argtypes = [vp]
            L.wsr_ctx_destroy.restype = None
            L.wsr_last_error.argtypes = [vp]
            L.wsr_last_error.restype = C.c_char_p
            L.wsr_closure_upload.argtypes = [vp, i, C.POINTER(d), i]
            L.wsr_euler2d_workspace_bytes.argtypes = [i, i]
            L.wsr_euler2d_workspace_bytes.restype = sz
            L.wsr_euler2d_stage.argtypes = [vp, vp, vp, vp, i, i, d, d, d, d, i, i, i, i, i, vp, sz, vp]
            L.wsr_euler2d_stage_at.argtypes = [vp, vp, vp, vp, i, i, d, d, d, d, i, i, i, i, i, d, vp, sz, vp]
            L.wsr_euler2d_stage_noalloc.argtypes = [vp, vp, vp, i, i, d, d, d, d, i, i, i, i, i, C.POINTER(d), vp]
            L.wsr_euler2d_w7_workspace_bytes.restype = sz
            L.wsr_euler2d_w7_workspace_bytes.argtypes = [i, i]
            L.wsr_euler2d_w7_rhs.argtypes = [vp, vp, vp, i, i, d, d, d, i, i, i, i, vp, sz, vp]
            L.wsr_euler2d_w7_run.argtypes = [vp, vp, i, i, d, d, d, d, d, d, i, i, i, i, C.POINTER(d), C.POINTER(i),
                                             C.POINTER(d), vp, sz, vp]
            L.wsr_euler2d_w7_counters.argtypes = [vp, vp, sz, i, i, C.POINTER(C.c_ulonglong)]
            L.wsr_euler2d_max_speed.argtypes = [vp, vp, i, i, d, C.POINTER(d), vp, sz, vp]
            L.wsr_euler2d_run.argtypes = [vp, C.POINTER(vp), i, i, d, d, d, d, d, d, i, i, i, i, i, i, i, i,
                                          C.POINTER(d), C.POINTER(i), C.POINTER(d), C.POINTER(i), C.POINTER(i),
                                          vp, sz, vp]
            L.wsr_euler2d_advance_host.argtypes = [vp, vp, C.POINTER(vp), i, i, d, d, d, d, i, i, i, i, i, i, i, vp,
                                                   sz, vp]
            L.wsr_euler2d_host_order.argtypes = [vp, vp]
            L.wsr_euler2d_host_wait.argtypes = [vp, C.POINTER(i), C.POINTER(i)]
            L.wsr_euler2d_slab_begin.argtypes = [vp, vp, i, i, d, d, d, d, d, d, i, vp, sz, vp]
            L.wsr_euler2d_slab_speed_slot.argtypes = [vp, vp, sz, i, i, C.POINTER(vp)]
            L.wsr_euler2d_slab_step.argtypes = [vp, i, i, i, d, d, vp, sz, vp]
            L.wsr_euler2d_slab_stage.argtypes = [vp, vp, vp, vp, i, i, d, d, d, i, i, i, i, i, vp, sz, vp]
            L.wsr_euler2d_slab_status.argtypes = [vp, vp, sz, i, i, C.POINTER(i), C.POINTER(d), C.POINTER(i),
                                                  C.POINTER(d), vp]
            L.wsr_adv1d_workspace_bytes.argtypes = []
            L.wsr_adv1d_workspace_bytes.restype = sz
            L.wsr_adv1d_run.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, i, i, i, i, i, i, C.POINTER(i), C.POINTER(i),
                                        C.POINTER(C.c_ulonglong), vp, sz, vp]
            L.wsr_train1d_workspace_bytes.argtypes = [i, i, i, i]
            L.wsr_train1d_workspace_bytes.restype = sz
            L.wsr_train1d_forward.argtypes = [vp, vp, vp, vp, i, i, d, d, i, i, i, vp, vp, vp, sz, vp]
            L.wsr_train1d_backward.argtypes = [vp, vp, i, i, d, d, i, i, i, vp, vp, vp, sz, vp]
            L.wsr_euler3d_workspace_bytes.argtypes = [i, i, i]
            L.wsr_euler3d_workspace_bytes.restype = sz
            L.wsr_euler3d_stage.argtypes = [vp, vp, i, i, i, d, d, d, d, i, i, i, i, vp, vp, sz, vp]
            L.wsr_euler3d_max_speed.argtypes = [vp, vp, i, i, i, C.POINTER(d), vp, sz, vp]
            L.wsr_euler3d_run.argtypes = [vp, vp, i, i, i, d, d, d, d, d, d, i, i, i, i, vp, vp, C.POINTER(i),
                                          C.POINTER(d), vp, sz, vp]
            L.wsr_euler3d_counters.argtypes = [vp, vp, sz, i, i, i, C.POINTER(C.c_ulonglong)]
            L.wsr_profile_enable.argtypes = [vp, i]
            L.wsr_profile_read.argtypes = [vp, C.POINTER(d), C.POINTER(C.c_longlong)]
            L.wsr_euler2d_counters.argtypes = [vp, vp, sz, i, i, C.POINTER(C.c_ulonglong)]
            L.wsr_probe_peak_flops.argtypes = [vp, i, C.POINTER(d), vp]
            L.wsr_probe_exp_tab.argtypes = [vp, vp, vp, i, vp]
            _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return ["wsr_ctx_create", "wsr_ctx_destroy", "wsr_last_error", "wsr_closure_upload",
            "wsr_euler2d_workspace_bytes", "wsr_euler2d_stage", "wsr_euler2d_stage_at", "wsr_euler2d_w7_workspace_bytes",
            "wsr_euler2d_w7_rhs", "wsr_euler2d_w7_run", "wsr_euler2d_w7_counters", "wsr_euler2d_max_speed", "wsr_euler2d_run",
            "wsr_profile_enable", "wsr_profile_read", "wsr_euler2d_counters", "wsr_probe_peak_flops", "wsr_probe_exp_tab",
            "wsr_adv1d_workspace_bytes", "wsr_adv1d_run", "wsr_train1d_workspace_bytes", "wsr_train1d_forward",
            "wsr_train1d_backward", "wsr_euler3d_workspace_bytes", "wsr_euler3d_stage", "wsr_euler3d_max_speed",
            "wsr_euler3d_run", "wsr_euler3d_counters", "wsr_euler2d_stage_noalloc", "wsr_euler2d_slab_begin",
            "wsr_euler2d_slab_speed_slot", "wsr_euler2d_slab_step", "wsr_euler2d_slab_stage", "wsr_euler2d_slab_status",
            "wsr_euler2d_advance_host", "wsr_euler2d_host_order", "wsr_euler2d_host_wait"]


def pack_params(params) -> np.ndarray:
    """w1..b4 (numpy, torch, leading dim 1 allowed) -> 189 FP64 values in the packed layout."""
    arrs = []
    for k in PARAM_NAMES:
        v = params[k]
        if hasattr(v, "detach"):
            v = v.detach().cpu().numpy()
        arrs.append(np.asarray(v, dtype=np.float64).reshape(-1))
    out = np.ascontiguousarray(np.concatenate(arrs))
    if out.size != N_PARAMS5:
        raise ValueError(f"expected {N_PARAMS5} WENO5 parameters, got {out.size}")
    return out


class Context:
    """One libwsr context per CUDA device (holds the uploaded closure parameters)."""

    def __init__(self, device: int = 0):
        self.device = device
        h = C.c_void_p()
        rc = lib().wsr_ctx_create(device, C.byref(h))
        if rc != WSR_OK:
            msg = lib().wsr_last_error(None).decode(errors="replace")
            raise RuntimeError(f"wsr_ctx_create failed with status {rc}: {msg}")
        self.handle = h
        self._closure_keys: dict[int, bytes] = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and _lib is not None:
            _lib.wsr_ctx_destroy(h)
            self.handle = None

    def check(self, rc: int) -> None:
        if rc == WSR_OK:
            return
        msg = lib().wsr_last_error(self.handle).decode(errors="replace")
        if rc == WSR_ERR_ARG:
            raise ValueError(msg)
        raise RuntimeError(f"libwsr status {rc}: {msg}")

    def profile_enable(self, on: bool = True) -> None:
        self.check(lib().wsr_profile_enable(self.handle, int(on)))

    def profile_read(self) -> dict:
        ms = (C.c_double * len(PROF_KINDS))()
        n = (C.c_longlong * len(PROF_KINDS))()
        self.check(lib().wsr_profile_read(self.handle, ms, n))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(PROF_KINDS)}

    def peak_tflops(self, bits: int, stream=None) -> float:
        out = C.c_double(0.0)
        self.check(lib().wsr_probe_peak_flops(self.handle, bits, C.byref(out), stream))
        return out.value

    def upload_closure(self, packed: np.ndarray) -> None:
        self.upload_closure_kind(5, packed)

    def upload_closure_kind(self, kind: int, packed: np.ndarray) -> None:
        packed = np.ascontiguousarray(packed, dtype=np.float64)
        key = packed.tobytes()
        if self._closure_keys.get(kind) == key:
            return
        self.check(lib().wsr_closure_upload(self.handle, kind, packed.ctypes.data_as(C.POINTER(C.c_double)),
                                            int(packed.size)))
        self._closure_keys[kind] = key


_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    with _lock:
        if device not in _contexts:
            _contexts[device] = None  # placeholder to keep the lock scope simple
    if _contexts[device] is None:
        _contexts[device] = Context(device)
    return _contexts[device]
