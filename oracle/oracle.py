"""ctypes front end of the CPU oracle (test infrastructure).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module. It is the
checker of the CUDA path and the timed CPU baseline, never part of the product path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

METHOD = {"js": 0, "sr_f64": 1, "sr_f32": 2, "sr_bf16": 3, "z": 4}
BC = {"transmissive": 0, "periodic": 1, "double-mach": 2}
FLUX = {"hllc": 0, "force": 1}
N_PARAMS5 = 189
PARAM_NAMES = ("w1", "b1", "w2", "b2", "w3", "b3", "w4", "b4")

_LIBS: dict[str, C.CDLL] = {}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def _lib(fast: bool = False) -> C.CDLL:
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name not in _LIBS:
        path = HERE / name
        if not path.exists():
            from oracle import build_oracle  # noqa: PLC0415
            build_oracle.build()
        lib = C.CDLL(str(path))
        lib.or_euler2d_run.restype = C.c_int
        lib.or_euler2d_run.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _fp,
                                       C.c_int, C.c_int, _dp, C.c_int, C.POINTER(C.c_double)]
        lib.or_euler2d_stage.restype = C.c_int
        lib.or_euler2d_stage.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _fp]
        lib.or_euler2d_stage_at.restype = C.c_int
        lib.or_euler2d_stage_at.argtypes = lib.or_euler2d_stage.argtypes + [C.c_double]
        lib.or_euler2d_max_speed.restype = C.c_double
        lib.or_euler2d_max_speed.argtypes = [_dp, C.c_int, C.c_int, C.c_double]
        lib.or_hllc_flux_flat.argtypes = [_dp, _dp, C.c_int, C.c_double, _dp]
        lib.or_force_flux_flat.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double, _dp]
        lib.or_closure_weights_batch.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp, _fp, _dp]
        lib.or_reconstruct_batch.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp, _fp, _dp]
        lib.or_reconstruct_h_batch.argtypes = [_dp, C.c_int, C.c_int, C.c_int, _dp, _fp, C.c_double, _dp]
        lib.or_mlp_ratios_batch.argtypes = [_dp, C.c_int, C.c_int, _dp, _fp, _dp]
        lib.or_num_threads.restype = C.c_int
        _vp = C.c_void_p
        lib.or_euler3d_run.restype = C.c_int
        lib.or_euler3d_run.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _fp,
                                       _vp, _dp, C.c_int]
        lib.or_euler3d_stage.restype = C.c_int
        lib.or_euler3d_stage.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_int, C.c_int, C.c_int, _dp, _fp, C.c_void_p, C.c_int]
        lib.or_euler3d_max_speed.restype = C.c_double
        lib.or_euler3d_max_speed.argtypes = [_dp, C.c_int, C.c_int, C.c_int]
        lib.or_hllc5_batch.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
        lib.or_w7_face.restype = C.c_double
        lib.or_w7_face.argtypes = [_dp, C.c_int]
        lib.or_w7_gauss.restype = C.c_double
        lib.or_w7_gauss.argtypes = [_dp, C.c_int]
        lib.or_w7_rhs.restype = C.c_int
        lib.or_w7_rhs.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                  C.c_int, _dp]
        lib.or_w7sr_beta.restype = None
        lib.or_w7sr_beta.argtypes = [_dp, _dp, _dp]
        lib.or_w7sr_face.restype = C.c_double
        lib.or_w7sr_face.argtypes = [_dp, C.c_int, _dp]
        lib.or_w7sr_gauss.restype = C.c_double
        lib.or_w7sr_gauss.argtypes = [_dp, C.c_int, _dp]
        lib.or_w7z_face.restype = C.c_double
        lib.or_w7z_face.argtypes = [_dp, C.c_int, C.c_double]
        lib.or_w7z_gauss.restype = C.c_double
        lib.or_w7z_gauss.argtypes = [_dp, C.c_int, C.c_double]
        lib.or_w7_run.restype = C.c_int
        lib.or_w7_run.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int, C.POINTER(C.c_double)]
        lib.or_evilin5_batch.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, _dp]
        _LIBS[name] = lib
    return _LIBS[name]


def pack_params(params: dict, dtype=np.float64) -> np.ndarray:
    """Flatten w1..b4 (leading dim 1 allowed) into the packed [in][out] row-major layout."""
    return np.ascontiguousarray(np.concatenate([np.asarray(params[k]).reshape(-1) for k in PARAM_NAMES]),
                                dtype=dtype)


def _params(params):
    if params is None:
        return np.zeros(N_PARAMS5), np.zeros(N_PARAMS5, dtype=np.float32)
    return pack_params(params, np.float64), pack_params(params, np.float32)


def closure_weights(q: np.ndarray, head: int, method: str, params=None) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 5)
    out = np.zeros((q.shape[0], 3))
    p64, p32 = _params(params)
    _lib().or_closure_weights_batch(q, q.shape[0], head, METHOD[method], p64, p32, out)
    return out


def reconstruct(q: np.ndarray, head: int, method: str, params=None) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 5)
    out = np.zeros(q.shape[0])
    p64, p32 = _params(params)
    _lib().or_reconstruct_batch(q, q.shape[0], head, METHOD[method], p64, p32, out)
    return out


def reconstruct_h(q: np.ndarray, head: int, method: str, h: float, params=None) -> np.ndarray:
    """reconstruct() with the grid spacing of the stencil's direction (WENO-Z's eps = h^2)."""
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 5)
    out = np.zeros(q.shape[0])
    p64, p32 = _params(params)
    _lib().or_reconstruct_h_batch(q, q.shape[0], head, METHOD[method], p64, p32, float(h), out)
    return out


def mlp_ratios(features: np.ndarray, method: str, params) -> np.ndarray:
    x = np.ascontiguousarray(features, dtype=np.float64).reshape(-1, 5)
    out = np.zeros((x.shape[0], 3))
    p64, p32 = _params(params)
    _lib().or_mlp_ratios_batch(x, x.shape[0], METHOD[method], p64, p32, out)
    return out


def hllc(ul, ur, direction: int, gamma: float = 1.4) -> np.ndarray:
    out = np.zeros(4)
    _lib().or_hllc_flux_flat(np.ascontiguousarray(ul, dtype=np.float64), np.ascontiguousarray(ur, dtype=np.float64),
                             direction, gamma, out)
    return out


def force(ul, ur, direction: int, c: float, gamma: float = 1.4) -> np.ndarray:
    out = np.zeros(4)
    _lib().or_force_flux_flat(np.ascontiguousarray(ul, dtype=np.float64), np.ascontiguousarray(ur, dtype=np.float64),
                              direction, c, gamma, out)
    return out


def max_speed(u: np.ndarray, nx: int, ny: int, gamma: float = 1.4) -> float:
    return float(_lib().or_euler2d_max_speed(np.ascontiguousarray(u, dtype=np.float64), nx, ny, gamma))


Y_HALO = 16


def euler2d_stage(u_stage, u0, u_out, nx, ny, dx, dy, dt, rk, method, bc="transmissive", flux="hllc",
                  params=None, gamma=1.4, boundary_time=0.0, y_halo=False) -> np.ndarray:
    """One SSPRK3 stage; returns a copy of u_out with its interior overwritten. y_halo: the y ghost rows of
    u_stage are used as given (a slab of a y-decomposed grid), x ghosts follow `bc`."""
    out = np.array(u_out, dtype=np.float64, copy=True)
    p64, p32 = _params(params)
    rc = _lib().or_euler2d_stage_at(np.ascontiguousarray(u_stage, dtype=np.float64),
                                    np.ascontiguousarray(u0, dtype=np.float64), out, nx, ny, dx, dy, gamma, dt, rk,
                                    METHOD[method], BC[bc] | (Y_HALO if y_halo else 0), FLUX[flux], p64, p32,
                                    float(boundary_time))
    if rc != 0:
        raise MemoryError("oracle stage allocation failed")
    return out


def euler2d_run(initial, nx, ny, dx, dy, cfl, t_end, method, bc="transmissive", flux="hllc", params=None,
                gamma=1.4, check_health=False, fixed_steps=0, max_steps=100000, fast=False):
    """Time loop of the reference adapters. Returns (final padded array, dts, steps, t)."""
    init = np.ascontiguousarray(initial, dtype=np.float64)
    out = np.zeros_like(init)
    dts = np.zeros(max_steps)
    t = C.c_double(0.0)
    p64, p32 = _params(params)
    steps = _lib(fast).or_euler2d_run(init, out, nx, ny, dx, dy, gamma, cfl, t_end, METHOD[method], BC[bc],
                                      FLUX[flux], p64, p32, int(check_health), fixed_steps, dts, max_steps,
                                      C.byref(t))
    if steps < 0:
        raise MemoryError("oracle run allocation failed")
    return out, list(dts[:min(steps, max_steps)]), steps, t.value


def num_threads(fast: bool = True) -> int:
    return int(_lib(fast).or_num_threads())


FLUX3 = {"evilin": 0, "hllc": 1}


def euler3d_run(q, nx, ny, nz, dx, dy, dz, cfl, steps, method, flux="evilin", params=None, inflow=None,
                t_start=0.0, t_end=1.0e30, stage_only=False, fast=False):
    """Advance the padded 3D state q[nz+6][ny+6][nx+6][5] by `steps` steps (a copy is returned with the
    per-step dt). stage_only: only the first RK stage of the first step."""
    out = np.array(q, dtype=np.float64, copy=True, order="C")
    p64, p32 = _params(params)
    dts = np.zeros(max(steps, 1))
    inf = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
    taken = _lib(fast).or_euler3d_run(out, nx, ny, nz, dx, dy, dz, cfl, t_start, t_end, steps, METHOD[method],
                                      FLUX3[flux], p64, p32, None if inf is None else inf.ctypes.data, dts,
                                      int(stage_only))
    if taken < 0:
        raise MemoryError("oracle allocation failed")
    return out, dts[:taken]


def euler3d_stage(q, q0, nx, ny, nz, dx, dy, dz, dt, stage, method, flux="evilin", params=None, inflow=None,
                  z_halo=False) -> None:
    """One RK stage of the 3D oracle on q in place (numpy, padded), q0 the caller's stage-start copy (written at
    stage 1, read at 2 and 3); z_halo: the z ghost planes of q are used as given."""
    p64, p32 = _params(params)
    keep = None if inflow is None else np.ascontiguousarray(inflow, dtype=np.float64)
    if not (q.flags.c_contiguous and q0.flags.c_contiguous and q.dtype == q0.dtype == np.float64):
        raise ValueError("q and q0 must be C-contiguous float64 arrays")
    rc = _lib().or_euler3d_stage(q, q0, nx, ny, nz, dx, dy, dz, dt, stage, METHOD[method], FLUX3[flux], p64, p32,
                                 None if keep is None else keep.ctypes.data_as(C.c_void_p), int(bool(z_halo)))
    if rc != 0:
        raise MemoryError("oracle allocation failed")


def euler3d_max_speed(q, nx, ny, nz) -> float:
    return float(_lib().or_euler3d_max_speed(np.ascontiguousarray(q, dtype=np.float64), nx, ny, nz))


def hllc5(ul, ur, direction: int) -> np.ndarray:
    ul = np.ascontiguousarray(ul, dtype=np.float64).reshape(-1, 5)
    ur = np.ascontiguousarray(ur, dtype=np.float64).reshape(-1, 5)
    out = np.empty_like(ul)
    _lib().or_hllc5_batch(ul, ur, ul.shape[0], direction, out)
    return out


def evilin5(ul, ur, direction: int, dt_dx: float) -> np.ndarray:
    ul = np.ascontiguousarray(ul, dtype=np.float64).reshape(-1, 5)
    ur = np.ascontiguousarray(ur, dtype=np.float64).reshape(-1, 5)
    out = np.empty_like(ul)
    _lib().or_evilin5_batch(ul, ur, ul.shape[0], direction, dt_dx, out)
    return out


# ------------------------------------------------------------------------------------------------
# 2D Euler WENO7-JS with Shu RK4 (padded [ny+8][nx+8][4], ghost width 4)
# ------------------------------------------------------------------------------------------------
BC7 = {"transmissive": 0, "outflow": 0, "periodic": 1}


def w7_face(q, lr: int) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    return np.array([_lib().or_w7_face(np.ascontiguousarray(r), lr) for r in q])


def w7_gauss(q, lr: int) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    return np.array([_lib().or_w7_gauss(np.ascontiguousarray(r), lr) for r in q])


def w7z_face(q, lr: int, h: float) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    return np.array([_lib().or_w7z_face(np.ascontiguousarray(r), lr, h) for r in q])


def w7z_gauss(q, lr: int, h: float) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    return np.array([_lib().or_w7z_gauss(np.ascontiguousarray(r), lr, h) for r in q])


W7_KIND = {"js": 0, "z": 1, "sr_f64": 2}
N_PARAMS7 = 908


def _w7_params(method: str, params) -> np.ndarray:
    if method not in W7_KIND:
        raise ValueError(f"unsupported WENO7 method {method!r}")
    if method != "sr_f64":
        return np.zeros(N_PARAMS7)
    packed = pack_params(params, np.float64) if isinstance(params, dict) else np.ascontiguousarray(params, np.float64)
    if packed.size != N_PARAMS7:
        raise ValueError(f"WENO7 closure needs {N_PARAMS7} parameters, got {packed.size}")
    return packed


def w7sr_beta(q, params) -> np.ndarray:
    """Betas of the WENO7-SR closure (the beta provider's _mlp_beta) on 7-point stencils, [n][4]."""
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    p = _w7_params("sr_f64", params)
    out = np.zeros((q.shape[0], 4))
    for r in range(q.shape[0]):
        b = np.zeros(4)
        _lib().or_w7sr_beta(np.ascontiguousarray(q[r]), p, b)
        out[r] = b
    return out


def w7sr_face(q, lr: int, params) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    p = _w7_params("sr_f64", params)
    return np.array([_lib().or_w7sr_face(np.ascontiguousarray(r), lr, p) for r in q])


def w7sr_gauss(q, lr: int, params) -> np.ndarray:
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 7)
    p = _w7_params("sr_f64", params)
    return np.array([_lib().or_w7sr_gauss(np.ascontiguousarray(r), lr, p) for r in q])


def w7_rhs(u, nx, ny, dx, dy, bc="periodic", reverse=False, gamma=1.4, method="js", params=None) -> np.ndarray:
    """L(u) (or L~(u)) on the interior [ny][nx][4]; method "js", "z" (WENO-Z, eps = h^3) or "sr_f64" (the
    FP64 WENO7 closure `params`, a checkpoint dict or 908 packed values)."""
    p = _w7_params(method, params)
    src = np.array(u, dtype=np.float64, copy=True, order="C")
    out = np.zeros((ny, nx, 4))
    if _lib().or_w7_rhs(src, out, nx, ny, dx, dy, gamma, BC7[bc], int(bool(reverse)), W7_KIND[method], p):
        raise MemoryError("oracle allocation failed")
    return out


def w7_run(u, nx, ny, dx, dy, cfl, t_end, bc="periodic", max_steps=1_000_000, gamma=1.4, fast=False,
           method="js", params=None):
    """run_from_initial of the WENO7 point RK4 path (run_from_initial_mlp for "sr_f64"). Returns (final padded
    state, dts, steps, t)."""
    p = _w7_params(method, params)
    out = np.array(u, dtype=np.float64, copy=True, order="C")
    dts = np.zeros(min(max_steps, 1 << 20))
    t = C.c_double(0.0)
    steps = _lib(fast).or_w7_run(out, nx, ny, dx, dy, gamma, cfl, t_end, BC7[bc], W7_KIND[method], p, max_steps,
                                 dts, dts.size, C.byref(t))
    if steps < 0:
        raise MemoryError("oracle allocation failed")
    return out, list(dts[:steps]), steps, t.value
