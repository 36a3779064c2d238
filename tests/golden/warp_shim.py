"""Pure-Python stand-in for the subset of NVIDIA Warp used by the reference's 2D kernels.

Test infrastructure only. It lets ``make_golden.py`` import and execute the reference's own
``@wp.kernel``/``@wp.func`` source (``warp_weno5_helpers.py``, the V20 deploy core, the FP32 core and
the HLLC adapters) on tiny grids in this container, where ``warp-lang`` is not installed, so that the
golden fixtures come from the reference's code rather than from a restatement of it.

Semantics reproduced:

* ``wp.float64`` values are Python floats (IEEE binary64); ``wp.float32`` values are numpy float32
  scalars, so float32 arithmetic stays float32 (NEP 50 weak Python scalars).
* vectors (``wp.vec4d``, ``wp.types.vector``) are fixed-length lists that cast on construction.
* ``wp.launch`` runs the kernel body once per index of ``dim`` with ``wp.tid()`` returning it.
* ``wp.atomic_add`` is a plain add (the launch loop is sequential).

Known difference from the GPU build: Warp compiles through NVRTC, which contracts ``a*b+c`` into
fused multiply-adds; Python does not. That changes FP64 results by a few ulp per operation.
"""
from __future__ import annotations

import math
import sys
import types as _types

import numpy as np

float64 = float


def float32(x):  # noqa: D401 - mirrors wp.float32(x)
    return np.float32(x)


int32 = int


class _Vec(list):
    LENGTH = 0
    DTYPE = float

    def __init__(self, *args):
        if len(args) == 0:
            super().__init__([self.DTYPE(0.0)] * self.LENGTH)
        elif len(args) == 1 and hasattr(args[0], "__len__"):
            super().__init__([self.DTYPE(a) for a in args[0]])
        else:
            if len(args) != self.LENGTH:
                raise TypeError(f"vector of length {self.LENGTH} built from {len(args)} values")
            super().__init__([self.DTYPE(a) for a in args])

    def __setitem__(self, k, v):
        super().__setitem__(k, self.DTYPE(v))


def _vector_type(length: int, dtype):
    cast = float if dtype is float64 else float32
    return type(f"vec{length}", (_Vec,), {"LENGTH": length, "DTYPE": staticmethod(cast)})


vec3d = _vector_type(3, float64)
vec4d = _vector_type(4, float64)
vec3f = _vector_type(3, float32)
vec4f = _vector_type(4, float32)

types_ns = _types.SimpleNamespace(vector=lambda length, dtype: _vector_type(length, dtype))


def constant(x):
    return x


def func(f):
    return f


def kernel(f=None, **_kwargs):
    if f is None:
        return lambda g: g
    return f


_TID = None


def tid():
    return _TID


class _Array(np.ndarray):
    def numpy(self):
        return np.asarray(self).copy()


def _np_dtype(dtype):
    return np.float32 if dtype is float32 else (np.int32 if dtype is int32 else np.float64)


def array(data=None, dtype=float64, device=None, requires_grad=False, shape=None):
    del device, requires_grad
    if data is None:
        data = np.zeros(shape, dtype=_np_dtype(dtype))
    return np.array(data, dtype=_np_dtype(dtype)).view(_Array)


def zeros(shape, dtype=float64, device=None, requires_grad=False):
    del device, requires_grad
    return np.zeros(shape, dtype=_np_dtype(dtype)).view(_Array)


def array2d(dtype=float64):
    return None


array3d = array2d


def launch(kernel_fn, dim, inputs, device=None, outputs=None):
    global _TID
    del device
    args = list(inputs) + list(outputs or [])
    if isinstance(dim, int):
        for i in range(dim):
            _TID = i
            kernel_fn(*args)
    else:
        for idx in np.ndindex(*dim):
            _TID = tuple(int(v) for v in idx)
            kernel_fn(*args)
    _TID = None


def atomic_add(arr, index, value):
    arr[index] = arr[index] + value


def _unary(f_np, f_math):
    def op(x):
        if isinstance(x, np.floating):
            return f_np(x)
        return f_math(x)
    return op


exp = _unary(np.exp, math.exp)
log = _unary(np.log, math.log)
tanh = _unary(np.tanh, math.tanh)
sqrt = _unary(np.sqrt, math.sqrt)


def abs(x):  # noqa: A001 - Warp name
    return x if x >= 0 else -x


def max(a, b):  # noqa: A001
    return a if a >= b else b


def min(a, b):  # noqa: A001
    return a if a <= b else b


def pow(a, b):  # noqa: A001
    if isinstance(a, np.floating):
        return np.power(a, b)
    return math.pow(a, b)


def init():
    return None


def set_device(_name):
    return None


def synchronize():
    return None


class Tape:  # pragma: no cover - the differentiable paths are not exercised
    def __init__(self, *a, **k):
        raise RuntimeError("warp_shim does not implement Tape")


def install() -> None:
    """Register this module as ``warp`` (and stub matplotlib) in ``sys.modules``."""
    mod = sys.modules[__name__]
    mod.types = types_ns
    sys.modules["warp"] = mod
    if "matplotlib" not in sys.modules:
        mpl = _types.ModuleType("matplotlib")
        mpl.use = lambda *a, **k: None
        plt = _types.ModuleType("matplotlib.pyplot")
        mpl.pyplot = plt
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = plt
