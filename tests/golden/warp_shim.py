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
* ``wp.atomic_add`` / ``atomic_max`` / ``atomic_min`` are plain updates (the launch loop is sequential).
* matrices (``wp.types.matrix``) are indexed ``m[row, column]``; arrays of any rank are numpy arrays.

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

class _Mat:
    SHAPE = (0, 0)
    DTYPE = float

    def __init__(self, *args):
        r, c = self.SHAPE
        self._v = [[self.DTYPE(0.0)] * c for _ in range(r)]
        if len(args) == 1 and isinstance(args[0], _Mat):
            self._v = [list(row) for row in args[0]._v]

    def __getitem__(self, rc):
        r, c = rc
        return self._v[r][c]

    def __setitem__(self, rc, value):
        r, c = rc
        self._v[r][c] = self.DTYPE(value)


def _matrix_type(shape, dtype):
    cast = float if dtype is float64 else float32
    return type(f"mat{shape[0]}{shape[1]}", (_Mat,), {"SHAPE": tuple(shape), "DTYPE": staticmethod(cast)})


types_ns = _types.SimpleNamespace(vector=lambda length, dtype: _vector_type(length, dtype),
                                  matrix=lambda shape, dtype: _matrix_type(shape, dtype))


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

    def __getitem__(self, idx):
        # Warp does not bounds-check reads: some reference kernels load a default stencil before they
        # pick the direction they use, reading one row past the array and discarding the value. Such a
        # read returns 0 here instead of raising.
        if isinstance(idx, tuple) and len(idx) == self.ndim and all(type(i) is int for i in idx):
            if any(i < 0 or i >= n for i, n in zip(idx, self.shape)):
                return 0.0
        return super().__getitem__(idx)

    def zero_(self):
        self[...] = 0
        return self


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
array4d = array2d


def empty(shape, dtype=float64, device=None, requires_grad=False):
    return zeros(shape, dtype, device, requires_grad)


def get_device(_name=None):
    return None


def synchronize_device(_device=None):
    return None


def set_module_options(_options):
    return None


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


def atomic_max(arr, index, value):
    if value > arr[index]:
        arr[index] = value


def atomic_min(arr, index, value):
    if value < arr[index]:
        arr[index] = value


def _unary(f_np, f_math):
    def op(x):
        if isinstance(x, np.float32):
            return f_np(x)
        return f_math(float(x))
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


def to_torch(arr):
    """A torch view of the array's memory (writes through it land in the array), as wp.to_torch."""
    import torch  # noqa: PLC0415

    return torch.from_numpy(np.asarray(arr))


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
