"""CPU: host-side logic of the WENO7 2D and slab modules that needs no GPU (closure loading and its errors, the
3D slab partition)."""
from __future__ import annotations

import numpy as np
import pytest

from weno_sr_publishing_b200 import euler2d_w7 as E7
from weno_sr_publishing_b200 import slabs as S
from weno_sr_publishing_b200.checkpoint import MODELS_DIR

CK7 = MODELS_DIR / "weno7_sr_fp64_step016750.npz"


def test_weno7_closure_from_path_dict_and_beta_model():
    a = E7.as_closure7(CK7)
    b = E7.as_closure7({k: v for k, v in np.load(CK7).items() if k != "meta_json"})
    c = E7.as_closure7(E7.Weno7PointBeta(CK7, "cpu", 1.4))
    assert a.kind == b.kind == c.kind == 7 and a.packed.size == 908
    np.testing.assert_array_equal(a.packed, b.packed)
    np.testing.assert_array_equal(a.packed, c.packed)


def test_weno7_closure_rejects_a_weno5_checkpoint_and_unknown_methods():
    with pytest.raises(ValueError):
        E7.as_closure7(MODELS_DIR / "weno5_sr_fp64_step012250.npz")
    with pytest.raises(ValueError):
        E7._method("sr_f32")
    assert E7.METHOD == {"js": 0, "z": 4, "sr_f64": 1}


def test_3d_slab_grids_cover_the_planes():
    for nz, world in ((88, 1), (88, 3), (88, 8), (30, 4)):
        grids = [S.slab_grid3(224, 88, nz, 0.01, 0.011, 0.012, world, r) for r in range(world)]
        assert grids[0].z0 == 0 and sum(g.nz for g in grids) == nz
        assert all(a.z0 + a.nz == b.z0 for a, b in zip(grids, grids[1:]))
        assert all(g.dz == 0.012 and g.padded_shape == (g.nz + 6, 94, 230, 5) for g in grids)
    q = np.arange(36 * 4 * 4 * 5, dtype=np.float64).reshape(36, 4, 4, 5)
    parts = [S.split3(q, 30, 4, r) for r in range(4)]
    assert sum(p.shape[0] - 6 for p in parts) == 30
    np.testing.assert_array_equal(np.concatenate([p[3:-3] for p in parts]), q[3:-3])
    with pytest.raises(ValueError):
        S.slab_grid3(8, 8, 8, 0.1, 0.1, 0.1, 3, 0)  # slabs of 2 planes
