"""The shipped-model geometry fixture (tests/golden/shipped_geometry.json)
against this library's host loader and classifier: each scene rebuilt from
the stored boxes and filter texts loads to the stored grid, voxels and
boundary list, and the host boundary rows agree with the per-group lists."""
import hashlib
import json
import os

import numpy as np
import pytest

from test_gpu_geometry import FIXTURE, sha, write_scene

SMALL = ["room_modes", "sabine-3x4x5-0.9", "dsp"]


@pytest.mark.parametrize("name", SMALL)
def test_fixture_scene_rebuilds_on_the_host(pkg, tmp_path, name):
    f = json.load(open(FIXTURE))[name]
    m = pkg.Model.load_kerkythea(write_scene(tmp_path, f["boxes"], f["dat"]), 0.02)
    (nx, ny, nz), nmat, ncoef = m.dims
    assert [nx, ny, nz] == f["dims"] and nmat == f["nmat"] and ncoef == f["ncoef"]
    assert m.material_names() == f["materials"]
    assert sha(m.voxels()) == f["voxels_sha256"]
    rows = m.boundary()
    assert sha(rows) == f["boundary_sha256"]
    assert np.array_equal(np.bincount(rows[:, 3], minlength=26), f["counts"])
    for g in (0, 7, 20):
        assert np.array_equal(rows[rows[:, 3] == g][:, [0, 1, 2, 4, 5, 6]], m.group_points(g))


def test_boundary_needs_a_device_for_the_gpu_form(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    m = pkg.Model.from_voxels(-np.ones((4, 4, 4), np.int32), np.ones((1, 1), np.float32),
                              np.ones((1, 1), np.float32))
    assert len(m.boundary()) == 0
    with pytest.raises(pkg.AfdError) as ei:
        m.boundary(device=0)
    assert ei.value.status == pkg.afd.ERR_CUDA
