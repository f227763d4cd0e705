"""Geometry set-up on the GPU (geometry.cu): the Kerkythea rasterisation and
the LRS boundary classification give the host loader's voxels and the host
classifier's boundary list bit for bit, in the same z-y-x order, and the same
error naming the same first unphysical cell. Pinned on the reference's
shipped models through tests/golden/shipped_geometry.json."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "shipped_geometry.json")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def write_scene(d, boxes, dat):
    models = []
    for name, a0, a1, b0, b1, c0, c1 in boxes:
        pts = "".join('<P xyz="%s %s %s"/>' % (a, b, c) for a in (a0, a1) for b in (b0, b1) for c in (c0, c1))
        models.append('<Object Type="Model" Name="%s"><Object Type="Surface"><Parameter Name="Vertex List">%s'
                      '</Parameter></Object></Object>' % (name, pts))
    (d / "model.xml").write_text('<Root><Object Type="Scene">%s</Object></Root>' % "".join(models))
    for fn, text in dat.items():
        (d / fn).write_text(text)
    return str(d / "model.xml")


def model(pkg, vox, nmat=3):
    return pkg.Model.from_voxels(vox, np.ones((nmat, 2), np.float32), np.ones((nmat, 2), np.float32))


@pytest.mark.parametrize("dims,seed", [((30, 26, 22), 1), ((37, 29, 23), 2), ((130, 67, 45), 3),
                                       ((300, 40, 24), 4), ((64, 64, 64), 5)])
def test_boundary_list_matches_host(pkg, dims, seed):
    W = pkg.workloads
    vox = W.room(*dims, 63, n_boxes=6, nmat=3, seed=seed, box_min=2, box_max=9)
    m = model(pkg, vox)
    host = m.boundary()
    dev = m.boundary(device=0)
    assert len(host) > 0
    assert dev.dtype == np.int32 and dev.shape == host.shape
    assert np.array_equal(dev, host)
    # rows agree with the per-group lists and counts of the host classifier
    counts = m.classify()
    assert np.array_equal(np.bincount(dev[:, 3], minlength=26), counts)
    g6 = m.group_points(6)
    assert np.array_equal(dev[dev[:, 3] == 6][:, [0, 1, 2, 4, 5, 6]], g6)


def test_small_and_degenerate_grids(pkg):
    # 3x3x3: the centre cell alone is interior
    for solid in ([(2, 1, 1)], [(2, 1, 1), (1, 2, 1)], [(2, 1, 1), (1, 0, 1), (1, 1, 2)], []):
        vox = -np.ones((3, 3, 3), np.int32)
        for k, (x, y, z) in enumerate(solid):
            vox[z, y, x] = k
        m = model(pkg, vox)
        assert np.array_equal(m.boundary(device=0), m.boundary())
    # a grid thinner than three cells has no interior rows
    vox = np.zeros((5, 5, 2), np.int32)
    vox[2, 2, :] = -1
    m = model(pkg, vox)
    assert len(m.boundary(device=0)) == 0 == len(m.boundary())


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_first_unphysical_cell_is_reported(pkg, seed):
    rng = np.random.default_rng(seed)
    vox = np.where(rng.random((20, 24, 40)) < 0.12, rng.integers(0, 3, (20, 24, 40)), -1).astype(np.int32)
    m = model(pkg, vox)
    with pytest.raises(pkg.AfdError) as eh:
        m.boundary()
    with pytest.raises(pkg.AfdError) as ed:
        m.boundary(device=0)
    assert ed.value.status == eh.value.status == pkg.afd.ERR_GEOMETRY
    assert str(ed.value) == str(eh.value)
    assert "Unphysical surfaces encountered at cell" in str(ed.value)


def test_rasterisation_later_boxes_overwrite(pkg, tmp_path):
    # overlapping boxes of three materials in file order, one box wholly
    # below zero (skipped) and one reaching below zero (clamped)
    rng = np.random.default_rng(21)
    boxes = []
    names = ["wall_concrete", "desk_wood", "pane_glass"]
    for k in range(40):
        lo = rng.uniform(-0.1, 1.1, 3)
        hi = lo + rng.uniform(0.0, 0.5, 3)
        a0, a1 = lo[0], hi[0]
        c0, c1 = lo[1], hi[1]
        b0, b1 = -hi[2], -lo[2]  # z = -b
        boxes.append([names[k % 3]] + ["%r" % float(np.float32(v)) for v in (a0, a1, b0, b1, c0, c1)])
    boxes.append(["under_wood", "-0.5", "-0.2", "0.1", "0.3", "0.1", "0.2"])
    dat = {"concrete_a.dat": "0.1\n0.02\n", "concrete_b.dat": "1.0\n0.1\n", "wood_a.dat": "0.5\n0.1\n",
           "wood_b.dat": "1.0\n-0.2\n", "glass_a.dat": "0.05\n0.0\n", "glass_b.dat": "1.0\n0.0\n"}
    path = write_scene(tmp_path, boxes, dat)
    for res in (0.02, 0.013):
        host = pkg.Model.load_kerkythea(path, res)
        dev = pkg.Model.load_kerkythea(path, res, device=0)
        assert dev.dims == host.dims
        assert np.array_equal(dev.voxels(), host.voxels())
        assert dev.material_names() == host.material_names()
        for x, y in zip(dev.coefs(), host.coefs()):
            assert np.array_equal(x, y)


def test_shipped_models(pkg, tmp_path):
    fx = json.load(open(FIXTURE))
    for name, f in sorted(fx.items()):
        d = tmp_path / name
        d.mkdir()
        path = write_scene(d, f["boxes"], f["dat"])
        m = pkg.Model.load_kerkythea(path, 0.02, device=0)
        (nx, ny, nz), nmat, ncoef = m.dims
        assert [nx, ny, nz] == f["dims"] and nmat == f["nmat"] and ncoef == f["ncoef"], name
        assert sha(m.voxels()) == f["voxels_sha256"], name
        rows = m.boundary(device=0)
        assert len(rows) == f["n_boundary"] and sha(rows) == f["boundary_sha256"], name


def test_simulation_load_uses_the_device_geometry(pkg, tmp_path):
    fx = json.load(open(FIXTURE))
    f = fx["room_modes"]
    path = write_scene(tmp_path, f["boxes"], f["dat"])
    sim = pkg.Simulation()
    sim.Load(path)
    info = sim.info()
    assert [info.nx, info.ny, info.nz] == f["dims"]
    assert info.n_boundary == f["n_boundary"]
    assert list(info.group_counts) == f["counts"]
    sim.close()
    # SetModel: the range check and the unphysical-pattern error
    vox = -np.ones((8, 8, 8), np.int32)
    vox[:, :, 3] = 0
    vox[:, :, 5] = 0
    sim = pkg.Simulation()
    with pytest.raises(pkg.AfdError) as ei:
        sim.SetModel(model(pkg, vox, nmat=1))
    assert ei.value.status == pkg.afd.ERR_GEOMETRY and "Unphysical" in str(ei.value)
    sim.close()


@pytest.mark.parametrize("faces,width", [(63, 6), (1 | 8 | 32, 9), (2 | 4 | 8, 40)])
def test_pml_cells_on_a_padded_grid(pkg, faces, width):
    """The FIXED-scheme PML cells (plain air, 2 <= x,y,z <= n-3, inside an
    enabled slab) as the device masks count them, on a grid that SetMinSize
    makes larger than the model (the cells past the model are air)."""
    W = pkg.workloads
    vox = W.room(40, 36, 30, 63, n_boxes=3, nmat=2, seed=31, box_min=3, box_max=7)
    m = model(pkg, vox, nmat=2)
    sim = pkg.Simulation(mode=1)
    sim.SetModel(m)
    sim.SetMinSize(0.02 * 70, 0.02 * 40, 0.02 * 30)
    sim.prepare(1)
    info = sim.info()
    gx, gy, gz = info.nx, info.ny, info.nz
    assert gx > 40
    sim.SetPml(width, faces=faces, ksi=W.ksi_arrays((gx, gy, gz), width, faces))
    sim.prepare(1)
    solid = np.zeros((gz, gy, gx), bool)
    solid[:30, :36, :40] = vox != -1
    lrs = np.zeros_like(solid)
    rows = m.boundary(device=0)
    lrs[rows[:, 2], rows[:, 1], rows[:, 0]] = True
    z, y, x = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
    slab = np.zeros_like(solid)
    for bit, c, n in ((1, x, gx), (4, y, gy), (16, z, gz)):
        if faces & bit:
            slab |= c < width
        if faces & (bit << 1):
            slab |= c > n - width - 1
    inner = (x >= 2) & (x <= gx - 3) & (y >= 2) & (y <= gy - 3) & (z >= 2) & (z <= gz - 3)
    want = int((~solid & ~lrs & inner & slab).sum())
    assert sim.info().n_pml_cells == want
    sim.close()
