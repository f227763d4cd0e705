"""C ABI and host-side logic, no GPU needed: the library loads and exports
every entry point include/afd.h declares; the Kerkythea loader, voxeliser
and boundary classification agree with independent restatements; the FP64
filter check works on the host; simulations fail cleanly without a device.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "afd.h")
# the reference tree, when present on this machine (the shipped-model checks
# skip without it); the oracle's build recipe reads the same variable
REFERENCE_MODELS = os.path.join(os.environ.get("ANC_FIELD_REFERENCE", "/root/reference"), "examples", "models")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(afd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_entry_point(pkg):
    lib = pkg.afd.library()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(pkg.afd.EXPORTS) == names


def test_default_params_are_the_reference_constants(pkg):
    p = pkg.default_params()
    # simulation.hpp:162-166, main.cpp:118
    assert np.float32(p.dx) == np.float32(0.02) and np.float32(p.c) == np.float32(340.0)
    assert np.float32(p.dt) == np.float32(3.125e-5) and p.fs == 32000.0
    assert p.mode == pkg.afd.MODE_REF and p.batch == 1


def test_create_without_device_fails_cleanly(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Simulation()
    assert ei.value.status == pkg.afd.ERR_CUDA
    assert "no CUDA device" in str(ei.value)


def test_fp16_storage_needs_fixed_scheme(pkg):
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Simulation(mode=pkg.afd.MODE_REF, storage=pkg.afd.STORE_FP16)
    assert ei.value.status == pkg.afd.ERR_ARG
    assert "FIXED" in str(ei.value)


# ---------------------------------------------------------------- classifier
_MASKS = [1, 2, 4, 8, 16, 32, 5, 9, 17, 33, 6, 10, 18, 34, 20, 36, 24, 40, 21, 37, 25, 41, 22, 38, 26, 42]


def classify_numpy(vox):
    """LrsData::Init (lrs-data.hpp:154-210) restated with numpy."""
    nz, ny, nx = vox.shape
    s = vox != -1
    c = (slice(1, -1),) * 3
    air = ~s[c]
    nb = [s[1:-1, 1:-1, 2:], s[1:-1, 1:-1, :-2], s[1:-1, 2:, 1:-1], s[1:-1, :-2, 1:-1], s[2:, 1:-1, 1:-1],
          s[:-2, 1:-1, 1:-1]]
    mask = sum(n.astype(np.int64) << d for d, n in enumerate(nb)) * air
    counts = np.zeros(26, np.int64)
    for g, m in enumerate(_MASKS):
        counts[g] = int((mask == m).sum())
    bad = int(((mask != 0) & ~np.isin(mask, _MASKS)).sum())
    return counts, bad


def shell_room(nx, ny, nz, seed):
    import ancfield_b200.workloads as W
    return W.room(nx, ny, nz, 63, n_boxes=3, nmat=3, seed=seed, box_min=3, box_max=8)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_classification_matches_numpy_restatement(pkg, seed):
    vox = shell_room(30, 26, 22, seed)
    m = pkg.Model.from_voxels(vox, np.ones((3, 2), np.float32), np.ones((3, 2), np.float32))
    counts, bad = classify_numpy(vox)
    assert bad == 0
    assert np.array_equal(m.classify(), counts)
    # per-group point lists: scan order z-y-x, materials in X_P..Z_M order
    for g in (0, 6, 25):
        pts = m.group_points(g)
        assert len(pts) == counts[g]
        if len(pts):
            keys = pts[:, 2] * 10**6 + pts[:, 1] * 10**3 + pts[:, 0]
            assert np.all(np.diff(keys) > 0)


def test_unphysical_pattern_is_rejected(pkg):
    vox = -np.ones((8, 8, 8), np.int32)
    vox[:, :, 3] = 0
    vox[:, :, 5] = 0  # one-cell gap between two slabs: opposite solid neighbours
    m = pkg.Model.from_voxels(vox, np.ones((1, 1), np.float32), np.ones((1, 1), np.float32))
    with pytest.raises(pkg.AfdError) as ei:
        m.classify()
    assert ei.value.status == pkg.afd.ERR_GEOMETRY
    assert "Unphysical" in str(ei.value)


# ---------------------------------------------------------- Kerkythea loader
XML = """<?xml version="1.0"?>
<!-- model.xml: a hand-written scene -->
<Root Label="Default Kernel" Name="" Type="Kernel">
<Object Identifier="./Cameras/x" Type="Camera"><Parameter Name="Vertex List"><P xyz="9 9 9"/></Parameter></Object>
<Object Identifier="./Scenes/Default" Label="Default Scene" Name="scene" Type="Scene">
{models}
</Object>
</Root>
"""
MODEL = """<Object Identifier="./Models/{name}" Label="Default Model" Name="{name}" Type="Model">
  <Object Identifier="Triangular Mesh" Label="Triangular Mesh" Name="" Type="Surface">
    <Parameter Name="Vertex List" Type="Point3D List" Value="8">
{points}
    </Parameter>
    <Parameter Name="Normal List" Type="Point3D List" Value="1"><P xyz="0 0 1"/></Parameter>
  </Object>
</Object>"""


def box_points(x0, x1, y0, y1, z0, z1):
    # file coordinates (a, b, c) with (x, y, z) = (a, c, -b)
    pts = []
    for x in (x0, x1):
        for y in (y0, y1):
            for z in (z0, z1):
                pts.append('      <P xyz="%r %r %r"/>' % (x, -z, y))
    return "\n".join(pts)


def kerkythea_numpy(boxes, res, mats):
    """LoadBoxes + Kerkythea ctor (kerkythea.hpp:63-196) restated with numpy
    FP32 arithmetic: AABB, clamp of the minimum at 0, grid RoundTo(int(max /
    res) + 1, 32), inclusive rasterisation in file order."""
    f32 = np.float32
    res = f32(res)
    ext = []
    for (x0, x1, y0, y1, z0, z1), m in boxes:
        e = [max(f32(x0), f32(0)), f32(x1), max(f32(y0), f32(0)), f32(y1), max(f32(z0), f32(0)), f32(z1)]
        ext.append((e, m))
    mx = [max(f32(0), max(e[k] for e, _ in ext)) for k in (1, 3, 5)]
    rt = lambda n: n if n % 32 == 0 else n + 32 - n % 32
    dims = [rt(int(f32(v) / res) + 1) for v in mx]
    vox = -np.ones((dims[2], dims[1], dims[0]), np.int32)
    names = sorted(set(m for _, m in ext))
    for e, m in ext:
        i = [int(f32(v) / res) for v in e]
        vox[i[4]:i[5] + 1, i[2]:i[3] + 1, i[0]:i[1] + 1] = names.index(m)
    return dims, vox, names


def test_kerkythea_loader_matches_restatement(pkg, tmp_path):
    boxes = [((0.0, 1.3, 0.0, 1.02, 0.0, 0.04), "floor_wood"),
             ((-0.2, 0.04, 0.0, 1.02, 0.0, 0.9), "wall_a_concrete"),
             ((0.5, 0.71, 0.3, 0.52, 0.3, 0.61), "desk_wood"),
             ((1.25, 1.3, 0.0, 1.02, 0.0, 0.9), "glass")]
    models = []
    for k, (ext, name) in enumerate(boxes):
        models.append(MODEL.format(name=name, points=box_points(*ext)))
    (tmp_path / "model.xml").write_text(XML.format(models="\n".join(models)))
    coefs = {"wood": ([0.5, 0.1], [1.0, -0.2]), "concrete": ([0.1, 0.02], [1.0, 0.1]),
             "glass": ([0.05, 0.0], [1.0, 0.0])}
    for m, (a, b) in coefs.items():
        (tmp_path / (m + "_a.dat")).write_text("\n".join("%.17g" % v for v in a) + "\n")
        (tmp_path / (m + "_b.dat")).write_text("\n".join("%.17g" % v for v in b) + "\n")
    model = pkg.Model.load_kerkythea(str(tmp_path / "model.xml"), 0.02)
    dims, vox, names = kerkythea_numpy([(e, n[n.rfind("_") + 1:]) for e, n in boxes], 0.02, None)
    (gx, gy, gz), nmat, ncoef = model.dims
    assert [gx, gy, gz] == dims
    assert model.material_names() == names == ["concrete", "glass", "wood"]
    assert ncoef == 2 and nmat == 3
    assert np.array_equal(model.voxels(), vox)
    a, b = model.coefs()
    assert np.array_equal(a, np.array([coefs[n][0] for n in names], np.float32))
    assert np.array_equal(b, np.array([coefs[n][1] for n in names], np.float32))


def test_kerkythea_errors(pkg, tmp_path):
    (tmp_path / "model.xml").write_text(XML.format(models=MODEL.format(name="x_m", points=box_points(
        0, 0.1, 0, 0.1, 0, 0.1))))
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Model.load_kerkythea(str(tmp_path / "model.xml"), 0.02)
    assert ei.value.status == pkg.afd.ERR_IO and "m_a.dat" in str(ei.value)
    (tmp_path / "m_a.dat").write_text("0.5\n0.1\n")
    (tmp_path / "m_b.dat").write_text("1.0\n")
    with pytest.raises(pkg.AfdError):  # filter orders differ between a and b
        pkg.Model.load_kerkythea(str(tmp_path / "model.xml"), 0.02)
    (tmp_path / "bad.xml").write_text("<Root><Object Type='Scene'>")
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Model.load_kerkythea(str(tmp_path / "bad.xml"), 0.02)
    assert ei.value.status == pkg.afd.ERR_IO


# Pinned on the reference's shipped models: grid and boundary counts as a
# separate numpy restatement of kerkythea.hpp and lrs-data.hpp computes them.
SHIPPED = {
    "ie224": ((416, 160, 576), 5, 1, 1056333, 6760, 22),
    "dsp": ((256, 128, 384), 5, 4, 627208, 6656, 29),
    "room_modes": ((160, 128, 256), 1, 1, 260399, 1916, 8),
    "sabine-3x4x5-0.9": ((224, 160, 256), 1, 1, 318786, 2364, 8),
}


@pytest.mark.skipif(not os.path.isdir(REFERENCE_MODELS), reason="reference models not present")
@pytest.mark.parametrize("name", sorted(SHIPPED))
def test_shipped_models(pkg, name):
    dims, nmat, ncoef, faces, edges, corners = SHIPPED[name]
    m = pkg.Model.load_kerkythea(os.path.join(REFERENCE_MODELS, name, "model.xml"), 0.02)
    d, nm, nc = m.dims
    assert d == dims and nm == nmat and nc == ncoef
    c = m.classify()
    assert (c[:6].sum(), c[6:18].sum(), c[18:].sum()) == (faces, edges, corners)


def test_filter_check_host_path(pkg):
    import ancfield_b200.workloads as W
    a, b = W.passive_filters(4, 4, 7)
    st, mr, rt = pkg.check_filters(a, b)
    assert not st.any()
    np.testing.assert_allclose(mr, W.admittance_real_min(a, b), rtol=1e-9)
    roots = [np.abs(np.roots(b[m])).max() for m in range(4)]
    np.testing.assert_allclose(rt, roots, rtol=1e-9)
    b2 = b.copy()
    b2[0] = [1.0, -2.5, 1.2, 0.1]  # a pole outside the unit circle
    a2 = a.copy()
    a2[1] = -a2[1]                 # negative real part: not passive
    st, _, _ = pkg.check_filters(a2, b2)
    assert st[0] & 1 and st[1] & 2


def test_library_exports_the_surrogate_entry_points(pkg):
    """include/afd_surrogate.h: the surrogate network and its GEMM."""
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "afd_surrogate.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(afd_[a-z0-9_]+)\s*\(", text)))
    lib = pkg.afd.library()
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(pkg.surrogate.EXPORTS) == names


def test_surrogate_rejects_untiled_sizes(pkg):
    with pytest.raises(pkg.AfdError) as ei:
        pkg.surrogate.Mlp(hidden=100)
    assert ei.value.status == pkg.afd.ERR_ARG
    assert "multiples of 128" in str(ei.value)


def test_gemm_entry_points_reject_bad_arguments_before_any_launch(pkg):
    """Null pointers and untiled sizes are refused on the host (no device
    work, so this runs without a GPU)."""
    import ctypes as C
    L = pkg.surrogate._lib()
    status = C.c_int32(0)
    assert L.afd_gemm_bf16_async(None, None, None, 128, 128, 64, None, C.byref(status)) == pkg.afd.ERR_ARG
    assert L.afd_gemm_bf16(None, None, None, 128, 128, 64, None) == pkg.afd.ERR_ARG
    buf = (C.c_uint16 * (128 * 64))()
    out = (C.c_float * (128 * 128))()
    st = L.afd_gemm_bf16_async(C.cast(buf, C.c_void_p), C.cast(buf, C.c_void_p), C.cast(out, C.c_void_p),
                               100, 128, 64, None, C.byref(status))
    assert st == pkg.afd.ERR_ARG


def test_device_kerkythea_loader_reports_missing_device_or_bad_file(pkg, tmp_path):
    import torch
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Model.load_kerkythea(str(tmp_path / "missing.xml"), 0.02, device=0)
    assert ei.value.status == pkg.afd.ERR_IO
    if torch.cuda.is_available():
        return
    (tmp_path / "model.xml").write_text(XML.format(models=MODEL.format(name="x_m", points=box_points(
        0, 0.1, 0, 0.1, 0, 0.1))))
    (tmp_path / "m_a.dat").write_text("0.5\n0.1\n")
    (tmp_path / "m_b.dat").write_text("1.0\n0.2\n")
    with pytest.raises(pkg.AfdError) as ei:
        pkg.Model.load_kerkythea(str(tmp_path / "model.xml"), 0.02, device=0)
    assert ei.value.status == pkg.afd.ERR_CUDA


def test_ctypes_structs_match_the_header(pkg, tmp_path):
    """sizeof and every field offset of afd_params, afd_info, afd_plan and
    afd_mlp_params as the C compiler lays them out from include/, against
    the ctypes mirrors."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"afd_params": pkg.afd.Params, "afd_info": pkg.afd.Info, "afd_plan": pkg.afd.Plan,
               "afd_mlp_params": pkg.surrogate.MlpParams}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "afd.h"', '#include "afd_surrogate.h"',
             "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {(a, b): int(c) for a, b, c in (line.split() for line in out if line)}
    for cname, py in structs.items():
        assert got[(cname, "sizeof")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_timeline_slots_match_the_header(pkg):
    text = open(HEADER).read()
    m = re.search(r"#define\s+AFD_TIMELINE_SLOTS\s+(\d+)", text)
    assert m and int(m.group(1)) == len(pkg.Simulation.TIMELINE_KINDS)
