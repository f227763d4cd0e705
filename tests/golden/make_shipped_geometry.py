"""Builds tests/golden/shipped_geometry.json from the reference's shipped
Kerkythea models (examples/models/*/model.xml and their filter files).

For every model it stores what a test needs to rebuild an equivalent scene
without the reference tree: per box the model name and the six extreme
coordinate strings of its vertex list in file axes (a_min, a_max, b_min,
b_max, c_min, c_max, as written in the file), and the text of every
<material>_a.dat / _b.dat. A scene written from those (the eight corners of
each box) has the same boxes as the original, so this library's host loader
gives the same voxels; that is checked here before anything is written.

The expected results come from this library's host loader and host
classifier on the ORIGINAL files: grid dims, material names, SHA-256 of the
int32 voxel grid and of the boundary rows (x, y, z, group, mat0..2), and the
per-group counts. The host loader and classifier are pinned separately, by
numpy restatements of kerkythea.hpp and lrs-data.hpp in tests/test_abi.py.

Usage: python tests/golden/make_shipped_geometry.py [reference_root]
"""
import hashlib
import importlib.util
import json
import os
import sys
import tempfile
import xml.etree.ElementTree as ET

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
RES = 0.02


def load_pkg():
    spec = importlib.util.spec_from_file_location("ancfield_b200", os.path.join(ROOT, "anc-field_b200", "__init__.py"),
                                                  submodule_search_locations=[os.path.join(ROOT, "anc-field_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ancfield_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def extract_boxes(path):
    """(model name, [a_min, a_max, b_min, b_max, c_min, c_max] strings) per
    vertex list, the traversal of LoadBoxes (kerkythea.hpp:63-130)."""
    root = ET.parse(path).getroot()
    out = []
    for scene in root.findall("Object"):
        if scene.get("Type") != "Scene":
            continue
        for model in scene.findall("Object"):
            if model.get("Type") != "Model":
                continue
            surf = model.find("Object")
            if surf is None:
                continue
            for prm in surf.findall("Parameter"):
                if prm.get("Name") != "Vertex List":
                    continue
                cols = [[], [], []]
                for p in prm.findall("P"):
                    for k, t in enumerate(p.get("xyz").split()):
                        cols[k].append(t)
                if not cols[0]:
                    continue
                ext = []
                for c in cols:
                    v = np.array([np.float32(float(t)) for t in c])
                    ext += [c[int(np.argmin(v))], c[int(np.argmax(v))]]
                out.append((model.get("Name"), ext))
    return out


def write_scene(d, boxes, dat):
    """The scene of `boxes` (from extract_boxes) and its filter files in d."""
    models = []
    for name, (a0, a1, b0, b1, c0, c1) in boxes:
        pts = "".join('<P xyz="%s %s %s"/>' % (a, b, c) for a in (a0, a1) for b in (b0, b1) for c in (c0, c1))
        models.append('<Object Type="Model" Name="%s"><Object Type="Surface"><Parameter Name="Vertex List">%s'
                      '</Parameter></Object></Object>' % (name, pts))
    with open(os.path.join(d, "model.xml"), "w") as f:
        f.write('<Root><Object Type="Scene">%s</Object></Root>' % "".join(models))
    for fn, text in dat.items():
        with open(os.path.join(d, fn), "w") as f:
            f.write(text)
    return os.path.join(d, "model.xml")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(ref=sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ANC_FIELD_REFERENCE", "/root/reference")):
    pkg = load_pkg()
    mdir = os.path.join(ref, "examples", "models")
    out = {}
    for name in sorted(os.listdir(mdir)):
        path = os.path.join(mdir, name, "model.xml")
        if not os.path.isfile(path):
            continue
        m = pkg.Model.load_kerkythea(path, RES)
        dims, nmat, ncoef = m.dims
        vox = m.voxels()
        rows = m.boundary()
        counts = m.classify()
        boxes = extract_boxes(path)
        mats = sorted(set(n[n.rfind("_") + 1:] for n, _ in boxes))
        dat = {}
        for mt in mats:
            for s in ("_a.dat", "_b.dat"):
                with open(os.path.join(mdir, name, mt + s)) as f:
                    dat[mt + s] = f.read()
        with tempfile.TemporaryDirectory() as d:
            m2 = pkg.Model.load_kerkythea(write_scene(d, boxes, dat), RES)
            assert m2.dims == m.dims and np.array_equal(m2.voxels(), vox), name
            a1, b1 = m.coefs()
            a2, b2 = m2.coefs()
            assert np.array_equal(a1, a2) and np.array_equal(b1, b2), name
        out[name] = {"dims": list(dims), "nmat": nmat, "ncoef": ncoef, "materials": m.material_names(),
                     "voxels_sha256": sha(vox), "boundary_sha256": sha(rows), "n_boundary": int(len(rows)),
                     "counts": [int(c) for c in counts], "boxes": [[n] + e for n, e in boxes], "dat": dat}
        print(name, dims, len(boxes), "boxes", len(rows), "boundary cells")
    with open(os.path.join(HERE, "shipped_geometry.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)


if __name__ == "__main__":
    main()
