"""The anc-field executable: the command loop, argument checks, error lines
and progress protocol of anc-field/src/main.cpp and commandline.hpp, as
anc_field_py/ancfield.py drives them (prompt '>> ', 'BEGIN', 'i/steps')."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "anc-field_b200", "bin", "anc-field")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def session(lines, timeout=120, cwd=None):
    r = subprocess.run([EXE], input="\n".join(lines) + "\n", capture_output=True, text=True, timeout=timeout,
                       cwd=cwd)
    return r.returncode, r.stdout, r.stderr


def replies(out):
    """Text printed after each prompt."""
    return [p.strip() for p in out.split(">> ")[1:]]


def test_prompt_and_quit():
    rc, out, _ = session(["quit"])
    assert rc == 0 and out == ">> "


def test_end_of_input_ends_the_loop():
    r = subprocess.run([EXE], input="", capture_output=True, text=True, timeout=20)
    assert r.returncode == 0 and r.stdout == ">> "


def test_error_lines():
    rc, out, _ = session(["frobnicate", "load", "run abc", "load /no/such/file.xml", "sdt tpu",
                          "minsize [1,x,3]", "pml 1.5", "addmic [1,2,3]", "", "precision fp8", "quit"])
    r = replies(out)
    assert r[0] == "Error: unrecognized command"
    assert r[1] == "Error: command load takes 1 argument(s)"
    assert r[2] == "Error: argument[0] should be a(n) float"
    assert r[3] == "Error: file /no/such/file.xml doesn't exist"
    assert r[4] == "Valid command arguments are 'cpu' or 'gpu'"
    assert r[5] == "Error: argument[0] should be a(n) float_list"
    assert r[6] == "Error: argument[0] should be a(n) int"
    assert r[7].startswith("Error: no active simulation")
    assert r[8] == ""  # empty line: prompt again
    assert r[9] == "Valid command arguments are 'fp32' or 'fp16'"


def test_cd_and_lsd_without_device():
    if has_gpu():
        pytest.skip("a CUDA device is present")
    rc, out, _ = session(["lsd", "cd", "sdt gpu", "quit"])
    r = replies(out)
    assert r[0] == "Available compute devices"
    assert r[1] == "Compute devices removed"
    assert r[2] == "Error: no CUDA device available"


def write_model(tmp):
    """A 1.0 x 0.8 x 0.7 m room (grid 64 x 64 x 64 at 2 cm) with a desk."""
    def pts(x0, x1, y0, y1, z0, z1):
        out = []
        for x in (x0, x1):
            for y in (y0, y1):
                for z in (z0, z1):
                    out.append('<P xyz="%r %r %r"/>' % (x, -z, y))
        return "".join(out)
    boxes = [("floor_wood", (0, 1.0, 0, 0.8, 0, 0.02)), ("ceil_wood", (0, 1.0, 0, 0.8, 0.68, 0.7)),
             ("w1_plaster", (0, 0.02, 0, 0.8, 0, 0.7)), ("w2_plaster", (0.98, 1.0, 0, 0.8, 0, 0.7)),
             ("w3_plaster", (0, 1.0, 0, 0.02, 0, 0.7)), ("w4_plaster", (0, 1.0, 0.78, 0.8, 0, 0.7)),
             ("desk_wood", (0.3, 0.5, 0.2, 0.4, 0.02, 0.3))]
    models = "".join('<Object Type="Model" Name="%s"><Object Type="Surface"><Parameter Name="Vertex List">%s'
                     '</Parameter></Object></Object>' % (n, pts(*e)) for n, e in boxes)
    (tmp / "model.xml").write_text('<Root><Object Type="Scene">%s</Object></Root>' % models)
    (tmp / "wood_a.dat").write_text("0.2\n0.05\n")
    (tmp / "wood_b.dat").write_text("1.0\n-0.3\n")
    (tmp / "plaster_a.dat").write_text("0.08\n0.01\n")
    (tmp / "plaster_b.dat").write_text("1.0\n0.2\n")
    sig = np.zeros(400)
    sig[1:40] = np.hanning(39)
    np.savetxt(tmp / "src.dat", sig)
    return sig.astype(np.float32)


@pytest.mark.gpu
def test_full_session_matches_oracle(pkg, tmp_path):
    sig = write_model(tmp_path)
    mics = ["[0.7,0.5,0.4]", "[0.25,0.25,0.5]", "[0.9,0.1,0.1]"]
    lines = ["sdt gpu", "load %s" % (tmp_path / "model.xml"), "addsource [0.3,0.6,0.35] %s" % (tmp_path / "src.dat")]
    lines += ["addmic %s" % m for m in mics]
    lines += ["vis 0.4", "run 0.0125", "save %s" % (tmp_path / "out.dat"), "visdump %s" % (tmp_path / "vis.npy"),
              "quit"]
    rc, out, err = session(lines, timeout=300)
    assert rc == 0, err
    assert "added to active devices" in out
    # progress protocol of simulation.hpp:403-409, 433 for 400 steps
    prog = re.findall(r"(BEGIN|\d+/\d+)", out)
    assert prog == ["BEGIN", "0/400", "200/400", "400/400"]
    text = (tmp_path / "out.dat").read_text()
    assert text.endswith("\n\n")
    rows = [r for r in text.split("\n") if r]
    assert all(r.endswith(" ") for r in rows)
    got = np.array([[float(v) for v in r.split()] for r in rows])
    # the same run through the oracle (REF semantics, reference constants)
    m = pkg.Model.load_kerkythea(str(tmp_path / "model.xml"), 0.02)
    a, b = m.coefs()
    cell = lambda p: tuple(int(np.float32(v) / np.float32(0.02)) for v in p)
    want, field = oracle.simulate(grid=m.dims[0], vox=m.voxels(), a=a, b=b, mode=0,
                                  sources=[(cell((0.3, 0.6, 0.35)), sig)],
                                  receivers=[cell(eval(s)) for s in mics], steps=400, want_field=True)
    # vis 0.4: the plane y = 20 after every third step (134 of 400), the newest
    # 64 kept on the device and dumped as .npy; the last is the final field's
    frames = np.load(tmp_path / "vis.npy")
    nx, ny, nz = m.dims[0]
    assert frames.shape == (64, nz, nx) and frames.dtype == np.float32
    assert np.array_equal(frames[-1], field[:, int(np.float32(0.4) / np.float32(0.02)), :])
    # the file holds ostream's 6 significant digits
    fmt = np.vectorize(lambda v: float("%.6g" % v))
    assert np.array_equal(got, fmt(want.astype(np.float64)))
