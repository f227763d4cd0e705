"""The CPU oracle restatement (oracle/afd_oracle.c) pinned against the
reference's own kernel sources (oracle/ref_harness.c -> oracle/_ref), through
the committed golden fixtures and, when the reference build is present, live.
"""
import json
import os
import sys

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import CASES, build_case  # noqa: E402


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_restatement_matches_reference_golden(name, prec):
    """Bit-exact: same expression order, no contraction (-ffp-contract=off)."""
    gold = np.load(os.path.join(HERE, "golden", "golden_%s.npz" % name))
    rcv, field = oracle.simulate(impl="ora", precision=prec, want_field=True, **build_case(CASES[name]))
    assert np.array_equal(rcv, gold["rcv_" + prec])
    assert np.array_equal(field, gold["field_" + prec])


def test_cases_json_matches_generator():
    with open(os.path.join(HERE, "golden", "cases.json")) as f:
        assert json.load(f) == CASES


@pytest.mark.skipif(not oracle.available("ref", "f32"), reason="reference kernels not built here")
@pytest.mark.parametrize("seed", [21, 22, 23])
def test_restatement_matches_reference_live(seed):
    rng = np.random.default_rng(seed)
    spec = {"grid": [int(v) for v in rng.integers(16, 30, 3)], "K": int(rng.integers(1, 5)), "seed": seed,
            "steps": 90, "pml": int(rng.integers(0, 2)) * 4, "runs": [90]}
    inp = build_case(spec)
    for prec in ("f32", "f64"):
        r1, f1 = oracle.simulate(impl="ora", precision=prec, want_field=True, **inp)
        r2, f2 = oracle.simulate(impl="ref", precision=prec, want_field=True, **inp)
        assert np.array_equal(r1, r2) and np.array_equal(f1, f2)


def test_fp32_error_against_fp64_is_small():
    """Every FP32 result states its error against the FP64 run of the same
    scheme; on these cases it stays far below the 1e-5 bar."""
    for name in ("k2", "k4", "k2_pml"):
        gold = np.load(os.path.join(HERE, "golden", "golden_%s.npz" % name))
        r32, r64 = gold["rcv_f32"].astype(np.float64), gold["rcv_f64"].astype(np.float64)
        err = np.linalg.norm(r32 - r64) / np.linalg.norm(r64)
        assert err < 1e-5, (name, err)


def test_fixed_mode_differs_from_ref_only_where_quirks_act():
    """FIXED removes the reference quirks: with K = 1, no PML and no corner
    cells the two schemes still differ because REF uses lambda^2 as the
    boundary Courant number; without any boundary cell they agree."""
    inp = build_case(CASES["k1"])
    inp.pop("mode")
    rr, _ = oracle.simulate(mode=0, **inp)
    rf, _ = oracle.simulate(mode=1, **inp)
    assert not np.array_equal(rr, rf)
    box = dict(inp)
    box.update(vox=None, a=None, b=None)
    rr, fr = oracle.simulate(mode=0, want_field=True, **box)
    rf, ff = oracle.simulate(mode=1, want_field=True, **box)
    assert np.array_equal(rr, rf) and np.array_equal(fr, ff)


def test_source_on_a_boundary_cell_persists_like_the_reference():
    """Outer cells are never updated: with three rotating levels a source
    there adds onto the value the level held three steps earlier."""
    inp = dict(grid=(12, 10, 9), sources=[((0, 4, 4), np.ones(9, np.float32))], receivers=[(0, 4, 4)],
               steps=9)
    rcv, _ = oracle.simulate(**inp)
    assert np.array_equal(rcv[0], np.array([1, 1, 1, 2, 2, 2, 3, 3, 3], np.float32))
    if oracle.available("ref", "f32"):
        r2, _ = oracle.simulate(impl="ref", **inp)
        assert np.array_equal(rcv, r2)


# ---------------------------------------------------------------- FP16 storage
def _f16_lib():
    import ctypes as C
    lib = C.CDLL(oracle.ORA_LIB)
    P = C.POINTER
    lib.ora_f16_round.argtypes = [P(C.c_float), P(C.c_float), C.c_int64, C.c_float]
    lib.ora_level_scale.argtypes = [P(C.c_float), P(C.c_float), C.c_int64, C.c_float]
    return lib, C


def test_f16_storage_rounding_matches_numpy():
    """The restatement's binary16 round trip (round to nearest even, own
    bit arithmetic) equals numpy's float32 -> float16 -> float32 on random
    bit patterns, the overflow and subnormal edges, and with scales."""
    lib, C = _f16_lib()
    rng = np.random.default_rng(0)
    x = rng.integers(0, 2**32, 1_000_000, dtype=np.uint64).astype(np.uint32).view(np.float32)
    x = x[np.isfinite(x)]
    edge = np.array([0.0, -0.0, 65504, 65519.99, 65520, 65536, 2**-14, 2**-24, 2**-25, 3 * 2**-26, -1e-8],
                    np.float32)
    x = np.concatenate([x, edge, np.arange(-70000, 70000, 0.37, dtype=np.float32)])
    for s in (1.0, 2.0**-20, 2.0**13, 2.0**40):
        out = np.empty_like(x)
        lib.ora_f16_round(x.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(C.POINTER(C.c_float)),
                          x.size, s)
        with np.errstate(over="ignore"):
            want = (x * np.float32(s)).astype(np.float16).astype(np.float32) * np.float32(1.0 / s)
        same = (out == want) | (np.isnan(out) & np.isnan(want))
        assert same.all(), (s, x[~same][:5])


def test_level_scale_rule():
    """2^(10 - e) with max(m, smax) < 2^e, clamped exponents, 1 for zero."""
    import math
    lib, C = _f16_lib()
    m = np.array([0.0, 1.0, 0.75, 1024.0, 1e-30, 3e38, 2.0**-130, 5.0, 6e-5], np.float32)
    for smax in (0.0, 0.5, 100.0):
        out = np.empty_like(m)
        lib.ora_level_scale(m.ctypes.data_as(C.POINTER(C.c_float)), out.ctypes.data_as(C.POINTER(C.c_float)),
                            m.size, smax)
        for v, s in zip(m, out):
            a = max(float(v), smax)
            if a == 0.0:
                assert s == 1.0
                continue
            e = math.frexp(a)[1]
            assert s == 2.0 ** max(-60, min(60, 10 - e))
            assert a * s < 2.0 ** 10 or 10 - e < -60


def test_fp16_storage_restatement_error():
    """FP16 storage of the FIXED scheme on a small room with PML: within
    -40 dB of the FP64 scheme, and FP32 within -80 dB."""
    sys.path.insert(0, os.path.join(HERE, ".."))
    import __graft_entry__ as ge
    W = ge.load().workloads
    rng = np.random.default_rng(3)
    vox = W.room(40, 34, 30, 63 & ~W.FACE_ZP, n_boxes=1, nmat=2, seed=4, box_min=4, box_max=8)
    a, b = W.passive_filters(2, 2, 5)
    ksi = W.ksi_arrays((40, 34, 30), 8, W.FACE_ZP)
    sig = W.gaussian_pulse(600, 24000.0)
    kw = dict(grid=(40, 34, 30), vox=vox, a=a, b=b, dx=0.025, c=343.0, dt=W.courant_dt(0.025, 343.0), mode=1,
              pml_width=8, faces=W.FACE_ZP, ksi=ksi, sources=[((12, 14, 10), sig)],
              receivers=[tuple(int(v) for v in rng.integers(5, 25, 3)) for _ in range(4)], steps=600)
    r64, _ = oracle.simulate(precision="f64", **kw)
    r32, _ = oracle.simulate(precision="f32", **kw)
    r16, _ = oracle.simulate(precision="f16", **kw)
    db = lambda x: 20 * np.log10(np.linalg.norm(x - r64) / np.linalg.norm(r64))
    assert db(r16.astype(np.float64)) <= -40.0
    assert db(r32.astype(np.float64)) <= -80.0
    assert not np.array_equal(r16, r32)
