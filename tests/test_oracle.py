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
