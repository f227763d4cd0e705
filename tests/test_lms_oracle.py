"""The LMS estimator's CPU restatement (oracle/lms_oracle.py) pinned on the
reference's own EstimateIr (anc_field_py/ancutil.py:24-37): known answers
in tests/golden/lms.npz (made by make_lms.py from the reference tree), and
the block form the GPU evaluates against the sample-serial one."""
import os
import re

import numpy as np
import pytest

import lms_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = ["fir4", "odd", "short_out", "room"]


def case(name):
    g = np.load(os.path.join(HERE, "golden", "lms.npz"))
    N, mu = g[name + "_meta"]
    return g[name + "_x"], g[name + "_y"], int(N), float(mu), g[name + "_w"]


@pytest.mark.parametrize("name", CASES)
def test_restatement_equals_reference_outputs(name):
    x, y, N, mu, w = case(name)
    assert np.array_equal(lms_oracle.estimate(x, y, N, mu), w)


@pytest.mark.parametrize("name", CASES[:3])
@pytest.mark.parametrize("B", [1, 7, 32])
def test_block_form_equals_sample_serial(name, B):
    x, y, N, mu, w = case(name)
    got = lms_oracle.estimate_block(x, y, N, mu, B=B)
    assert np.linalg.norm(got - w) / np.linalg.norm(w) < 1e-13


def test_library_exports_the_lms_entry_points(pkg):
    root = os.path.dirname(HERE)
    text = re.sub(r"/\*.*?\*/", "", open(os.path.join(root, "include", "afd_lms.h")).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(afd_[a-z0-9_]+)\s*\(", text)))
    lib = pkg.afd.library()
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(pkg.lms.EXPORTS) == names


def test_lms_argument_errors(pkg):
    with pytest.raises(pkg.AfdError) as ei:
        pkg.lms.estimate_ir(np.zeros(10), np.zeros(10), 0)
    assert ei.value.status == pkg.afd.ERR_ARG
