"""The CPU FP64 oracle of the surrogate network (oracle/surrogate_oracle.py)
checked on its own: analytic gradients against central differences, and
its bfloat16 rounding against torch's."""
import numpy as np
import pytest

import surrogate_oracle as so


def small_net(seed, dims=(8, 6, 6, 4)):
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal((dims[l + 1], dims[l])) * 0.7, rng.standard_normal(dims[l + 1]) * 0.1)
            for l in range(len(dims) - 1)]


@pytest.mark.parametrize("seed", [0, 1])
def test_fp64_gradients_match_finite_differences(seed):
    rng = np.random.default_rng(100 + seed)
    W = small_net(seed)
    feat = rng.standard_normal((5, 8))
    y = rng.standard_normal((5, 4))
    loss, grads = so.gradients(feat, W, y, bf16=False)
    h = 1e-6
    for l, (w, b) in enumerate(W):
        for arr, g in ((w, grads[l][0]), (b, grads[l][1])):
            num = np.zeros_like(arr)
            it = np.nditer(arr, flags=["multi_index"])
            for _ in it:
                i = it.multi_index
                old = arr[i]
                arr[i] = old + h
                lp, _ = so.gradients(feat, W, y, bf16=False)
                arr[i] = old - h
                lm, _ = so.gradients(feat, W, y, bf16=False)
                arr[i] = old
                num[i] = (lp - lm) / (2 * h)
            assert np.allclose(g, num, rtol=1e-5, atol=1e-8)
    assert loss > 0


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(100000).astype(np.float32) * 10.0 ** rng.integers(-30, 30, 100000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38, 1e-40], np.float32)])
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    got = so.to_bf16(x)
    assert np.array_equal(got, want)
