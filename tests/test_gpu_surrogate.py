"""The surrogate's hand-written tcgen05 BF16 kernels on the GPU: the GEMM
against the FP64 product of the same BF16 operands, the network's
gradients against the CPU FP64 oracle (oracle/surrogate_oracle.py), and
training on a smooth target.

Tolerances (relative L2 per tensor):
  GEMM vs FP64 product of the BF16 inputs     1e-5 (FP32 accumulation)
  gradients vs oracle rounding as the GPU     1e-3
  gradients vs the plain FP64 network         5e-2 (BF16 activations)
"""
import numpy as np
import pytest

import surrogate_oracle as so

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# M and N multiples of 256 take the CTA-pair kernel (cta_group::2, 256 x 256
# tiles; 4096 x 2048 and 8192 x 2048 give every pair two and three or four
# tiles, so both TMEM accumulators are reused); other M with N a multiple of
# 256 the persistent single-CTA 128 x 256 kernel (128 x 256 x 4096,
# 384 x 1024, 1152 x 512); other N the 128 x 128 kernel.
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 512), (1024, 512, 256), (512, 2048, 1024),
                                   (128, 256, 4096), (4096, 2048, 128), (8192, 2048, 64), (2048, 768, 192),
                                   (384, 1024, 256), (1152, 512, 128)])
def test_gemm_matches_fp32_product(pkg, M, N, K):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    a = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.full((M, N), float("nan"), device="cuda", dtype=torch.float32)
    pkg.surrogate.gemm_bf16(a, b, c, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = a.double() @ b.double().T
    assert torch.isfinite(c).all()
    assert rel(c.cpu().numpy(), want.cpu().numpy()) < 1e-5


def test_gemm_async_in_a_cuda_graph(pkg):
    """The unsynchronised form queued inside stream capture and replayed."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(9)
    a = torch.randn(512, 256, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(512, 256, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.zeros(512, 512, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    pkg.surrogate.gemm_bf16(a, b, c, torch.cuda.current_stream().cuda_stream)  # attributes set outside capture
    c.zero_()
    graph = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        with torch.cuda.graph(graph, stream=s):
            pkg.surrogate.gemm_bf16_async(a, b, c, status, s.cuda_stream)
    graph.replay()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    want = a.double() @ b.double().T
    assert rel(c.cpu().numpy(), want.cpu().numpy()) < 1e-5


def small_mlp(pkg, seed=3, **kw):
    p = dict(n_in=10, n_freq=64, hidden=128, n_layers=3, n_out=128, batch=128, seed=seed, fourier_sigma=1.5)
    p.update(kw)
    return pkg.surrogate.Mlp(**p)


# wide: 256 features, 256 hidden units and outputs, so the GEMMs of the
# forward and backward passes (bias + ReLU, ReLU mask, FP32) run in the
# 128 x 256 kernels (weight gradients, M = 256: the CTA-pair kernel; the
# others, M = 128 rows: the single-CTA one); otherwise all run in the
# 128 x 128 kernel.
@pytest.mark.parametrize("n,wide", [(128, False), (77, False), (77, True)])
def test_gradients_match_cpu_oracle(pkg, n, wide):
    S = pkg.surrogate
    m = small_mlp(pkg, **(dict(n_freq=128, hidden=256, n_out=256) if wide else {}))
    n_out = 256 if wide else 128
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, (n, 10)).astype(np.float32)
    y = (0.3 * rng.standard_normal((n, n_out))).astype(np.float32)
    loss = m.gradients(x, y)
    feat = m.get(S.FEATURES)[:n]
    W = m.weights()
    # the features are the Fourier map of x rounded to BF16
    f64 = so.fourier(x, m.get(S.FOURIER))
    assert np.abs(feat - so.to_bf16(f64)).max() <= 2.0 ** -8
    want_loss, want = so.gradients(feat, W, y, bf16=True)
    _, plain = so.gradients(feat, W, y, bf16=False)
    assert abs(loss - want_loss) / want_loss < 1e-5
    for l in range(3):
        gw, gb = m.get(S.GRAD_WEIGHT, l), m.get(S.GRAD_BIAS, l)
        assert rel(gw, want[l][0]) < 1e-3, (l, rel(gw, want[l][0]))
        assert rel(gb, want[l][1]) < 1e-3, (l, rel(gb, want[l][1]))
        assert rel(gw, plain[l][0]) < 5e-2
        assert rel(gb, plain[l][1]) < 5e-2
    m.close()


def test_predict_matches_cpu_forward(pkg):
    S = pkg.surrogate
    m = small_mlp(pkg, seed=4)
    x = np.random.default_rng(6).uniform(0, 1, (100, 10)).astype(np.float32)
    out = m.predict(x)
    feat = m.get(S.FEATURES)[:100]
    _, want = so.forward(feat, m.weights(), bf16=True)
    assert rel(out, want) < 1e-4
    m.close()


def test_training_fits_a_smooth_target(pkg):
    """Adam on the GPU kernels: a smooth map from 10 inputs to 128 outputs
    is learned to well below its variance."""
    m = small_mlp(pkg, seed=7, lr=2e-3)
    rng = np.random.default_rng(8)
    x = rng.uniform(0, 1, (4096, 10)).astype(np.float32)
    t = np.linspace(0, 1, 128)
    y = (np.sin(2 * np.pi * (x[:, :1] * 2 + t[None, :] * (1 + x[:, 1:2]))) * (0.5 + x[:, 2:3])).astype(np.float32)
    first = None
    for it in range(1500):
        idx = rng.integers(0, 4096, 128)
        loss = m.train_step(x[idx], y[idx])
        first = loss if first is None else first
    pred = m.predict(x[:128])
    err = rel(pred, y[:128])
    print("loss %.4g -> %.4g, relative L2 %.3g" % (first, loss, err))
    # measured: loss 1.45 -> 0.06, relative L2 0.30 after 1500 steps
    assert loss < 0.1 * first
    assert err < 0.45
    m.close()


def test_split_gemm_reaches_fp32_accuracy(pkg):
    """The readout's normal equations use the tcgen05 GEMM on BF16 value and
    remainder parts: the three-product sum matches the FP64 product of the
    FP32 operands to FP32-level accuracy (one BF16 product alone is ~1e-3)."""
    import torch
    import ancfield_b200.surrogate_workflow as SW
    g = torch.Generator(device="cpu").manual_seed(3)
    a = torch.randn(300, 700, generator=g).cuda()
    b = torch.randn(260, 700, generator=g).cuda()
    c = SW.gemm_split(pkg, a, b)
    want = a.double() @ b.double().t()
    err = float((c.double() - want).norm() / want.norm())
    assert c.shape == (300, 260)
    assert err < 1e-5, err


def test_field_readout_gain_over_fdtd(pkg):
    """The learned readout (random Fourier features of the receiver position
    and the source's 1/R near-field features, output layer fitted through
    the normal equations on the tcgen05 GEMM) against the FDTD at receiver
    positions the generating run did not train on: the fraction of pairs
    within 1 % relative L2, the IRs/s with FDTD fallback for the pairs whose
    predicted error exceeds 1 %, and the gain over the FDTD alone. Where the
    query pairs arrive one at a time after the runs, the FDTD pays one
    source's share of a batched run per pair and the readout only for its
    rejected pairs; where every position is known before the runs, one
    batched FDTD run answers them all and the readout with its fallback runs
    cannot beat it (that gain is printed, and bounded below only)."""
    import ancfield_b200.surrogate_workflow as SW
    r = SW.run_field_readout(pkg, n_sets=1, n_src=4, n_query=64, n_val=64, plain=False)
    print({k: r[k] for k in ("query_rel_l2", "within_bound", "accepted", "accepted_but_over_bound",
                             "fallback_runs", "irs_per_s", "gain_over_fdtd", "queries_after_runs")})
    assert r["within_bound"] >= 0.6
    # accepted pairs whose true error exceeds the bound: at most 3 %
    assert r["accepted_but_over_bound"] <= 0.03 * r["query_pairs"]
    assert r["queries_after_runs"]["gain_over_fdtd"] > 1.5
    assert r["gain_over_fdtd"] > 0.9
