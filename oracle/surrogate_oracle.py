"""CPU FP64 restatement of the surrogate network of
anc-field_b200/csrc/mlp.cu (TEST INFRASTRUCTURE ONLY: the gradient check of
the CUDA forward and backward kernels; the product never calls it).

The network has no counterpart in the reference. Forward: Fourier
features f = [sin(2 pi x B), cos(2 pi x B)], hidden layers
h = relu(a W^T + b), output p = a W^T + b; loss = mean((p - y)^2).

`bf16=True` rounds to bfloat16 (round to nearest even) wherever the GPU
stores a BF16 value: the weights used by the GEMMs, the hidden
activations and the loss and layer gradients. With it the only difference
from the GPU is the FP32 accumulation order inside the GEMMs; without it
this is the plain FP64 network on the same FP32 weights.
"""
import numpy as np


def to_bf16(a):
    """float -> nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    out = (r.astype(np.uint32) << 16).view(np.float32)
    return out.astype(np.float64)


def fourier(x, B):
    ph = 2.0 * np.pi * (np.asarray(x, np.float64) @ np.asarray(B, np.float64))
    return np.concatenate([np.sin(ph), np.cos(ph)], axis=1)


def forward(feat, weights, bf16=True):
    """feat [n, F]; weights [(W [out, in], b [out])]. Returns the layer
    inputs (a_0 = feat, a_l = hidden activations) and the prediction."""
    q = to_bf16 if bf16 else (lambda v: np.asarray(v, np.float64))
    acts = [np.asarray(feat, np.float64)]
    n_l = len(weights)
    for l, (W, b) in enumerate(weights):
        z = acts[-1] @ q(W).T + np.asarray(b, np.float64)
        if l < n_l - 1:
            acts.append(q(np.maximum(z, 0.0)))
        else:
            pred = z
    return acts, pred


def gradients(feat, weights, y, bf16=True):
    """Loss and gradients [(dW, db)] of mean((pred - y)^2) over all elements
    of the n valid rows."""
    q = to_bf16 if bf16 else (lambda v: np.asarray(v, np.float64))
    acts, pred = forward(feat, weights, bf16)
    y = np.asarray(y, np.float64)
    n, n_out = y.shape
    e = pred - y
    loss = float(np.mean(e * e))
    d = q(2.0 * e / (n * n_out))
    grads = [None] * len(weights)
    for l in range(len(weights) - 1, -1, -1):
        W = q(weights[l][0])
        grads[l] = (d.T @ acts[l], d.sum(axis=0))
        if l > 0:
            d = q((d @ W) * (acts[l] > 0))
    return loss, grads
