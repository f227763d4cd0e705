"""CPU restatement of the reference's LMS impulse-response estimator,
EstimateIr (anc_field_py/ancutil.py:24-37) (TEST INFRASTRUCTURE ONLY: the
checker of the GPU estimator in anc-field_b200/csrc/lms.cu).

Algorithm (FP64): weights w (N taps) start at zero; `epochs` passes over
the first min(len(x), len(d)) samples; each pass starts with an empty
delay line u; per sample k: u <- [x_k, u_0 .. u_{N-2}], e = d_k - w.u,
w <- w + (2 mu e) u. The weights carry over from pass to pass.

`estimate` keeps the reference's operations (a shifted delay-line array
and a dot product per sample); `estimate_block` is the block form the GPU
evaluates, restated in numpy: within a block the errors follow from the
weights at the block start, the sliding-window autocorrelations of x and
a triangular recursion, and the block's updates are applied afterwards in
sample order.
"""
import numpy as np


def estimate(x, d, N, mu=1e-4, epochs=16):
    N = int(N)
    w = np.zeros(N)
    steps = min(len(x), len(d))
    for _ in range(epochs):
        u = np.zeros(N)
        for k in range(steps):
            u = np.concatenate((np.array([x[k]]), u[:-1]))
            e = d[k] - np.dot(w, u)
            w = w + 2 * mu * e * u
    return w


def estimate_block(x, d, N, mu=1e-4, epochs=16, B=128):
    N = int(N)
    steps = min(len(x), len(d))
    xs = np.concatenate([np.zeros(N + B), np.asarray(x[:steps], np.float64), np.zeros(2 * B)])
    o = N + B  # xs[o + t] = x_t, zero outside 0 .. steps-1
    w = np.zeros(N)
    for _ in range(epochs):
        r = np.zeros(B)  # r[dl] = sum_j x[m-j] x[m+dl-j] at the last m seen
        for k0 in range(0, steps, B):
            nb = min(B, steps - k0)
            ks = np.arange(k0, k0 + nb)
            # y0_k = sum_j w_j x_{k-j}
            X = xs[o + ks[:, None] - np.arange(N)[None, :]]
            y0 = X @ w
            R = np.zeros((nb, B))
            for dl in range(1, B):
                for i, m in enumerate(ks):
                    r[dl] += xs[o + m] * xs[o + m + dl] - xs[o + m - N] * xs[o + m + dl - N]
                    R[i, dl] = r[dl]
            e = np.zeros(nb)
            for i in range(nb):
                acc = sum(e[p] * R[p, i - p] for p in range(i))
                e[i] = d[k0 + i] - (y0[i] + 2 * mu * acc)
            for i in range(nb):
                w = w + (2 * mu * e[i]) * X[i]
    return w
