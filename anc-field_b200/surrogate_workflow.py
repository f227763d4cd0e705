"""Secondary-path impulse responses: the batched FDTD that generates them,
the plain single-source FDTD path they are compared with, and the learned
surrogate with its error model and FDTD fallback. No counterpart in the
reference (its IR identification is an offline LMS fit, ie224-impulse.py).

Room: 4 x 3 x 2.5 m at dx = 2.5 cm (160 x 120 x 100 cells), c = 343 m/s,
Courant 0.99/sqrt(3) (fs = 24.0 kHz), FIXED scheme, a one-cell solid shell
with four wall materials (floor, ceiling, x walls, y walls), each a
first-order passive admittance filter a = [g, -g/2], b = [1, 0] whose gain
g in [0.05, 0.5] is one of the four wall parameters. A source is a Ricker
wavelet (zero DC, band-limited around F0); the IR is the receiver signal
decimated by 3 (8.0 kHz, alias-free because the source is band-limited),
2048 samples (6144 steps).

Surrogate input (10 values in [0, 1]): source xyz / room size, receiver
xyz / room size, (g - 0.05) / 0.45 for the four walls. Output: the IR
divided by a global scale (the RMS of the training IRs).
"""
import math
import time

import numpy as np

ROOM = (160, 120, 100)
DX, C = 0.025, 343.0
DECIM = 3
IR_LEN = 2048
G_LO, G_HI = 0.05, 0.5
MARGIN = 10  # cells between a source/receiver and the wall
F0 = 80.0    # Hz, peak frequency of the source wavelet (energy below about 250 Hz)


def dt():
    return 0.99 / math.sqrt(3.0) * DX / C


def steps():
    return IR_LEN * DECIM


def room_voxels():
    nx, ny, nz = ROOM
    vox = -np.ones((nz, ny, nx), np.int32)
    vox[:, :, 0] = vox[:, :, -1] = 2   # x walls
    vox[:, 0, :] = vox[:, -1, :] = 3   # y walls
    vox[0, :, :] = 0                   # floor
    vox[-1, :, :] = 1                  # ceiling
    return vox


def wall_filters(g):
    g = np.asarray(g, np.float64)
    a = np.stack([g, -0.5 * g], axis=1)
    b = np.tile([1.0, 0.0], (len(g), 1))
    return a.astype(np.float32), b.astype(np.float32)


def source_signal(n, f0=None):
    """Ricker wavelet (second derivative of a Gaussian) with peak frequency
    f0 at fs = 1/dt, centred at 1.5/f0 and zero-padded to n samples: zero
    DC, spectrum f^2 exp(-f^2/f0^2), i.e. a band-limited loudspeaker drive
    in the active-noise-control band (below about 3 f0)."""
    f0 = F0 if f0 is None else f0
    t = np.arange(n) * dt() - 1.5 / f0
    a = (np.pi * f0 * t) ** 2
    w = (1.0 - 2.0 * a) * np.exp(-a)
    w[np.abs(t) > 3.0 / f0] = 0.0
    return w.astype(np.float32)


def random_cells(rng, n):
    nx, ny, nz = ROOM
    lo = MARGIN
    return np.stack([rng.integers(lo, nx - lo, n), rng.integers(lo, ny - lo, n), rng.integers(lo, nz - lo, n)],
                    axis=1).astype(np.int32)


def features(src, rcv, g):
    """Surrogate inputs for pairs: src, rcv [n, 3] cells, g [n, 4]."""
    size = np.asarray(ROOM, np.float32)
    return np.concatenate([(np.asarray(src, np.float32) + 0.5) / size, (np.asarray(rcv, np.float32) + 0.5) / size,
                           (np.asarray(g, np.float32) - G_LO) / (G_HI - G_LO)], axis=1).astype(np.float32)


def make_sim(pkg, g, batch, graphs=1, storage=0):
    a, b = wall_filters(g)
    sim = pkg.Simulation(mode=1, dx=DX, c=C, dt=dt(), batch=batch, graphs=graphs, storage=storage)
    sim.SetModel(pkg.Model.from_voxels(room_voxels(), a, b))
    return sim


def batched_irs(pkg, g, src_cells, rcv_cells, storage=0):
    """One batched launch sequence: every source in its own batch member,
    all receivers shared. Returns IRs [n_src, n_rcv, IR_LEN] and the wall
    time of the run (seconds, setup excluded)."""
    n_src = len(src_cells)
    sim = make_sim(pkg, g, n_src, storage=storage)
    sig = source_signal(steps())
    for m, s in enumerate(src_cells):
        sim.AddSourceCell(tuple(int(v) for v in s), sig, batch=m)
    for r in rcv_cells:
        sim.AddMicCell(tuple(int(v) for v in r))
    sim.prepare(steps())
    t = time.perf_counter()
    sim.Run(steps())
    out = np.stack([sim.mics(batch=m)[:, ::DECIM][:, :IR_LEN] for m in range(n_src)])
    wall = time.perf_counter() - t
    sim.close()
    return out, wall


def plain_irs(pkg, g, src_cell, rcv_cells):
    """The plain single-source FP32 path: one source per run, per-step
    kernel launches, no CUDA graph, no batching. Returns IRs [n_rcv,
    IR_LEN] and the wall time of the run (seconds, setup excluded)."""
    sim = make_sim(pkg, g, 1, graphs=0)
    sim.AddSourceCell(tuple(int(v) for v in src_cell), source_signal(steps()))
    for r in rcv_cells:
        sim.AddMicCell(tuple(int(v) for v in r))
    sim.prepare(steps())
    t = time.perf_counter()
    sim.Run(steps())
    out = sim.mics()[:, ::DECIM][:, :IR_LEN]
    wall = time.perf_counter() - t
    sim.close()
    return out, wall


def generate(pkg, n_sets, n_src, n_rcv, seed):
    """(parameter set) x (batched sources) x (receivers): n_sets * n_src *
    n_rcv pairs. Returns x [N, 10], irs [N, IR_LEN], FDTD seconds."""
    rng = np.random.default_rng(seed)
    xs, ys, total = [], [], 0.0
    for _ in range(n_sets):
        g = rng.uniform(G_LO, G_HI, 4)
        src = random_cells(rng, n_src)
        rcv = random_cells(rng, n_rcv)
        irs, wall = batched_irs(pkg, g, src, rcv)
        total += wall
        si, ri = np.meshgrid(np.arange(n_src), np.arange(n_rcv), indexing="ij")
        xs.append(features(src[si.ravel()], rcv[ri.ravel()], np.tile(g, (si.size, 1))))
        ys.append(irs.reshape(-1, IR_LEN))
    return np.concatenate(xs), np.concatenate(ys).astype(np.float32), total


def rel_err(pred, ref):
    return np.linalg.norm(pred - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)


class Surrogate:
    """The IR network and its error model (a second network of the same
    kernels that predicts log10 of the IR network's relative L2 error)."""

    def __init__(self, pkg, seed=1, steps_ir=6000, steps_err=3000, batch=1024, lr=1e-3, sigma=1.0, n_in=10):
        self.pkg = pkg
        S = pkg.surrogate
        self.net = S.Mlp(batch=batch, seed=seed, lr=lr, fourier_sigma=sigma, n_in=n_in)
        self.errnet = S.Mlp(batch=batch, seed=seed + 1, n_out=128, n_layers=4, hidden=256, lr=lr, n_in=n_in)
        self.steps_ir, self.steps_err, self.batch = steps_ir, steps_err, batch
        self.scale = 1.0

    def fit(self, x, y, calib_frac=0.1, seed=0):
        """Trains the IR network on part of (x, y) and the error model on
        the network's errors over the held-back rest."""
        import torch
        rng = np.random.default_rng(seed)
        n = len(x)
        perm = rng.permutation(n)
        n_cal = max(self.batch // 4, int(calib_frac * n))
        cal, tr = perm[:n_cal], perm[n_cal:]
        self.scale = float(np.sqrt(np.mean(y[tr] ** 2)))
        xd = torch.from_numpy(x).cuda()
        yd = torch.from_numpy(y / self.scale).cuda()
        trd = torch.from_numpy(tr).cuda()
        losses = []
        for it in range(self.steps_ir):
            idx = trd[torch.randint(0, len(tr), (self.batch,), device="cuda")]
            want = it % 500 == 0 or it == self.steps_ir - 1
            loss = self.net.train_step(xd[idx].contiguous(), yd[idx].contiguous(), want_loss=want)
            if want:
                losses.append((it, loss))
        self.net.sync()
        train_err = float(np.median(rel_err(self.predict(x[tr[:2048]]), y[tr[:2048]])))
        # error model on the held-back calibration rows
        pred = self.predict(x[cal])
        e = np.log10(np.maximum(rel_err(pred, y[cal]), 1e-6)).astype(np.float32)
        t_err = np.zeros((len(cal), 128), np.float32)
        t_err[:, 0] = e
        xe = torch.from_numpy(x[cal]).cuda()
        ye = torch.from_numpy(t_err).cuda()
        for it in range(self.steps_err):
            idx = torch.randint(0, len(cal), (self.batch,), device="cuda")
            self.errnet.train_step(xe[idx].contiguous(), ye[idx].contiguous(), want_loss=False)
        self.errnet.sync()
        return {"train_pairs": int(len(tr)), "calibration_pairs": int(n_cal), "loss_curve": losses,
                "train_median_rel_l2": train_err}

    def predict(self, x):
        out = []
        for i in range(0, len(x), self.batch):
            out.append(self.net.predict(x[i:i + self.batch]))
        return np.concatenate(out) * self.scale

    def predicted_error(self, x):
        out = []
        for i in range(0, len(x), self.batch):
            out.append(self.errnet.predict(x[i:i + self.batch])[:, 0])
        return 10.0 ** np.concatenate(out)


def nearest_neighbour(x_train, y_train, x_query):
    """Baseline without a network: the IR of the closest training input."""
    import torch
    d = torch.cdist(torch.from_numpy(x_query).cuda(), torch.from_numpy(x_train).cuda())
    return y_train[d.argmin(dim=1).cpu().numpy()]


def run_c5(pkg, n_sets=40, n_src=32, n_rcv=16, test_sets=4, test_src=16, test_rcv=16, steps_ir=8000, bound=0.01,
           seed=11, surrogate_kw=None, featurize=None):
    """Generates the training pairs with the batched FDTD, trains the IR
    network and its error model, and evaluates held-out pairs (new wall
    parameters and positions) against their FDTD IRs: errors, baselines,
    the fallback decision at `bound`, and IRs/s of each path."""
    import torch
    featurize = featurize or (lambda v: v)
    t0 = time.perf_counter()
    x, y, fd_train = generate(pkg, n_sets, n_src, n_rcv, seed)
    t_gen = time.perf_counter() - t0
    xt, yt, fd_test = generate(pkg, test_sets, test_src, test_rcv, seed + 1000)
    xf, xtf = featurize(x), featurize(xt)
    sur = Surrogate(pkg, steps_ir=steps_ir, n_in=xf.shape[1], **(surrogate_kw or {}))
    t0 = time.perf_counter()
    info = sur.fit(xf, y)
    t_fit = time.perf_counter() - t0
    sur.predict(xtf[:16])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pred = sur.predict(xtf)
    pe = sur.predicted_error(xtf)
    t_pred = time.perf_counter() - t0
    e = rel_err(pred, yt)
    e_mean = rel_err(np.tile(y.mean(axis=0), (len(yt), 1)), yt)
    e_nn = rel_err(nearest_neighbour(x, y, xt), yt)
    # fallback: every (wall set, source) with a pair whose predicted error
    # exceeds the bound needs one FDTD run (its receivers come with it)
    fb = (pe > bound).reshape(test_sets, test_src, test_rcv)
    runs_needed = int(fb.any(axis=2).sum())
    run_s = fd_test / (test_sets * test_src)  # batched seconds per source
    t_fallback = runs_needed * run_s
    rng = np.random.default_rng(seed + 2000)
    g = rng.uniform(G_LO, G_HI, 4)
    _, t_plain = plain_irs(pkg, g, random_cells(rng, 1)[0], random_cells(rng, test_rcv))
    n = len(xt)
    return {
        "train_pairs": int(len(x)), "train_fdtd_s": fd_train, "train_generation_wall_s": t_gen,
        "fit_s": t_fit, "fit": info,
        "held_out_pairs": n, "held_out_rel_l2": {"median": float(np.median(e)), "p10": float(np.percentile(e, 10)),
                                                 "p90": float(np.percentile(e, 90))},
        "baselines_median_rel_l2": {"zero": 1.0, "mean_ir": float(np.median(e_mean)),
                                    "nearest_neighbour": float(np.median(e_nn))},
        "within_bound": int((e <= bound).sum()), "accepted": int((pe <= bound).sum()),
        "accepted_and_within": int(((pe <= bound) & (e <= bound)).sum()),
        "error_model_log_corr": float(np.corrcoef(np.log10(pe), np.log10(e))[0, 1]),
        "irs_per_s": {"surrogate_only": n / t_pred, "surrogate_with_fallback": n / (t_pred + t_fallback),
                      "batched_fdtd": n / fd_test, "plain_fdtd": test_rcv / t_plain},
        "bound": bound,
    }


def geometric_inputs(x):
    """The 10 surrogate inputs plus seven path lengths that follow from
    them: source-receiver distance and the distances from the receiver to
    the six first-order image sources of the shoebox, divided by the room
    diagonal."""
    size = np.asarray(ROOM, np.float64) * DX
    s = x[:, 0:3].astype(np.float64) * size
    r = x[:, 3:6].astype(np.float64) * size
    diag = float(np.linalg.norm(size))
    d = [np.linalg.norm(s - r, axis=1)]
    for ax in range(3):
        for wall in (0.0, size[ax]):
            img = s.copy()
            img[:, ax] = 2 * wall - s[:, ax]
            d.append(np.linalg.norm(img - r, axis=1))
    return np.concatenate([x, (np.stack(d, axis=1) / diag).astype(np.float32)], axis=1).astype(np.float32)


# ---------------------------------------------------------------------------
# Field readout: the IR at any receiver position of a (wall set, source)
# whose batched FDTD run recorded a grid of receivers.
# ---------------------------------------------------------------------------
GRID_H = 0.15  # m, spacing of the recorded receiver grid (about 9 points per wavelength at 250 Hz)


def receiver_grid(h=GRID_H):
    """Receiver cells on a regular grid of spacing h metres inside the
    MARGIN-cell band of the walls, in x-fastest order."""
    nx, ny, nz = ROOM
    step = max(1, int(round(h / DX)))
    axes = [np.arange(MARGIN, n - MARGIN, step) for n in (nx, ny, nz)]
    zz, yy, xx = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1).astype(np.int32)


def _pad_rows(t, m):
    import torch
    r = (-t.shape[0]) % m
    return t if r == 0 else torch.cat([t, t.new_zeros((r,) + tuple(t.shape[1:]))])


def _pad_cols(t, m):
    import torch
    r = (-t.shape[1]) % m
    return t if r == 0 else torch.cat([t, t.new_zeros((t.shape[0], r))], dim=1)


def gemm_split(pkg, a, b):
    """c = a @ b^T in FP32 from FP32 device matrices through the tcgen05 BF16
    GEMM: each operand split into a BF16 value and a BF16 remainder (about
    16 significant bits together), and three of the four products summed;
    the remainder-by-remainder product, about 2^-18 of the whole, is
    dropped. Relative accuracy near 1e-5, between BF16 and FP32. Rows are
    padded to 128 and the shared dimension to 64 with zeros."""
    import torch
    M, N = a.shape[0], b.shape[0]
    a = _pad_cols(_pad_rows(a, 128), 64)
    b = _pad_cols(_pad_rows(b, 128), 64)
    ah = a.to(torch.bfloat16)
    al = (a - ah.float()).to(torch.bfloat16)
    bh = b.to(torch.bfloat16)
    bl = (b - bh.float()).to(torch.bfloat16)
    c = torch.empty(a.shape[0], b.shape[0], dtype=torch.float32, device=a.device)
    t = torch.empty_like(c)
    st = torch.cuda.current_stream().cuda_stream
    G = pkg.surrogate.gemm_bf16
    G(ah, bh, c, st)
    G(ah, bl, t, st)
    c += t
    G(al, bh, t, st)
    c += t
    return c[:M, :N]


class FieldReadout:
    """IR at a receiver position as a linear readout of D random Fourier
    features of the position (metres): phi(r) = sqrt(2 / D) cos(W r + c),
    W ~ N(0, sigma^2) rad/m, c ~ U(0, 2 pi) -- a one-hidden-layer network
    whose hidden layer is fixed and whose output layer is fitted by ridge
    regression through the normal equations: the Gram matrix Phi^T Phi and
    Phi^T Y come from the tcgen05 GEMM (split BF16), the D x D system is
    solved in FP64. One readout serves every (wall set, source) recorded at
    the same receiver positions: their IRs are the columns of Y."""

    def __init__(self, pkg, n_feat=4096, sigma=6.0, ridge=1e-4, seed=0, source=None):
        import torch
        self.pkg = pkg
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.W = (torch.randn(3, n_feat, generator=g, dtype=torch.float64) * sigma).float().cuda()
        self.c = (torch.rand(n_feat, generator=g, dtype=torch.float64) * 2 * math.pi).float().cuda()
        self.base, self.ridge = n_feat, ridge
        # a readout of one source can carry the direct sound's 1/R near the
        # source: the features again, weighted by R0 / max(R, R_MIN)
        self.source = None if source is None else np.asarray(source, np.float64) * DX
        self.n_feat = n_feat * (2 if source is not None else 1)
        self.beta = None

    R0, R_MIN = 0.5, 0.1  # m

    def features(self, cells):
        import torch
        r = torch.as_tensor(np.asarray(cells, np.float64) * DX, dtype=torch.float32, device="cuda")
        phi = math.sqrt(2.0 / self.base) * torch.cos(r @ self.W + self.c)
        if self.source is None:
            return phi
        d = np.linalg.norm(np.asarray(cells, np.float64) * DX - self.source, axis=1)
        w = torch.as_tensor(self.R0 / np.maximum(d, self.R_MIN), dtype=torch.float32, device="cuda")
        return torch.cat([phi, phi * w[:, None]], dim=1).contiguous()

    def fit(self, cells, y):
        """cells [N, 3]; y [N, L] (device or host, FP32): one column block per
        (wall set, source)."""
        import torch
        phi = self.features(cells)                          # [N, D]
        pt = phi.t().contiguous()                           # [D, N]
        y = torch.as_tensor(y, dtype=torch.float32, device="cuda")
        gram = gemm_split(self.pkg, pt, pt).double()        # [D, D]
        rhs = gemm_split(self.pkg, pt, y.t().contiguous()).double()  # [D, L]
        # ridge relative to the mean diagonal; the Gram matrix of smooth
        # random features is numerically singular, so a ridge too small for
        # the factorisation is raised tenfold until it factors
        mean_diag = float(torch.trace(gram)) / self.n_feat
        ridge = self.ridge
        while True:
            a = gram.clone()
            a.diagonal().add_(ridge * mean_diag)
            L, info = torch.linalg.cholesky_ex(a)
            if int(info) == 0:
                break
            ridge *= 10.0
            if ridge > 1.0:
                raise RuntimeError("readout normal equations do not factor")
        self.ridge_used = ridge
        self.beta = torch.cholesky_solve(rhs, L).float()    # [D, L]
        self.beta_t = self.beta.t().contiguous()            # [L, D]
        return self

    def predict(self, cells):
        """[Q, L] FP32 device tensor: the readout at receiver cells."""
        return gemm_split(self.pkg, self.features(cells), self.beta_t)


def field_irs(pkg, g, src_cells, rcv_cells):
    """One batched FDTD run of wall set g: IRs [n_src, n_rcv, IR_LEN] on
    the device, and the run's wall seconds (setup excluded)."""
    import torch
    irs, wall = batched_irs(pkg, g, src_cells, rcv_cells)
    return torch.from_numpy(irs).cuda(), wall


def field_data(pkg, n_sets=2, n_src=8, n_query=96, n_val=96, seed=21, grid_h=GRID_H):
    """The batched FDTD runs behind the readout: per wall set one run of
    n_src sources whose receivers are the grid, n_query query and n_val
    validation positions. IRs stay on the device, [n_sets, n_src, n, L]."""
    import torch
    rng = np.random.default_rng(seed)
    grid = receiver_grid(grid_h)
    gsets = [rng.uniform(G_LO, G_HI, 4) for _ in range(n_sets)]
    srcs = [random_cells(rng, n_src) for _ in range(n_sets)]
    q_cells = random_cells(rng, n_query)
    v_cells = random_cells(rng, n_val)
    rcv = np.concatenate([grid, q_cells, v_cells])
    ng = len(grid)
    Y_grid, Y_q, Y_v, fd_s = [], [], [], []
    for w in range(n_sets):
        irs, wall = field_irs(pkg, gsets[w], srcs[w], rcv)
        fd_s.append(wall)
        Y_grid.append(irs[:, :ng])
        Y_q.append(irs[:, ng:ng + n_query])
        Y_v.append(irs[:, ng + n_query:])
        del irs
    # grid IRs as columns (wall set, source, sample)
    yg = torch.cat([t.permute(1, 0, 2).reshape(ng, -1) for t in Y_grid], dim=1)
    return {"grid": grid, "q_cells": q_cells, "v_cells": v_cells, "yg": yg, "yq": torch.stack(Y_q),
            "yv": torch.stack(Y_v), "fd_s": fd_s, "gsets": gsets, "srcs": srcs, "n_sets": n_sets, "n_src": n_src,
            "grid_h": grid_h, "seed": seed}


def readout_accounting(accept, t_pred, fd_s, t_plain=None):
    """IRs/s of the readout with its FDTD fallback against the FDTD alone.
    accept [n_sets, n_src, n_query]: pairs whose predicted error is within
    the bound; t_pred: seconds of the readout's predictions for every pair;
    fd_s: seconds of the batched FDTD run of each wall set (all its
    sources); t_plain: seconds of one plain single-source run (else one
    source's share of a batched run).
    Queries known before the runs: the FDTD answers every pair with one
    batched run per wall set; the readout falls back to one single-source
    run per (wall set, source) with a rejected pair.
    Query pairs arriving one at a time after the runs: the FDTD answers each
    with one source's share of a batched run (measured no slower than a
    plain single-source run); the readout pays that share for each rejected
    pair only."""
    accept = np.asarray(accept, bool)
    n_sets, n_src, n_query = accept.shape
    n_pairs = n_sets * n_src * n_query
    t_share = float(np.mean(fd_s)) / n_src
    t_single = t_plain if t_plain is not None else t_share
    runs_needed = int((~accept).any(axis=2).sum())
    rejected = int((~accept).sum())
    irs_fdtd = n_pairs / float(np.sum(fd_s))
    irs_readout = n_pairs / (t_pred + runs_needed * t_single)
    irs_fdtd_after = 1.0 / t_share
    irs_readout_after = n_pairs / (t_pred + rejected * t_share)
    return {"query_pairs": n_pairs, "fallback_runs": runs_needed, "rejected_pairs": rejected,
            "irs_fdtd": irs_fdtd, "irs_readout": irs_readout, "gain": irs_readout / irs_fdtd,
            "t_pair": t_share, "irs_fdtd_after": irs_fdtd_after, "irs_readout_after": irs_readout_after,
            "gain_after": irs_readout_after / irs_fdtd_after}


def run_field_readout(pkg, n_sets=2, n_src=8, n_query=96, n_val=96, bound=0.01, seed=21, n_feat=4096,
                      sigma=2.0, ridge=1e-4, grid_h=GRID_H, plain=True, data=None, near=True, calib_q=0.8):
    """The learned readout against the FDTD for receiver positions that the
    generating runs did not record as training data (new positions, the
    runs' own wall sets and sources; the query and validation receivers are
    recorded in the same runs as the FDTD answer). Per wall set: one batched
    FDTD run of n_src sources with the receiver grid, n_query query and n_val
    validation receivers (field_data; `data` reuses earlier runs). The
    readout is fitted on the grid; a committee of two readouts fitted on the
    two halves of the grid gives each pair a predicted error (their
    disagreement, calibrated on the validation receivers), and a pair whose
    predicted error exceeds `bound` falls back to the FDTD: one plain
    single-source run per (wall set, source) that has such a pair. Without
    the readout every query pair needs the FDTD: one batched run per wall
    set. That is the setting where every query position is known before the
    runs (the top-level gain); where query pairs arrive one at a time after
    the runs ("queries_after_runs"), the FDTD answers each pair with one
    source's share of a batched run of its wall set, and the readout pays
    that share for each rejected pair. The committee's
    disagreement is scaled to a predicted error by the `calib_q` quantile of
    true error / disagreement over the validation receivers. Reports
    errors, the fraction within the bound, IRs/s of each path and the gain
    in both settings."""
    import torch
    d = data or field_data(pkg, n_sets, n_src, n_query, n_val, seed, grid_h)
    n_sets, n_src = d["n_sets"], d["n_src"]
    grid, q_cells, v_cells = d["grid"], d["q_cells"], d["v_cells"]
    n_query, n_val, ng = len(q_cells), len(v_cells), len(grid)
    yg, fd_s = d["yg"], d["fd_s"]
    scale = float(yg.pow(2).mean().sqrt())
    ygs = yg / scale

    def triple(cols, src):
        def make():
            return FieldReadout(pkg, n_feat=n_feat, sigma=sigma, ridge=ridge, seed=seed, source=src)
        return (make().fit(grid, ygs[:, cols]), make().fit(grid[0::2], ygs[0::2, cols]),
                make().fit(grid[1::2], ygs[1::2, cols]))

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if near:
        # one readout per (wall set, source), with the source's 1/R features
        models = [[triple(slice((w * n_src + k) * IR_LEN, (w * n_src + k + 1) * IR_LEN), d["srcs"][w][k])
                   for k in range(n_src)] for w in range(n_sets)]
    else:
        models = triple(slice(None), None)  # one readout for every (wall set, source)
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t0

    def predict(cells, which):
        """[n_sets, n_src, n, L] predictions of readout `which` (0 full, 1, 2 halves)."""
        n = len(cells)
        if near:
            return torch.stack([torch.stack([models[w][k][which].predict(cells) for k in range(n_src)])
                                for w in range(n_sets)])
        return models[which].predict(cells).reshape(n, n_sets, n_src, IR_LEN).permute(1, 2, 0, 3)

    def rel(a, b):
        return ((a - b).norm(dim=-1) / b.norm(dim=-1).clamp_min(1e-30)).cpu().numpy()

    yv = d["yv"] / scale
    pv = predict(v_cells, 0)
    dv = rel(predict(v_cells, 1), predict(v_cells, 2))
    ev = rel(pv, yv)
    # true error per unit of committee disagreement, a high quantile so that
    # few accepted pairs exceed the bound
    calib = float(np.quantile(ev / np.maximum(dv, 1e-12), calib_q))
    yq = d["yq"] / scale
    predict(q_cells[:8], 0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pq = predict(q_cells, 0)
    dq = rel(predict(q_cells, 1), predict(q_cells, 2))
    torch.cuda.synchronize()
    t_pred = time.perf_counter() - t0
    eq = rel(pq, yq)                           # [n_sets, n_src, n_query]
    dist = np.stack([np.stack([np.linalg.norm((q_cells - np.asarray(d["srcs"][w][k])) * DX, axis=1)
                               for k in range(n_src)]) for w in range(n_sets)])
    far = dist >= 0.5
    pe = calib * dq
    accept = pe <= bound
    t_plain = None
    if plain:
        _, t_plain = plain_irs(pkg, d["gsets"][0], d["srcs"][0][0], q_cells[:16])
    acc = readout_accounting(accept, t_pred, fd_s, t_plain)
    n_pairs = acc["query_pairs"]
    runs_needed, rejected = acc["fallback_runs"], acc["rejected_pairs"]
    irs_fdtd, irs_sur = acc["irs_fdtd"], acc["irs_readout"]
    irs_fdtd_after, irs_sur_after = acc["irs_fdtd_after"], acc["irs_readout_after"]
    t_pair = acc["t_pair"]
    return {
        "wall_sets": n_sets, "sources_per_set": n_src, "grid_receivers": ng, "grid_spacing_m": d["grid_h"],
        "query_pairs": n_pairs, "validation_pairs": n_sets * n_src * n_val, "features": n_feat,
        "sigma_rad_per_m": sigma, "near_field_features": bool(near), "fit_s": t_fit, "fdtd_run_s": fd_s,
        "query_rel_l2": {"median": float(np.median(eq)), "p90": float(np.percentile(eq, 90)),
                         "max": float(eq.max())},
        "validation_median_rel_l2": float(np.median(ev)),
        "query_rel_l2_beyond_half_metre": {"median": float(np.median(eq[far])) if far.any() else None,
                                           "within_bound": float((eq[far] <= bound).mean()) if far.any() else None,
                                           "pairs": int(far.sum())},
        "within_bound": float((eq <= bound).mean()), "accepted": float(accept.mean()),
        "accepted_but_over_bound": int((accept & (eq > bound)).sum()),
        "fallback_runs": runs_needed,
        "irs_per_s": {"readout_only": n_pairs / t_pred, "readout_with_fallback": irs_sur,
                      "batched_fdtd": irs_fdtd, "plain_fdtd": (16 / t_plain) if t_plain else None},
        "gain_over_fdtd": irs_sur / irs_fdtd, "bound": bound, "calibration_quantile": calib_q,
        "queries_after_runs": {"fallback_runs": rejected, "fdtd_s_per_pair": t_pair,
                               "irs_per_s": {"readout_with_fallback": irs_sur_after, "fdtd": irs_fdtd_after},
                               "gain_over_fdtd": irs_sur_after / irs_fdtd_after},
    }
