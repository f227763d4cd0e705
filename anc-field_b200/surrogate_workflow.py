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
