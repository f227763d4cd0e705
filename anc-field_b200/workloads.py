"""Seeded synthetic rooms, filters and signals for the benchmark
configurations (no datasets: every input is generated from a seed).

Room construction: a solid one-cell shell on the chosen faces of the grid
box, seeded axis-aligned boxes inside, material per wall and per box, then
a closing pass that fills one-cell gaps so that no air cell has solid
neighbours on opposite sides or more than three solid neighbours (the
patterns lrs-data.hpp:327 rejects as unphysical).

Filters: admittance Y(z) = A(z)/B(z) as a sum of first-order sections
g_k (1 + alpha_k z^-1) / (1 + beta_k z^-1) with g_k > 0 and |alpha_k|,
|beta_k| < 1. Each section is positive real, so the sum is passive
(Re Y >= 0 on the unit circle), and B has its roots at -beta_k, inside the
unit circle (stable). n sections give K = n + 1 coefficients.
"""
import math

import numpy as np

FACE_XM, FACE_XP, FACE_YM, FACE_YP, FACE_ZM, FACE_ZP = 1, 2, 4, 8, 16, 32


def courant_dt(dx, c, courant=0.99 / math.sqrt(3.0)):
    """Time step for a Courant number lambda = c dt / dx."""
    return courant * dx / c


def passive_filters(nmat, K, seed, gain=(0.05, 0.6), pole=0.6, zero=0.6):
    """a, b float64 [nmat, K]: stable, passive admittance filters."""
    rng = np.random.default_rng(seed)
    a = np.zeros((nmat, K))
    b = np.zeros((nmat, K))
    for m in range(nmat):
        if K == 1:
            a[m, 0] = rng.uniform(*gain)
            b[m, 0] = 1.0
            continue
        n = K - 1
        g = rng.uniform(gain[0] / n, gain[1] / n, n)
        al = rng.uniform(-zero, zero, n)
        be = rng.uniform(-pole, pole, n)
        den = np.array([1.0])
        for k in range(n):
            den = np.convolve(den, [1.0, be[k]])
        num = np.zeros(K)
        for k in range(n):
            part = np.array([g[k], g[k] * al[k]])
            for j in range(n):
                if j != k:
                    part = np.convolve(part, [1.0, be[j]])
            num += part
        a[m] = num
        b[m] = den
    return a, b


def admittance_real_min(a, b, n=4096):
    w = np.linspace(0.0, np.pi, n)
    z = np.exp(-1j * np.outer(w, np.arange(a.shape[-1])))
    return np.real((z @ a.T) / (z @ b.T)).min(axis=0)


def _unphysical(solid):
    """Air cells (interior) with opposite solid neighbours or > 3 solid ones."""
    s = solid
    air = ~s[1:-1, 1:-1, 1:-1]
    xp, xm = s[1:-1, 1:-1, 2:], s[1:-1, 1:-1, :-2]
    yp, ym = s[1:-1, 2:, 1:-1], s[1:-1, :-2, 1:-1]
    zp, zm = s[2:, 1:-1, 1:-1], s[:-2, 1:-1, 1:-1]
    cnt = xp.astype(np.int8) + xm + yp + ym + zp + zm
    bad = ((xp & xm) | (yp & ym) | (zp & zm) | (cnt > 3)) & air
    return bad


def close_gaps(vox):
    """Fills unphysical air cells with a neighbouring material until none is left."""
    vox = vox.copy()
    for _ in range(64):
        bad = _unphysical(vox != -1)
        if not bad.any():
            return vox
        zz, yy, xx = np.nonzero(bad)
        zz, yy, xx = zz + 1, yy + 1, xx + 1
        for dz, dy, dx in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
            m = vox[zz + dz, yy + dy, xx + dx]
            take = (vox[zz, yy, xx] == -1) & (m != -1)
            vox[zz[take], yy[take], xx[take]] = m[take]
    raise RuntimeError("could not make the geometry physical")


def room(nx, ny, nz, walls, n_boxes, nmat, seed, box_min=4, box_max=None):
    """int32 voxels [nz, ny, nx]: shell on the faces in `walls`, seeded boxes."""
    rng = np.random.default_rng(seed)
    vox = -np.ones((nz, ny, nx), np.int32)
    face_mat = rng.integers(0, nmat, 6)
    if walls & FACE_XM:
        vox[:, :, 0] = face_mat[0]
    if walls & FACE_XP:
        vox[:, :, -1] = face_mat[1]
    if walls & FACE_YM:
        vox[:, 0, :] = face_mat[2]
    if walls & FACE_YP:
        vox[:, -1, :] = face_mat[3]
    if walls & FACE_ZM:
        vox[0, :, :] = face_mat[4]
    if walls & FACE_ZP:
        vox[-1, :, :] = face_mat[5]
    box_max = box_max or max(box_min + 1, min(nx, ny, nz) // 4)
    for _ in range(n_boxes):
        sx, sy, sz = rng.integers(box_min, box_max + 1, 3)
        x0 = rng.integers(3, max(4, nx - sx - 3))
        y0 = rng.integers(3, max(4, ny - sy - 3))
        z0 = rng.integers(3, max(4, nz - sz - 3))
        vox[z0:z0 + sz, y0:y0 + sy, x0:x0 + sx] = rng.integers(0, nmat)
    return close_gaps(vox)


def air_cells(vox, n, seed, margin=2, near_wall=False):
    """n distinct seeded air cells (x, y, z); near_wall picks cells with a
    solid face neighbour (wall-adjacent loudspeaker positions)."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = vox.shape
    solid = vox != -1
    cand = ~solid
    if near_wall:
        nb = np.zeros_like(solid)
        nb[:, :, :-1] |= solid[:, :, 1:]
        nb[:, :, 1:] |= solid[:, :, :-1]
        nb[:, :-1, :] |= solid[:, 1:, :]
        nb[:, 1:, :] |= solid[:, :-1, :]
        nb[:-1, :, :] |= solid[1:, :, :]
        nb[1:, :, :] |= solid[:-1, :, :]
        cand &= nb
    m = np.zeros_like(cand)
    m[margin:nz - margin, margin:ny - margin, margin:nx - margin] = True
    cand &= m
    zz, yy, xx = np.nonzero(cand)
    pick = rng.choice(len(xx), size=n, replace=False)
    return [(int(xx[i]), int(yy[i]), int(zz[i])) for i in pick]


def gaussian_pulse(n, fs, f0=500.0, sigma=1.5e-3, t0=6e-3):
    t = np.arange(n) / fs
    return (np.exp(-((t - t0) / sigma) ** 2) * np.sin(2 * np.pi * f0 * (t - t0))).astype(np.float32)


def band_noise(n, fs, lo=50.0, hi=2000.0, seed=0, taps=1023):
    """Seeded white noise band-limited by a windowed-sinc FIR (as
    ancutil.bandnoise filters uniform noise), scaled to unit RMS."""
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1.0, 1.0, n + taps)
    k = np.arange(taps) - (taps - 1) / 2.0
    w = np.hamming(taps)

    def lp(fc):
        return 2 * fc / fs * np.sinc(2 * fc / fs * k) * w

    h = lp(hi) - lp(lo)
    x = np.convolve(z, h, mode="valid")[:n]
    return (x / np.sqrt(np.mean(x ** 2))).astype(np.float32)


def unit_impulse(n):
    x = np.zeros(n, np.float32)
    x[0] = 1.0
    return x


def ksi_profile(length, kmax=8000.0):
    """Damping values of generate_ksi.m:1-7 for one slab, outermost first:
    kmax (d - sin(2 pi d)/(2 pi)) at normalised depth d = (L-i)/L."""
    i = np.arange(length)
    d = (length - i) / float(length)
    return (kmax * (d - np.sin(2 * np.pi * d) / (2 * np.pi))).astype(np.float32)


def ksi_arrays(dims, width, faces, kmax=8000.0):
    """Per-axis ksi arrays with the profile on the faces in `faces`."""
    prof = ksi_profile(width, kmax)
    out = []
    for ax, n in enumerate(dims):
        k = np.zeros(n, np.float32)
        if faces & (1 << (2 * ax)):
            k[:width] = prof
        if faces & (2 << (2 * ax)):
            k[n - width:] = prof[::-1]
        out.append(k)
    return tuple(out)


class Config:
    """One FDTD workload: grid, voxels, filters, PML, sources, receivers."""

    def __init__(self, name, dims, vox, a, b, dx, c, dt, steps, sources, receivers, pml_width=0,
                 pml_faces=0, ksi=None, mode=1, batch_sources=None):
        self.name = name
        self.dims = dims
        self.vox = vox
        self.a = a
        self.b = b
        self.dx, self.c, self.dt = dx, c, dt
        self.steps = steps
        self.sources = sources              # [((i,j,k), signal)] of batch member 0
        self.batch_sources = batch_sources  # [[((i,j,k), signal)], ...] per member, or None
        self.receivers = receivers
        self.pml_width = pml_width
        self.pml_faces = pml_faces
        self.ksi = ksi
        self.mode = mode

    @property
    def cells(self):
        nx, ny, nz = self.dims
        return nx * ny * nz


def config_c1(variant="fixed", steps=2000, seed=1):
    """160x120x100, dx 2.5 cm, c 343, Courant 0.99/sqrt(3), one seeded box,
    first-order filters (K = 2), LRS walls on five faces, 12-cell PML on the
    sixth (z+), Gaussian-modulated 500 Hz pulse, 8 receivers.
    variant "ref": sixth face also a wall, no PML, REF semantics.
    variant "refpml": like "ref" plus the reference PML (whole interior) of
    width 12 with the generate_ksi profile on all faces."""
    nx, ny, nz = 160, 120, 100
    dx, c = 0.025, 343.0
    dt = courant_dt(dx, c)
    fs = 1.0 / dt
    walls = 63 if variant in ("ref", "refpml") else 63 & ~FACE_ZP
    vox = room(nx, ny, nz, walls, n_boxes=1, nmat=3, seed=seed, box_min=10, box_max=30)
    a, b = passive_filters(3, 2, seed + 100)
    src_cell = air_cells(vox, 1, seed + 200, margin=10)[0]
    rcv = air_cells(vox, 8, seed + 300, margin=3)
    sig = gaussian_pulse(steps, fs)
    if variant == "fixed":
        ksi = ksi_arrays((nx, ny, nz), 12, FACE_ZP)
        return Config("c1", (nx, ny, nz), vox, a, b, dx, c, dt, steps, [(src_cell, sig)], rcv, 12,
                      FACE_ZP, ksi, mode=1)
    if variant == "refpml":
        ksi = ksi_arrays((nx, ny, nz), 12, 63)
        return Config("c1-refpml", (nx, ny, nz), vox, a, b, dx, c, dt, steps, [(src_cell, sig)], rcv, 12,
                      63, ksi, mode=0)
    return Config("c1-ref", (nx, ny, nz), vox, a, b, dx, c, dt, steps, [(src_cell, sig)], rcv, mode=0)


def config_c2(steps=5000, seed=2, dims=(512, 384, 320)):
    """512x384x320 (~63M cells), 4 materials with third-order filters
    (K = 4), 20 seeded furniture boxes, PML on two faces (x+ and z+),
    band-limited white noise (50-2000 Hz, unit RMS), 32 receivers.
    `dims` scales the same construction (profiling captures)."""
    nx, ny, nz = dims
    dx, c = 0.025, 343.0
    dt = courant_dt(dx, c)
    fs = 1.0 / dt
    faces = FACE_XP | FACE_ZP
    vox = room(nx, ny, nz, 63 & ~faces, n_boxes=20, nmat=4, seed=seed, box_min=8,
               box_max=max(9, min(60, min(dims) // 3)))
    a, b = passive_filters(4, 4, seed + 100)
    src_cell = air_cells(vox, 1, seed + 200, margin=20)[0]
    rcv = air_cells(vox, 32, seed + 300, margin=3)
    sig = band_noise(steps, fs, seed=seed + 400)
    ksi = ksi_arrays((nx, ny, nz), 12, faces)
    return Config("c2", (nx, ny, nz), vox, a, b, dx, c, dt, steps, [(src_cell, sig)], rcv, 12, faces, ksi,
                  mode=1)


def config_c3(steps=8192, seed=3, n_src=16, dims=(256, 192, 160)):
    """Shared room (C1 construction at 256x192x160), 16 wall-adjacent
    sources each a unit impulse in its own batch member, 16 receivers."""
    nx, ny, nz = dims
    dx, c = 0.025, 343.0
    dt = courant_dt(dx, c)
    vox = room(nx, ny, nz, 63 & ~FACE_ZP, n_boxes=1, nmat=3, seed=seed, box_min=10, box_max=40)
    a, b = passive_filters(3, 2, seed + 100)
    srcs = air_cells(vox, n_src, seed + 200, margin=2, near_wall=True)
    rcv = air_cells(vox, 16, seed + 300, margin=3)
    imp = unit_impulse(1)
    ksi = ksi_arrays((nx, ny, nz), 12, FACE_ZP)
    cfg = Config("c3", (nx, ny, nz), vox, a, b, dx, c, dt, steps, [(srcs[0], imp)], rcv, 12, FACE_ZP, ksi,
                 mode=1, batch_sources=[[(s, imp)] for s in srcs])
    return cfg


def pack_rooms(rooms, filler=0):
    """Packs rooms of uneven size into one voxel grid so that one simulation
    (one launch per kernel per step) advances them all. Each room is
    int32 voxels [nz, ny, nx] with solid walls on every face except z+ (its
    PML face). Rooms are placed on shelves along x, rows along y, all
    top-aligned so that every open z+ face lies on the grid's z+ face (the
    PML slab then covers the same top layers of every room); everything
    outside the rooms is solid. In the FIXED scheme no air cell reads across
    a wall, so each packed room evolves exactly as it does alone.
    Returns (voxels, offsets [(ox, oy, oz)] per room)."""
    dims = [r.shape[::-1] for r in rooms]  # (nx, ny, nz)
    nz = max(d[2] for d in dims)
    order = sorted(range(len(rooms)), key=lambda i: -dims[i][1])
    width = int(np.ceil(np.sqrt(sum(d[0] * d[1] for d in dims)) * 1.3))
    width = max(width, max(d[0] for d in dims))
    offsets = [None] * len(rooms)
    x = y = row_h = 0
    for i in order:
        nx_i, ny_i, nz_i = dims[i]
        if x + nx_i > width:
            x, y, row_h = 0, y + row_h, 0
        offsets[i] = (x, y, nz - nz_i)
        x += nx_i
        row_h = max(row_h, ny_i)
    gx = max(o[0] + d[0] for o, d in zip(offsets, dims))
    gy = max(o[1] + d[1] for o, d in zip(offsets, dims))
    vox = np.full((nz, gy, gx), filler, np.int32)
    for r, (ox, oy, oz) in zip(rooms, offsets):
        vox[oz:oz + r.shape[0], oy:oy + r.shape[1], ox:ox + r.shape[2]] = r
    return vox, offsets


def config_c3_rooms(n_rooms=8, lo=96, hi=256, steps=2048, seed=5, n_rcv=16):
    """Uneven batch of rooms (C1 construction, edges drawn from lo..hi
    cells): one unit-impulse source near a wall and n_rcv receivers per
    room, all rooms packed into one grid. Returns (Config of the packed
    grid, per-room list of (voxels, source cell, receiver cells) in room
    coordinates, offsets)."""
    rng = np.random.default_rng(seed)
    a, b = passive_filters(3, 2, seed + 100)
    rooms, parts = [], []
    for k in range(n_rooms):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, 3))
        vox = room(nx, ny, nz, 63 & ~FACE_ZP, n_boxes=1, nmat=3, seed=seed + 10 + k, box_min=8,
                   box_max=max(9, min(nx, ny, nz) // 4))
        src = air_cells(vox, 1, seed + 200 + k, margin=2, near_wall=True)[0]
        rcv = air_cells(vox, n_rcv, seed + 300 + k, margin=3)
        rooms.append(vox)
        parts.append((vox, src, rcv))
    packed, offsets = pack_rooms(rooms)
    gz, gy, gx = packed.shape
    dx, c = 0.025, 343.0
    imp = unit_impulse(1)
    srcs, rcvs = [], []
    for (vox, s, r), (ox, oy, oz) in zip(parts, offsets):
        srcs.append(((s[0] + ox, s[1] + oy, s[2] + oz), imp))
        rcvs += [(q[0] + ox, q[1] + oy, q[2] + oz) for q in r]
    ksi = ksi_arrays((gx, gy, gz), 12, FACE_ZP)
    cfg = Config("c3-rooms", (gx, gy, gz), packed, a, b, dx, c, courant_dt(dx, c), steps, srcs, rcvs, 12, FACE_ZP,
                 ksi, mode=1)
    return cfg, parts, offsets
