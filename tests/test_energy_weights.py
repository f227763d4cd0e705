"""The weighted discrete energy that afd_energy sums on the GPU, restated in
numpy, checked on the FP64 oracle's FIXED-scheme fields of a walled box:
constant for rigid walls (admittance 0) and non-increasing for passive
one-coefficient LRS walls (admittance > 0).

A boundary cell's update (lrs-data.hpp update forms, the mirror of the
missing neighbour across each wall) makes it a half cell per walled axis, so
the energy is 1/2 sum w_i (u1_i-u0_i)^2 + lambda2/2 sum w_e (u1_i-u1_j)
(u0_i-u0_j) over the air cells 1..n-2 and the edges between air cells, with
w_i = 1/2 per axis on which cell i has a wall and w_e = 1/2 per other axis on
which both ends have the same wall. The scheme is self-adjoint under these
weights only where the air region is a box: at the edge of an obstacle a half
cell meets a whole cell across an unwalled axis, and no diagonal weighting
balances that, so the check is stated for box-shaped rooms.
"""
import numpy as np

import oracle

LAMBDA2 = float(np.float32(np.float32(3.125e-5 * 340.0 / 0.02) ** 2))


def wall_bits(solid):
    """Bit d of cell i set when its neighbour in direction d (x+, x-, y+, y-,
    z+, z-) is solid; cells outside the grid are air."""
    nz, ny, nx = solid.shape
    sp = np.pad(solid, 1)
    m = np.zeros(solid.shape, np.int64)
    for d, (dz, dy, dx) in enumerate([(0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)]):
        m |= sp[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx].astype(np.int64) << d
    return m


def walled_axes(m, skip=-1):
    return sum((((m >> (2 * b)) & 3) != 0).astype(np.int64) for b in range(3) if b != skip)


def weighted_energy(u1, u0, solid, lam2):
    u1 = np.asarray(u1, np.float64)
    u0 = np.asarray(u0, np.float64)
    nz, ny, nx = u1.shape
    m = wall_bits(solid)
    core = (slice(1, nz - 1), slice(1, ny - 1), slice(1, nx - 1))
    node = ~solid[core]
    e = 0.5 * np.sum((0.5 ** walled_axes(m[core]) * (u1 - u0)[core] ** 2)[node])
    pot = 0.0
    for ax, arr_ax in ((0, 2), (1, 1), (2, 0)):
        for sgn in (1, -1):  # the edge to the next cell, and at index 1 the edge to the outer face
            i = list(core)
            if sgn < 0:
                i[arr_ax] = slice(1, 2)
            j = list(i)
            j[arr_ax] = slice(i[arr_ax].start + sgn, i[arr_ax].stop + sgn)
            i, j = tuple(i), tuple(j)
            ok = ~solid[i] & ~solid[j]
            we = 0.5 ** walled_axes(m[i] & m[j], ax)
            pot += np.sum((we * (u1[i] - u1[j]) * (u0[i] - u0[j]))[ok])
    return e + 0.5 * lam2 * pot


def walled_box(nx, ny, nz):
    """Air box inside one-cell walls of three materials."""
    vox = -np.ones((nz, ny, nx), np.int32)
    vox[0], vox[-1] = 0, 1
    vox[:, 0], vox[:, -1] = 2, 0
    vox[:, :, 0], vox[:, :, -1] = 1, 2
    return vox


PULSE = np.zeros(30, np.float32)
PULSE[:5] = [0.2, 1.0, 0.5, -0.3, 0.1]


def oracle_energies(vox, a, b, checkpoints, precision):
    nz, ny, nx = vox.shape
    out = []
    for n in checkpoints:
        f = [oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=[((9, 8, 7), PULSE)], receivers=[(5, 5, 5)],
                             steps=s, want_field=True, precision=precision)[1] for s in (n, n + 1)]
        out.append(weighted_energy(f[1], f[0], vox != -1, LAMBDA2))
    return np.array(out)


def test_rigid_walls_conserve_weighted_energy():
    vox = walled_box(24, 20, 16)
    a = np.zeros((3, 1))
    e = oracle_energies(vox, a, np.ones((3, 1)), (40, 160, 320), "f64")
    assert e[0] > 0
    assert np.ptp(e) / e[0] < 1e-7


def test_passive_walls_weighted_energy_non_increasing():
    vox = walled_box(24, 20, 16)
    a = np.array([[0.15], [0.4], [0.25]])
    e = oracle_energies(vox, a, np.ones((3, 1)), range(40, 281, 40), "f64")
    assert np.all(e[1:] <= e[:-1])
    assert e[-1] < 0.1 * e[0]


def test_weights_are_one_without_walls():
    rng = np.random.default_rng(3)
    u1, u0 = rng.standard_normal((2, 7, 6, 5))
    solid = np.zeros((7, 6, 5), bool)
    want = 0.5 * np.sum((u1 - u0)[1:-1, 1:-1, 1:-1] ** 2)
    pot = 0.0
    for ax in range(3):
        for lo, hi in ((slice(1, -1), slice(2, None)), (slice(1, 2), slice(0, 1))):
            i = [slice(1, -1)] * 3
            j = [slice(1, -1)] * 3
            i[ax], j[ax] = lo, hi
            i, j = tuple(i), tuple(j)
            pot += np.sum((u1[i] - u1[j]) * (u0[i] - u0[j]))
    want += 0.5 * 0.25 * pot
    assert abs(weighted_energy(u1, u0, solid, 0.25) - want) <= 1e-12 * abs(want)
