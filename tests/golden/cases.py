"""Seeded small rooms for the golden fixtures (reference semantics)."""
import numpy as np

CASES = {
    # name: grid, filter length, seeds, steps, PML, runs
    "k1": {"grid": [28, 22, 18], "K": 1, "seed": 1, "steps": 160, "pml": 0, "runs": [160]},
    "k2": {"grid": [28, 22, 18], "K": 2, "seed": 2, "steps": 160, "pml": 0, "runs": [160]},
    "k3": {"grid": [24, 26, 20], "K": 3, "seed": 3, "steps": 150, "pml": 0, "runs": [150]},
    "k4": {"grid": [30, 20, 22], "K": 4, "seed": 4, "steps": 150, "pml": 0, "runs": [150]},
    "k2_pml": {"grid": [28, 24, 20], "K": 2, "seed": 5, "steps": 140, "pml": 5, "runs": [140]},
    "k3_runs": {"grid": [26, 22, 18], "K": 3, "seed": 6, "steps": 180, "pml": 0, "runs": [1, 70, 109]},
    "k1_pml_8000": {"grid": [20, 18, 16], "K": 1, "seed": 7, "steps": 8003, "pml": 4, "runs": [8003]},
}


def build_case(spec):
    """Room with a solid shell on all faces and two boxes (one touching a
    wall so that edge and corner groups occur, including X_M_Y_M_Z_M),
    three materials, two sources and four receivers."""
    nx, ny, nz = spec["grid"]
    K = spec["K"]
    rng = np.random.default_rng(spec["seed"])
    vox = -np.ones((nz, ny, nx), np.int32)
    vox[0], vox[-1] = 0, 1
    vox[:, 0], vox[:, -1] = 2, 0
    vox[:, :, 0], vox[:, :, -1] = 1, 2
    vox[4:8, 5:9, 6:11] = 1           # free-standing box
    vox[1:5, 1:4, 1:5] = 2            # box in the (0,0,0) corner
    a = np.zeros((3, K))
    b = np.zeros((3, K))
    for m in range(3):
        a[m] = rng.uniform(0.02, 0.5, K) * np.array([1.0] + [0.3] * (K - 1))
        b[m] = np.array([1.0] + list(rng.uniform(-0.4, 0.4, K - 1)))
    a = a.astype(np.float32).astype(np.float64)
    b = b.astype(np.float32).astype(np.float64)
    T = spec["steps"]
    s1 = rng.standard_normal(T).astype(np.float32)
    s2 = (0.5 * rng.standard_normal(T // 2)).astype(np.float32)
    sources = [((nx // 2, ny // 2, nz // 2), s1), ((nx - 4, 3, nz - 5), s2)]
    receivers = [(nx // 3, ny // 3, nz // 3), (1, 1, 1), (nx - 2, ny - 2, nz - 2), (5, 5, 5)]
    inp = dict(grid=(nx, ny, nz), vox=vox, a=a, b=b, dx=0.02, c=340.0, dt=3.125e-5, mode=0,
               sources=sources, receivers=receivers, runs=spec["runs"])
    if spec["pml"]:
        L = 6
        prof = np.linspace(7000.0, 0.0, L).astype(np.float32)
        ksi = []
        for n in (nx, ny, nz):
            k = np.zeros(n, np.float32)
            for i in range(L):
                k[i] = prof[L - 1 - i]
                k[n - 1 - i] = prof[L - 1 - i]
            ksi.append(k)
        inp.update(pml_width=spec["pml"], ksi=tuple(ksi))
    return inp
