"""z-slab domain decomposition of one FDTD grid over several simulations.

The reference advances one grid on one device (simulation.hpp:176-178,
356-402). Here the interior planes 1..NZ-2 of a grid are split into
contiguous parts; part r owns global planes [a_r, b_r) and simulates the
planes a_r - 1 .. b_r, whose two end planes are halos (or the global end
faces) refreshed from its neighbours. Every kernel treats a grid's end planes
as faces it never writes, so a part runs the interior and boundary updates
unchanged; the PML cell rule and the z slabs follow global planes
(afd_set_slab).

Per time step (FIXED scheme, FP32):
  phase 1 on every part   interior, boundary and PML pressure updates
  exchange A              each part's high-z halo of the new pressure (and
                          of the new psi when it is kept) from the part
                          above: the auxiliary update of a part's last plane
                          reads both at z + 1
  phase 2 on every part   PML auxiliary updates, sources, receivers
  exchange B              both halos of the new pressure (the next step's
                          stencils read z - 1 and z + 1) and the high-z
                          halos of the new auxiliary fields (the next PML
                          pressure update reads them at z + 1)

Each exchange moves whole planes: nothing crosses between parts but these
planes, and every part's cells get exactly the arithmetic of the undivided
grid, so a decomposed run equals the undivided run bit for bit.

Transports: `run_local` for parts in one process (device-to-device copies
through one staging buffer), `run_rank` for one part per rank of a
torch.distributed process group (NCCL between GPUs, gloo on CPU), both built
on `halo_plan`, the list of plane transfers of an exchange.
"""
import numpy as np

PRESSURE, FI_X, FI_Y, FI_Z, PSI = 0, 1, 2, 3, 4
LOW, HIGH = 0, 1          # side of a part
READ, WRITE = 0, 1        # afd_halo direction


def split_planes(nz, parts):
    """Contiguous split of the interior planes 1..nz-2 into `parts` ranges
    [a, b), sizes differing by at most one."""
    n = nz - 2
    if parts < 1 or n < parts:
        raise ValueError("cannot split %d interior planes into %d parts" % (n, parts))
    base, extra = divmod(n, parts)
    out, a = [], 1
    for r in range(parts):
        b = a + base + (1 if r < extra else 0)
        out.append((a, b))
        a = b
    return out


def exchange_fields(faces, psi_on, which):
    """Fields of exchange `which` ("A" or "B") travelling downwards (from a
    part to the one below it, into its high-z halo) and upwards."""
    if which == "A":
        return [PRESSURE] + ([PSI] if psi_on else []), []
    axes = [FI_X + ax for ax in range(3) if faces & (3 << (2 * ax))]
    return [PRESSURE] + axes, [PRESSURE]


def halo_plan(rank, world, faces, psi_on, which):
    """Plane transfers of one exchange for part `rank` of `world`:
    a list of ("send", peer, side, field) and ("recv", peer, side, field),
    in the order every rank issues them (sends before receives, fields in
    a fixed order), so that matching transfers pair up."""
    down, up = exchange_fields(faces, psi_on, which)
    ops = []
    # downwards: the low-z own plane of part r goes to the high-z halo of r-1
    for f in down:
        if rank > 0:
            ops.append(("send", rank - 1, LOW, f))
    for f in up:
        if rank < world - 1:
            ops.append(("send", rank + 1, HIGH, f))
    for f in down:
        if rank < world - 1:
            ops.append(("recv", rank + 1, HIGH, f))
    for f in up:
        if rank > 0:
            ops.append(("recv", rank - 1, LOW, f))
    return ops


class Part:
    """One slab: the simulation of global planes a-1 .. b and the map of its
    receivers to the global receiver list."""

    def __init__(self, sim, a, b, rcv_index):
        self.sim = sim
        self.a, self.b = a, b
        self.rcv_index = rcv_index


def make_part(pkg, vox, a_coef, b_coef, a, b, nz_global, sources, receivers, pml=None, device=0, batch=1,
              **params):
    """The simulation of global planes a-1 .. b of a FIXED-scheme grid.
    vox int32 [NZ, NY, NX]; sources [(batch, (x, y, z), signal)] and
    receivers [(x, y, z)] in global cells (each kept by the part owning its
    plane); pml = (width, faces, (kx, ky, kz)) with global ksi arrays."""
    z0 = a - 1
    sub = np.ascontiguousarray(vox[z0:b + 1])
    sim = pkg.Simulation(mode=1, batch=batch, device=device, graphs=0, **params)
    sim.SetModel(pkg.Model.from_voxels(sub, a_coef, b_coef))
    sim.set_slab(z0, nz_global)
    if pml is not None:
        width, faces, (kx, ky, kz) = pml
        sim.SetPml(width, faces=faces, ksi=(kx, ky, np.ascontiguousarray(kz[z0:b + 1])))
    for m, (x, y, z), sig in sources:
        if a <= z < b:
            sim.AddSourceCell((x, y, z - z0), sig, batch=m)
    idx = []
    for k, (x, y, z) in enumerate(receivers):
        if a <= z < b:
            sim.AddMicCell((x, y, z - z0))
            idx.append(k)
    return Part(sim, a, b, idx)


def _plane_floats(sim):
    i = sim.info()
    pitch = (i.nx + 31) // 32 * 32
    return i.batch * i.ny * pitch


def run_local(parts, steps, faces, psi_on, torch_device="cuda"):
    """Advances parts that live in this process (on one or several GPUs of
    it) by `steps` steps, exchanging through a device staging buffer."""
    import torch
    n = max(_plane_floats(p.sim) for p in parts)
    buf = torch.empty(n, dtype=torch.float32, device=torch_device)
    for p in parts:
        p.sim.prepare(steps)

    def exchange(which):
        world = len(parts)
        for r in range(world):
            for op, peer, side, f in halo_plan(r, world, faces, psi_on, which):
                if op != "recv":
                    continue
                # the peer reads its own plane facing part r; part r writes its halo
                parts[peer].sim.halo(1 - side, READ, f, buf.data_ptr(), n)
                parts[r].sim.halo(side, WRITE, f, buf.data_ptr(), n)

    for _ in range(steps):
        for p in parts:
            p.sim.step_phase(1)
        exchange("A")
        for p in parts:
            p.sim.step_phase(2)
        exchange("B")


def run_rank(part, steps, faces, psi_on, rank, world, device="cuda"):
    """Advances this rank's part by `steps` steps, exchanging halo planes with
    the neighbouring ranks through torch.distributed (point-to-point sends
    and receives of one plane buffer per transfer, all transfers of an
    exchange posted together and then waited on)."""
    import torch
    import torch.distributed as dist
    n = _plane_floats(part.sim)
    part.sim.prepare(steps)

    def exchange(which):
        ops, bufs = [], []
        for op, peer, side, f in halo_plan(rank, world, faces, psi_on, which):
            t = torch.empty(n, dtype=torch.float32, device=device)
            if op == "send":
                part.sim.halo(side, READ, f, t.data_ptr(), n)
                ops.append(dist.P2POp(dist.isend, t, peer))
            else:
                ops.append(dist.P2POp(dist.irecv, t, peer))
            bufs.append((op, side, f, t))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if device != "cpu":
            torch.cuda.synchronize()
        for op, side, f, t in bufs:
            if op == "recv":
                part.sim.halo(side, WRITE, f, t.data_ptr(), n)

    for _ in range(steps):
        part.sim.step_phase(1)
        exchange("A")
        part.sim.step_phase(2)
        exchange("B")


def gather_receivers(parts, n_receivers, steps, batch=0):
    """The global receiver array [n_receivers, steps] of parts in this
    process."""
    out = np.zeros((n_receivers, steps), np.float32)
    for p in parts:
        if p.rcv_index:
            out[p.rcv_index] = p.sim.mics(batch=batch)[:, :steps]
    return out
