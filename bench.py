"""Benchmark of the B200 FDTD step on the 512x384x320 single-source
throughput workload (4 materials with third-order wall filters, 20 furniture
boxes, PML on two faces, band-limited noise source, 32 receivers).

One step = one time step of the whole grid. Prints one JSON line.
  value : interior cell-updates/s (Mcell/s) over K device-timed steps,
          inputs resident in HBM (three FP32 levels of 252 MB each, larger
          than L2, so no flush is needed between steps)
  e2e   : the same through the public API with the step's source samples
          copied host->device and the receiver samples device->host
  timeline_us: per-kernel start/end inside the replayed step (device clock,
          median over 32 steps after the timed runs)
  roofline: the step kernel's algorithmic bytes / its CUDA-event duration
  cpu_baseline: the reference's own kernels (oracle/_ref) on host cores

--impl reference times the reference's CPU kernels instead (rank 0 only).
Multi-GPU: one independent replica per rank (the path has no exchange
step), scaling "weak", value = all ranks' cell-updates / max-over-ranks time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None,
                    help="NX,NY,NZ: the same construction at another size (profiling captures)")
    ap.add_argument("--legs", default="device,e2e,timeline,roofline,parity,cpu",
                    help="comma list of device,e2e,timeline,roofline,parity,cpu")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c3rooms", "c5", "lms", "gemm"],
                    help="c2: the single-source throughput line (default); c3: batched secondary-path IRs/s; "
                         "c3rooms: 8 uneven rooms in one launch; "
                         "c5: the learned surrogate against the FDTD; lms: LMS impulse-response estimation "
                         "at the ie224-noise size; gemm: the surrogate's tcgen05 GEMM")
    ap.add_argument("--shard", action="store_true",
                    help="c3: shard the sources over the job's ranks and gather the receivers (the default "
                         "when the job has more than one rank)")
    ap.add_argument("--plan", default=None,
                    help="WxH[:DZ]: force the streaming plan (tile W x H cells, z-chunk depth DZ) instead of "
                         "letting the autotuner choose (profiling captures of one plan)")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16"],
                    help="field storage: fp32, or fp16 levels with per-level power-of-two scales")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples the SM clock and the clock-event (throttle) reasons of one GPU
    during the timed region: through NVML every ~2 ms (a timed region of a
    few milliseconds still gets samples), else nvidia-smi every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8 | 0x80, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []
        self.stop_flag = False
        self.max_mhz = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        h = None
        try:
            # the CUDA device's UUID: NVML numbers the GPUs of the machine,
            # which differs from CUDA's ordinal under CUDA_VISIBLE_DEVICES
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
        except Exception:
            h = None
        if h is None:
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        return pynvml, h

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self.stop_flag:
                    try:
                        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                             int(reasons(h))))
                    except Exception:
                        pass
                    time.sleep(0.002)
            self.th = threading.Thread(target=poll, daemon=True)
            self.th.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_flag = True
            self.th.join(timeout=2)
            sm = [v for v, _ in self.samples]
            reasons = sorted(k for k, bit in self.BITS.items() if any(r & bit for _, r in self.samples))
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def max_over_ranks(value, device="cpu"):
    """Maximum of a per-rank number over all ranks (the timing rule: a
    multi-GPU time is the slowest rank's); the value itself with one rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(cells_per_replica, steps, world, ms):
    """Whole-job cell-updates/s in millions for `world` independent replicas
    timed by the slowest one (weak scaling)."""
    return cells_per_replica * steps * world / (ms / 1e3) / 1e6


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference(cfg, steps=50, repeats=3, zs=64):
    """Times the reference's own kernels (oracle/_ref: leapfrog.cl, the 26
    lrs_*.cl launches, pml.cl when the workload has a PML, source.cl, mic.cl)
    with every host thread, on a zs-plane z-slab of the workload grid closed
    by a wall on top. The reference has one PML form, the whole-interior
    kernel of pml.cl:154-265 (its face profile only sets ksi), so a workload
    with PML slabs runs that kernel over every cell, its NDRange spread over
    the threads as a CPU OpenCL device runs it. Per-step time from the
    harness's step-loop timer (set-up excluded), median of `repeats` runs of
    `steps` steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import ancfield_b200.workloads as W
    nx, ny, nz = cfg.dims
    zs = min(zs, nz)
    vox = cfg.vox[:zs].copy()
    vox[-1] = np.where(vox[-1] == -1, 0, vox[-1])  # close the slab with a wall
    vox = W.close_gaps(vox)
    src = [((cfg.sources[0][0][0], cfg.sources[0][0][1], min(cfg.sources[0][0][2], zs - 3)),
            np.resize(cfg.sources[0][1], steps))]
    rcv = [(r[0], r[1], min(r[2], zs - 2)) for r in cfg.receivers]
    pml = cfg.pml_width if cfg.pml_width else 0
    ksi = W.ksi_arrays((nx, ny, zs), pml, cfg.pml_faces) if pml else None
    cells = (nx - 2) * (ny - 2) * (zs - 2)
    if oracle.available("ref", "f32"):
        impl, kind = "ref", "reference"
        loop_s = oracle.ref_timing(True)
    else:
        impl, kind, loop_s = "ora", "port", None
    times = []
    try:
        for _ in range(repeats):
            t = time.perf_counter()
            oracle.simulate((nx, ny, zs), vox, cfg.a, cfg.b, dx=cfg.dx, c=cfg.c, dt=cfg.dt, mode=0,
                            pml_width=pml, faces=63, ksi=ksi, sources=src, receivers=rcv, steps=steps, impl=impl)
            times.append(loop_s() if loop_s else time.perf_counter() - t)
    finally:
        if loop_s:
            oracle.ref_timing(False)  # parity users of the harness get the serial PML order back
    t = statistics.median(times)
    return {"value": cells * steps / t / 1e6, "unit": "Mcell-updates/s", "cores": os.cpu_count(),
            "kind": kind,
            "sample": "%dx%dx%d z-slab of the workload grid, %d steps, median of %d runs (%s s), step loop only; "
                      "the reference's kernels leapfrog + 26 LRS%s + source + mic in REF semantics, OpenMP %d "
                      "threads" % (nx, ny, zs, steps, repeats, ", ".join("%.2f" % v for v in times),
                                   " + its whole-interior PML kernel (width %d; the GPU arm updates the PML "
                                   "slabs only, FIXED scheme)" % pml if pml else "", os.cpu_count())}


def bench_c3(pkg, args):
    """Secondary-path identification: 16 wall-adjacent unit-impulse sources
    in a 256x192x160 room (16 receivers, 8192 steps). IRs/s = sources x
    receivers / wall seconds of the run (launches included, setup and
    graph instantiation excluded), for the plain single-source path (one
    source, per-step launches, no graph), the batched FP32 path (all 16
    sources as batch members, graph-replayed chunks) and the batched FP16
    path."""
    import torch
    W = pkg.workloads
    cfg = W.config_c3()
    steps = cfg.steps

    def run(batch, graphs, storage):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, batch=batch, graphs=graphs, storage=storage)
        sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
        for m in range(batch):
            for cell, sig in cfg.batch_sources[m]:
                sim.AddSourceCell(cell, sig, batch=m)
        for r in cfg.receivers:
            sim.AddMicCell(r)
        sim.prepare(steps)
        torch.cuda.synchronize()
        t = time.perf_counter()
        sim.Run(steps)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t
        out = sim.mics(batch=0)
        sim.close()
        return wall, out

    n_rcv = len(cfg.receivers)
    n_src = len(cfg.batch_sources)
    clocks = Clocks(0)
    clocks.start()
    t_plain, y_plain = run(1, 0, 0)
    t_b32, y_b32 = run(n_src, 1, 0)
    t_b16, y_b16 = run(n_src, 1, 1)
    clk = clocks.stop()
    v = n_src * n_rcv / t_b32
    nx, ny, nz = cfg.dims
    return {"metric": "secondary-path IRs/s", "value": v, "unit": "IRs/s", "n_gpus": 1, "steps": steps,
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "%dx%dx%d room (C1 construction, PML z+), %d wall-adjacent unit-impulse sources "
                                   "as batch members, %d receivers, %d steps" % (nx, ny, nz, n_src, n_rcv, steps),
                       "ir_error": "batched member 0 equals the single-source run bit for bit: %s"
                                   % bool(np.array_equal(y_plain, y_b32))},
            "paths": {"plain_single_source_fp32": {"irs_per_s": n_rcv / t_plain, "run_s": t_plain},
                      "batched_fp32": {"irs_per_s": v, "run_s": t_b32},
                      "batched_fp16": {"irs_per_s": n_src * n_rcv / t_b16, "run_s": t_b16,
                                       "member0_rel_l2_vs_fp32": float(np.linalg.norm(y_b16 - y_b32) /
                                                                       np.linalg.norm(y_b32))}},
            "clocks": clk}


def bench_c3_sharded(pkg, args, rank, world, local):
    """The batched C3 run with its 16 sources sharded over the job's ranks
    (one GPU each, no exchange during the run) and the receiver arrays
    gathered in source order (sharding.run_batch_sharded). IRs/s = all
    sources x receivers / the slowest rank's device-timed run (strong
    scaling: the total work is fixed)."""
    import torch
    W = pkg.workloads
    cfg = W.config_c3()
    steps = cfg.steps

    def make_sim(batch):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, batch=batch, device=local)
        sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
        for r in cfg.receivers:
            sim.AddMicCell(r)
        return sim

    clocks = Clocks(local)
    clocks.start()
    torch.distributed.barrier()
    y, run_s = pkg.sharding.run_batch_sharded(pkg, make_sim, cfg.batch_sources, steps, world, rank, device="cuda")
    clk = clocks.stop()
    t = max_over_ranks(run_s, "cuda")
    n_src, n_rcv = len(cfg.batch_sources), len(cfg.receivers)
    nx, ny, nz = cfg.dims
    return {"metric": "secondary-path IRs/s", "value": n_src * n_rcv / t, "unit": "IRs/s", "n_gpus": world,
            "steps": steps, "warmup": 0, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "%dx%dx%d room (C1 construction, PML z+), %d wall-adjacent unit-impulse sources "
                                   "sharded over %d GPUs as batch members, %d receivers, %d steps"
                                   % (nx, ny, nz, n_src, world, n_rcv, steps),
                       "parallelism": "sources sharded, receivers gathered (all_gather)",
                       "gathered": list(y.shape)},
            "ms_per_step": t * 1e3 / steps, "clocks": clk}


def bench_c3_rooms(pkg, args):
    """Uneven batch: 8 rooms (C1 construction, edges 96-256 cells, PML z+,
    one wall-adjacent unit impulse and 16 receivers each) packed into one
    grid and advanced by one simulation (one launch per kernel per step),
    against the same 8 rooms run one after another. Metric: room
    cell-updates/s (interior cells of the rooms x steps / wall seconds)."""
    import torch
    W = pkg.workloads
    cfg, parts, offsets = W.config_c3_rooms()
    steps = cfg.steps

    def make(vox, dims, srcs, rcvs):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt)
        sim.SetModel(pkg.Model.from_voxels(vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=W.ksi_arrays(dims, cfg.pml_width, cfg.pml_faces))
        for cell, sig in srcs:
            sim.AddSourceCell(cell, sig)
        for r in rcvs:
            sim.AddMicCell(r)
        sim.prepare(steps)
        return sim

    room_cells = sum((v.shape[0] - 2) * (v.shape[1] - 2) * (v.shape[2] - 2) for v, _, _ in parts)
    clocks = Clocks(0)
    clocks.start()
    sim = make(cfg.vox, cfg.dims, cfg.sources, cfg.receivers)
    torch.cuda.synchronize()
    t = time.perf_counter()
    sim.Run(steps)
    torch.cuda.synchronize()
    t_packed = time.perf_counter() - t
    y_packed = sim.mics()
    sim.close()
    t_seq, same = 0.0, True
    n_rcv = len(parts[0][2])
    for k, (vox, src, rcv) in enumerate(parts):
        nz, ny, nx = vox.shape
        s1 = make(vox, (nx, ny, nz), [(src, cfg.sources[k][1])], rcv)
        torch.cuda.synchronize()
        t = time.perf_counter()
        s1.Run(steps)
        torch.cuda.synchronize()
        t_seq += time.perf_counter() - t
        same &= bool(np.array_equal(s1.mics(), y_packed[k * n_rcv:(k + 1) * n_rcv]))
        s1.close()
    clk = clocks.stop()
    v = room_cells * steps / t_packed / 1e6
    gx, gy, gz = cfg.dims
    return {"metric": "Mcell-updates/s", "value": v, "unit": "Mcell-updates/s", "n_gpus": 1, "steps": steps,
            "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "8 uneven rooms (edges 96-256, C1 construction, PML z+) packed into one "
                                   "%dx%dx%d grid, one launch per kernel per step, %d steps" % (gx, gy, gz, steps),
                       "room_cells": room_cells, "packed_grid_cells": gx * gy * gz,
                       "rooms": [list(p[0].shape[::-1]) for p in parts],
                       "each_room_equals_its_own_run": same},
            "paths": {"packed_one_launch": {"run_s": t_packed, "mcell_per_s": v},
                      "rooms_one_after_another": {"run_s": t_seq,
                                                  "mcell_per_s": room_cells * steps / t_seq / 1e6}},
            "clocks": clk}


def bench_lms(pkg, args):
    """EstimateIr (anc_field_py/ancutil.py:24-37) at the size of
    examples/ie224-noise.py: 64000 taps, 10 s at 32 kHz (320000 samples), 16
    passes, mu 1e-4; synthetic band-limited noise through a decaying random
    64000-tap response. Metric: LMS sample updates per second (samples x
    passes / s). CPU baseline: the reference's loop (the bit-exact numpy
    restatement) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lms_oracle
    W = pkg.workloads
    N, steps, epochs, mu = 64000, 320000, 16, 1e-4
    rng = np.random.default_rng(21)
    x = 0.1 * W.band_noise(steps, 32000.0, seed=22).astype(np.float64)  # mu N var(x) = 0.064 < 1: stable
    h = rng.standard_normal(N) * np.exp(-np.arange(N) / 6000.0) * 0.05
    d = np.fft.irfft(np.fft.rfft(x, 2 * steps) * np.fft.rfft(h, 2 * steps), 2 * steps)[:steps]
    pkg.lms.estimate_ir(x[:4096], d[:4096], N, mu, epochs=1)  # warm-up
    clocks = Clocks(0)
    clocks.start()
    t = time.perf_counter()
    w = pkg.lms.estimate_ir(x, d, N, mu, epochs=epochs)
    wall = time.perf_counter() - t
    clk = clocks.stop()
    value = steps * epochs / wall
    # reference loop on a bounded sample: one pass over 3000 samples
    ns = 3000
    t = time.perf_counter()
    lms_oracle.estimate(x[:ns], d[:ns], N, mu, epochs=1)
    t_cpu = time.perf_counter() - t
    return {"metric": "LMS sample updates/s", "value": value, "unit": "samples/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "LMS impulse-response estimation, %d taps, %d samples, %d passes, mu %g "
                                   "(examples/ie224-noise.py size)" % (N, steps, epochs, mu),
                       "run_s": wall, "w_rel_l2_vs_true_response": float(np.linalg.norm(w - h) / np.linalg.norm(h))},
            "cpu_baseline": {"value": ns / t_cpu, "unit": "samples/s", "cores": 1, "kind": "port",
                             "sample": "the reference's sample-serial loop (numpy, bit-exact restatement), "
                                       "one pass over %d samples, %.1f s" % (ns, t_cpu)},
            "clocks": clk}


def bench_gemm(pkg, args):
    """The surrogate's tcgen05 BF16 GEMM (FP32 accumulation) on 8192 x 4096
    x 4096, device-timed with CUDA events, against the measured bf16 peak."""
    import torch
    M, N, K = 8192, 4096, 4096
    a = torch.randn(M, K, device="cuda").to(torch.bfloat16)
    b = torch.randn(N, K, device="cuda").to(torch.bfloat16)
    c = torch.empty(M, N, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        pkg.surrogate.gemm_bf16(a, b, c, st)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    # launches queued back to back (no host synchronisation between them)
    e0.record()
    for _ in range(reps):
        pkg.surrogate.gemm_bf16_async(a, b, c, status, st)
    e1.record()
    torch.cuda.synchronize()
    if int(status.item()):
        raise RuntimeError("GEMM pipeline wait timed out")
    ms = e0.elapsed_time(e1) / reps
    tf = 2.0 * M * N * K / (ms / 1e3) / 1e12
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        src = "measured"
    except Exception:
        peak, src = 1590.0, "fallback"
    err = float((c.double() - a.double() @ b.double().T).norm() / (a.double() @ b.double().T).norm())
    return {"metric": "GEMM TFLOP/s", "value": tf, "unit": "TFLOP/s", "n_gpus": 1, "steps": reps, "warmup": 3,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic", "config": {"workload": "C = A B^T, %dx%dx%d, BF16 in, FP32 accumulate" % (M, N, K),
                                            "rel_l2_vs_fp64": err},
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "peak_source": src, "unit": "TFLOP/s",
                         "frac": tf / peak, "traffic": None}}


def bench_c5(pkg, args):
    """The learned surrogates against the FDTD: the random-Fourier-feature
    readout over receiver positions (surrogate_workflow.run_field_readout:
    IRs at receiver positions the generating runs did not record, query
    pairs arriving after the runs, 1% L2 fallback bound) gives the line's
    value; the deep MLP over all ten inputs
    (surrogate_workflow.run_c5) is reported beside it."""
    import ancfield_b200.surrogate_workflow as SW
    ro = SW.run_field_readout(pkg, n_sets=4, n_src=8, n_query=96, n_val=96)
    r = SW.run_c5(pkg)
    r["fit"]["loss_curve"] = r["fit"]["loss_curve"][::4]
    after = ro["queries_after_runs"]
    return {"metric": "secondary-path IRs/s", "value": after["irs_per_s"]["readout_with_fallback"], "unit": "IRs/s",
            "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16", "data": "synthetic (FDTD-generated IRs)",
            "config": {"workload": "readout surrogate: %d wall sets x %d sources, %d-receiver grid, %d query pairs at "
                                   "new receiver positions arriving one at a time after the FDTD runs, 1%% L2 "
                                   "fallback bound; the FDTD answers a pair with one source's share of a batched run"
                                   % (ro["wall_sets"], ro["sources_per_set"], ro["grid_receivers"], ro["query_pairs"]),
                       "fdtd_irs_per_s": after["irs_per_s"]["fdtd"], "gain_over_fdtd": after["gain_over_fdtd"],
                       "gain_with_queries_known_before_runs": ro["gain_over_fdtd"]},
            "readout": ro, "mlp_surrogate": r}


def main():
    args = parse()
    rank, world, local = dist_env()
    import __graft_entry__ as ge
    pkg = ge.load()
    if args.workload == "c3" and args.impl == "b200" and (world > 1 or args.shard):
        import datetime
        import torch
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            line = bench_c3_sharded(pkg, args, rank, world, local)
            if rank == 0:
                print(json.dumps(line), flush=True)
        finally:
            torch.distributed.destroy_process_group()
        return
    if args.workload != "c2" and args.impl == "b200":
        if rank == 0:
            line = {"c3": bench_c3, "c3rooms": bench_c3_rooms, "c5": bench_c5, "lms": bench_lms,
                    "gemm": bench_gemm}[args.workload](pkg, args)
            print(json.dumps(line), flush=True)
        return
    W = pkg.workloads
    legs = set(args.legs.split(","))
    dims = tuple(int(v) for v in args.grid.split(",")) if args.grid else (512, 384, 320)
    # the source covers warm-up, the device leg and the e2e leg, so the e2e
    # leg's per-chunk source updates land in place
    cfg = W.config_c2(steps=max(args.warmup, 3) + 2 * max(args.steps, 1) + 8 * 1001 + 400 + TIMELINE_RUN,
                      dims=dims)
    nx, ny, nz = cfg.dims
    interior = (nx - 2) * (ny - 2) * (nz - 2)
    metric = "Mcell-updates/s"
    f16 = args.storage == "fp16"
    lvl_mb = interior * (2 if f16 else 4) / 1e6
    config = {"workload": "%dx%dx%d single-source %s (4 materials K=4, 20 boxes, PML x+/z+ "
                          "width 12, 32 receivers)" % (nx, ny, nz, "FP16-storage" if f16 else "FP32"),
              "grid": [nx, ny, nz], "interior_cells": interior, "mode": "FIXED", "storage": args.storage,
              "l2_flush": "not needed: three %.0f MB field levels exceed the 126 MB L2" % lvl_mb
              if 3 * lvl_mb > 126 else "none: the field levels fit in L2 (L2-resident workload)",
              "parallelism": "replicas" if world > 1 else "single"}

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_reference(cfg)
        line = {"metric": metric, "value": cb["value"], "unit": cb["unit"], "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "impl": "reference", "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config, "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    stream = torch.cuda.Stream()

    def make_sim(profile=0, graphs=1):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, device=local, profile=profile,
                             graphs=graphs, storage=1 if f16 else 0)
        sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
        sim.AddSourceCell(cfg.sources[0][0], cfg.sources[0][1])
        for r in cfg.receivers:
            sim.AddMicCell(r)
        sim.set_stream(stream.cuda_stream)
        return sim

    sim = make_sim()
    if args.plan:
        tile, _, dz = args.plan.partition(":")
        tw, th = (int(v) for v in tile.split("x"))
        sim.set_plan(tile=(tw, th), dz=int(dz) if dz else 0)
    K, Wm = args.steps, max(args.warmup, 3)
    if "device" not in legs:
        legs.add("device")
    sim.Run(Wm)
    # the online autotuner tries its streaming plans on full 200-step chunks;
    # let it finish before the timed run (these steps count as warm-up)
    for _ in range(8):
        if sim.info().tuned:
            break
        sim.Run(1001)
        Wm += 1001
    sim.prepare(K)  # graphs of the timed run's chunk lengths, built before the clock starts
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.Run(K)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    launches = sim.info().kernel_launches
    ms = max_over_ranks(ms, "cuda")
    value = replica_rate(interior, K, world, ms)

    line = {"metric": metric, "value": value, "unit": metric, "n_gpus": world, "steps": K, "warmup": Wm,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "plan": {"tile": [sim.info().tile_x, sim.info().tile_y, sim.info().tile_z],
                     "stream_blocks": sim.info().stream_blocks, "per_sm": sim.info().stream_per_sm,
                     "beside": bool(sim.info().stream_beside), "tuned": bool(sim.info().tuned)},
            "dtype": "f32", "data": "synthetic", "config": config, "gpu_launches": launches, "clocks": clk}
    info = sim.info()
    step_bytes, step_parts = step_algorithmic_bytes(info, 6.0 if f16 else 12.0, interior)
    if "e2e" in legs:
        line["e2e"] = e2e_leg(sim, cfg, K, interior, world, metric)
    if "timeline" in legs:
        line["timeline_us"] = timeline_leg(sim)
    sim.close()
    if "roofline" in legs:
        line["roofline"] = roofline_leg(make_sim, K, interior, 6.0 if f16 else 12.0,
                                        traffic_key=(tuple(cfg.dims), "fp16" if f16 else "fp32"), plan=info,
                                        step_parts=step_parts)
        peak = line["roofline"]["peak"]
        line["roofline"]["step"] = {"bytes": step_bytes, "parts": step_parts,
                                    "achieved": step_bytes / (ms / K / 1e3) / 1e9, "unit": "GB/s",
                                    "frac": step_bytes / (ms / K / 1e3) / 1e9 / peak}
    if "parity" in legs and rank == 0:
        line["parity"] = parity_leg(make_sim, cfg, info, f16)
    if rank == 0 and world == 1 and "cpu" in legs and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference(cfg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


TIMELINE_RUN = 240  # steps of the timeline leg (32 recorded)


def step_algorithmic_bytes(info, interior_bytes, interior):
    """Algorithmic bytes of one whole step: interior_bytes per interior cell
    (read p^n, read p^{n-1}, write p^{n+1}); per boundary point 4 B of index
    plus, per filter face, 8 K B of filter history read and 8 B of state
    written; 32 B per PML cell (auxiliary fields and psi read and written)."""
    K = info.ncoef
    faces = [1] * 6 + [2] * 12 + [3] * 8
    lrs = sum(int(info.group_counts[g]) * (4 + 8 * K * faces[g] + 8 * faces[g]) for g in range(26))
    pml = 32 * int(info.n_pml_cells)
    parts = {"interior": interior_bytes * interior, "boundary": lrs, "pml": pml}
    return float(sum(parts.values())), parts


PARITY_STEPS = 240


def parity_leg(make_sim, cfg, info, f16):
    """The error of this line's own configuration: the benchmark workload run
    again for PARITY_STEPS steps with the timed run's streaming plan, against
    the CPU restatement of the same scheme in FP32 (bit for bit expected) and
    in FP64 (receivers and the whole field; the receivers farther than
    PARITY_STEPS * lambda cells from the source are still silent)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    sim = make_sim()
    sim.set_plan(per_sm=info.stream_per_sm, dz=info.tile_z, beside=bool(info.stream_beside))
    sim.Run(PARITY_STEPS)
    got, field = sim.mics(), sim.field()
    sim.close()
    src = [(cfg.sources[0][0], cfg.sources[0][1][:PARITY_STEPS])]
    kw = dict(dx=cfg.dx, c=cfg.c, dt=cfg.dt, mode=1, pml_width=cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi,
              sources=src, receivers=cfg.receivers, steps=PARITY_STEPS, want_field=True)
    a, b = cfg.a.astype(np.float32), cfg.b.astype(np.float32)
    w32, f32 = oracle.simulate(cfg.dims, cfg.vox, a, b, precision="f16" if f16 else "f32", **kw)
    w64, f64 = oracle.simulate(cfg.dims, cfg.vox, a, b, precision="f64", **kw)

    def rl(x, y):
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))
    live = np.abs(w64).max(axis=1) > 0
    return {"steps": PARITY_STEPS, "plan": [info.stream_per_sm, info.tile_z, bool(info.stream_beside)],
            "oracle": "fp16-storage restatement" if f16 else "fp32 restatement",
            "receivers_bitexact": bool(np.array_equal(got, w32)), "field_bitexact": bool(np.array_equal(field, f32)),
            "receiver_rel_l2_vs_oracle": rl(got, w32), "receiver_rel_l2_vs_fp64": rl(got[live], w64[live]),
            "field_rel_l2_vs_fp64": rl(field, f64), "receivers_with_signal": int(live.sum())}


def timeline_leg(sim):
    """Per-kernel device timeline of 32 steps after the timed runs (same
    plan): median start and end of every kernel kind relative to its step's
    streaming-kernel start, and the median step period, in microseconds."""
    g0 = sim.info().steps_done + 100
    sim.set_timeline(g0, 32)
    sim.prepare(TIMELINE_RUN)
    sim.Run(TIMELINE_RUN)
    t = sim.timeline()
    sim.set_timeline(0, 0)
    if t.shape[0] == 0:
        return None
    base = t[:, 0, 0]
    out = {"step": round(float(np.median(np.diff(base))), 2)}
    for k, name in enumerate(sim.TIMELINE_KINDS):
        if np.all(np.isnan(t[:, k, 0])):
            continue
        out[name] = [round(float(np.nanmedian(t[:, k, 0] - base)), 2), round(float(np.nanmedian(t[:, k, 1] - base)), 2)]
    return out


def e2e_leg(sim, cfg, K, interior, world, metric):
    """Same metric through the public API: per step the source sample goes
    host->device and the receiver samples come back device->host."""
    import torch
    chunk = 200
    sig = np.ascontiguousarray(cfg.sources[0][1], dtype=np.float32)
    host_rcv = np.empty((len(cfg.receivers), chunk), np.float32)
    t_start = sim.info().steps_done
    sim.prepare(K)  # the receiver record for all K steps, so no chunk reallocates it
    sim.prepare(chunk)
    if K % chunk:
        sim.prepare(K % chunk)
    # one untimed read of the newest samples: the library's page-locked
    # staging for receiver reads is allocated on first use
    n0 = min(chunk, t_start)
    if n0 > 0:
        sim.mics_range(t_start - n0, t_start, out=host_rcv[:, :n0])
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    done = 0
    while done < K:
        n = min(chunk, K - done)
        t0 = t_start + done
        sim.update_source(0, t0, sig[(t0 % len(sig)):(t0 % len(sig)) + n]
                          if (t0 % len(sig)) + n <= len(sig) else np.resize(sig, n))
        sim.Run(n)
        sim.mics_range(t0, t0 + n, out=host_rcv[:, :n] if n == chunk else None)
        done += n
    e2e_s = time.perf_counter() - w0
    e2e_ms = max_over_ranks(e2e_s * 1e3, "cuda")
    return {"value": replica_rate(interior, K, world, e2e_ms), "unit": metric,
            "h2d_bytes_per_step": 4, "d2h_bytes_per_step": 4 * len(cfg.receivers)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# dominant kernel, from one single-pass ncu capture of that kernel on the
# full-size workload under the forced plan of the key (`--plan 64x16:8`,
# `--plan 128x8:8`, `--storage fp16 --plan 64x32:16`), keyed by grid,
# storage, tile and tail warps; the line
# reports it with traffic_source "ncu capture".
MEASURED_TRAFFIC = {((512, 384, 320), "fp32", (64, 16), False): ("interior_stream", 740.42e6),
                    ((512, 384, 320), "fp32", (128, 8), False): ("interior_stream", 724.12e6),
                    ((512, 384, 320), "fp16", (64, 32), False): ("interior_stream", 353.99e6)}


def roofline_leg(make_sim, K, interior, bytes_per_cell=12.0, traffic_key=None, plan=None, step_parts=None):
    """Roofline of the dominant kernel from per-launch CUDA events, with the
    timed run's streaming plan. The interior kernel moves bytes_per_cell per
    interior cell: read p^n, read p^{n-1}, write p^{n+1} (4-byte values, or
    2-byte FP16 storage); with tail warps it also does the boundary points
    (their bytes of the step's count) and the PML pressure update (16 of
    the 32 bytes a PML cell counts per step; the auxiliary half follows in
    its own kernel)."""
    psim = make_sim(profile=1, graphs=0)
    tail = bool(plan is not None and plan.stream_tail)
    if plan is not None:
        psim.set_plan(tile=(plan.tile_x, plan.tile_y), per_sm=plan.stream_per_sm, dz=plan.tile_z, tail=tail)
    psim.Run(min(K, 400) + 1)
    stats = psim.kernel_stats()
    psim.close()
    top = max(stats.items(), key=lambda kv: kv[1][1])
    name, (n_launch, tot_ms) = top
    avg_ms = tot_ms / max(n_launch, 1)
    step_kernel_bytes = bytes_per_cell * interior
    if tail and step_parts:
        step_kernel_bytes += step_parts["boundary"] + step_parts["pml"] / 2
    peak, peak_kind = peaks()
    achieved = step_kernel_bytes / (avg_ms / 1e3) / 1e9
    traffic = None
    key = traffic_key
    if key is not None and plan is not None:
        key = tuple(key) + ((plan.tile_x, plan.tile_y), tail)
    known = MEASURED_TRAFFIC.get(key)
    if known and known[0] == name:
        traffic = known[1]
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "peak_source": peak_kind,
            "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
            "traffic_source": "ncu capture of one full-size launch of this kernel (not measured by this run)"
            if traffic else None,
            "bytes_per_launch": step_kernel_bytes, "avg_launch_ms": avg_ms,
            "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in stats.items() if v[0]}}


if __name__ == "__main__":
    main()
