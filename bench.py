"""Benchmark of the velocity-stress time-stepping hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (default ``terrain_fault``): the curvilinear CGFDM configuration,
400 x 400 x 200 points, DH = 100 m, eight-hill terrain, perturbed layered
medium, 40 x 20 finite fault, 400 surface stations (cgfdm.configs).  A step
is one RK4 time step of the whole grid.  Metric: Mpts*step/s, interior
points x steps / seconds.

Our arm: W untimed steps, then K steps timed with CUDA events on the
session's stream (barrier + device sync on both sides, max over ranks);
inputs (7.3 GB of model and wavefield) are resident and larger than L2.
``e2e`` is the same metric through the C ABI from host files: create the
session from the run directory (model build, host->device copies), run K
steps, read the station traces back, destroy.  ``roofline`` uses the mean
device time of one fused stage launch (events around each launch) and the
algorithmic bytes of a launch.  ``cpu_baseline`` runs the reference's own
CPU build (oracle/_ref/cgfdm_ref) on a sample of the workload on the host
cores.

Reference arm (--impl reference): the reference's CPU build, one process per
host core on the sample grid, timed steps differenced against a run with
only the warm-up steps so set-up is excluded.

With N > 1 (torchrun), every rank advances its own replica of the workload
on its own GPU; there is no exchange between ranks ("scaling": "weak").
"""

from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cgfdm3d-eqr-sc_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "Mpts*step/s"
WORK = os.environ.get("CGFDM_BENCH_DIR", os.path.join(tempfile.gettempdir(), "cgfdm_bench"))
SAMPLE_GRID = (160, 160, 100)
SAMPLE_GRID_SC = (48, 48, 40)    # the reference's SCFDM CPU path is ~50x slower per point


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ME-AWENO arithmetic per interior point and step (54 WENO5 reconstructions
# of about 90 flops and 4 divides, Lax-Friedrichs fluxes, flux differences
# with their corrections, three TVD stages): about 19.4 kflop.
SC_FLOP_PER_PT_STEP = 19.4e3


def fp32_peak_tflops():
    """FP32 (non-tensor) peak: 148 SMs x 128 FP32 lanes x 2 flop x the
    maximum SM clock.  Nominal: no measured FP32 figure is provided."""
    mhz = 1965.0
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def traffic_ratio():
    """DRAM traffic of the stage kernel over its algorithmic bytes, from the
    committed ncu summary (profiles/cg_stage_traffic.txt), or None."""
    path = os.path.join(ROOT, "profiles", "cg_stage_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_traffic_over_algorithmic:"):
            return float(line.split(":", 1)[1])
    return None


def adj_traffic_per_point_stage():
    """DRAM bytes per point and stage of the adjoint kernels, from the
    committed ncu summary (profiles/adj_stage_traffic.txt), or None."""
    path = os.path.join(ROOT, "profiles", "adj_stage_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_point_stage:"):
            return float(line.split(":", 1)[1])
    return None


def make_workload(name, steps, directory):
    from cgfdm import cases, configs

    marker = os.path.join(directory, f".done_{steps}")
    if os.path.exists(marker):
        return directory
    if os.path.exists(directory):
        shutil.rmtree(directory)
    if name == "terrain_fault":
        configs.terrain_fault(directory, steps=steps)
    elif name.startswith("terrain_fault_"):
        # terrain_fault_<nx>x<ny>x<nz>[_pml<n>]
        parts = name[len("terrain_fault_"):].split("_")
        nx, ny, nz = (int(v) for v in parts[0].split("x"))
        npml = int(parts[1][3:]) if len(parts) > 1 else 12
        configs.terrain_fault(directory, steps=steps, NX=nx, NY=ny, NZ=nz, nPML=npml)
    elif name == "aweno_basin":
        configs.aweno_basin(directory, steps=steps)
    elif name.startswith("aweno_basin_"):
        nx, ny, nz = (int(v) for v in name.split("_")[-1].split("x"))
        configs.aweno_basin(directory, steps=steps, NX=nx, NY=ny, NZ=nz)
    elif name == "halfspace":
        cases.write_case(configs.halfspace(steps=steps), directory)
    else:
        raise SystemExit(f"unknown workload {name}")
    open(marker, "w").close()
    return directory


def workload_desc(name):
    if name == "terrain_fault":
        return ("terrain_fault: CGFDM RK4, 400x400x200 (32.0 Mpts interior), DH=100 m, 8-hill terrain, "
                "4 layers + half-space with +-3% correlated perturbation, 40x20 finite fault, 400 stations, "
                "12-layer PML on 5 faces, FP32")
    if name == "halfspace":
        return "halfspace: CGFDM RK4, 128x128x96, DH=100 m, homogeneous half-space, Mxy point source, 16 stations"
    if name == "aweno_basin":
        return ("aweno_basin: ME-AWENO (SCFDM) TVD-RK3, 512x512x256 (67.1 Mpts interior), DH=50 m, 8-hill terrain, "
                "6 dipping planar interfaces (Vs 1200-3600 m/s) + ellipsoidal basin Vs=400 m/s, 5 Hz Ricker point "
                "source, 100 stations, exponential sponge, characteristic free surface, FP32")
    return name


def fp64_error(run_dir, steps, device, options=None):
    """Error of an FP32 run (the session, as benched) against the FP64 run
    of the same model (cgfdm_run_precise, bits 64) after ``steps`` steps:
    relative L2 of the station velocity traces and of the final wavefield.
    The station figure is None while the waves have not reached the
    stations (their FP64 peak below 1e-3 of the wavefield's peak velocity):
    a ratio of rounding noise to near-zero traces says nothing."""
    import numpy as np

    from cgfdm import Session

    with Session(run_dir, options=options, device=device) as s:
        steps = min(steps, s.info.NT)
        t0 = time.perf_counter()
        s.run(steps)
        t32 = time.perf_counter() - t0
        st32 = s.stations()[:, :steps, :3].astype(np.float64)
        w32 = s.wavefield().astype(np.float64)
        t0 = time.perf_counter()
        st64, _, w64 = s.run_precise(steps, bits=64, wavefield=True)
        t64 = time.perf_counter() - t0
    st64 = st64[:, :, :3]

    def rel(a, b):
        nb = float(np.linalg.norm(b))
        return float(np.linalg.norm(a - b)) / nb if nb > 0 else None

    w64 = np.asarray(w64, dtype=np.float64)
    vpeak = float(np.abs(w64[..., :3]).max())   # [z][y][x][field]: velocities are fields 0-2
    reached = float(np.abs(st64).max()) >= 1e-3 * vpeak if vpeak > 0 else False
    return {"steps": steps, "stations_velocity_rel_l2": rel(st32, st64) if reached else None,
            "stations_reached": reached, "wavefield_rel_l2": rel(w32, w64),
            "against": "cgfdm_run_precise bits=64: the same time loop, state and arithmetic in FP64",
            "options": options, "fp32_run_s": t32, "fp64_run_s": t64}


def is_scfdm(name):
    return name.startswith("aweno")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self

        def reader():
            for line in self.proc.stdout:
                self.samples.append([v.strip() for v in line.split(",")])

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        smax = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ------------------------------------------------------------ CPU baseline
def pml_point_fraction(nx, ny, nz, npml):
    """Share of the grid's points inside the PML (x and y faces both sides,
    the bottom z face; the top is the free surface)."""
    return 1.0 - max(nx - 2 * npml, 0) * max(ny - 2 * npml, 0) * max(nz - npml, 0) / (nx * ny * nz)


def sample_npml(sample, full=(400, 400, 200), npml_full=12):
    """PML thickness of the CPU sample grid whose PML-point share is closest
    to the full workload's: the reference's per-point cost is higher inside
    the PML, so a sample with a thicker relative PML would understate its
    rate on the full grid."""
    f_full = pml_point_fraction(*full, npml_full)
    return min(range(1, npml_full + 1), key=lambda n: abs(pml_point_fraction(*sample, n) - f_full))


def cpu_reference_rate(name, warmup_steps, timed_steps, procs):
    """Reference CPU build on the sample grid: `procs` concurrent processes,
    wall time of (warmup + timed) steps minus (warmup) steps, aggregate rate."""
    import refrun

    if not refrun.available("SCFDM" if is_scfdm(name) else "CGFDM"):
        return None, "reference CPU build (oracle/_ref) not built"
    sc = is_scfdm(name)
    nx, ny, nz = SAMPLE_GRID_SC if sc else SAMPLE_GRID
    npml = None
    if name.startswith("terrain_fault"):
        npml = sample_npml((nx, ny, nz))
        sample_name = f"terrain_fault_{nx}x{ny}x{nz}_pml{npml}"
    elif sc:
        sample_name = f"aweno_basin_{nx}x{ny}x{nz}"
    else:
        sample_name = name
    scheme = "SCFDM" if sc else "CGFDM"
    base = os.path.join(WORK, "cpu_sample")
    runs = {}
    for nt in (warmup_steps, warmup_steps + timed_steps):
        d = make_workload(sample_name, nt, os.path.join(base, f"{sample_name}_{nt}"))
        copies = []
        for p in range(procs):
            c = os.path.join(base, f"run_{nt}_{p}")
            if os.path.exists(c):
                shutil.rmtree(c)
            os.makedirs(os.path.join(c, "output"))
            for f in os.listdir(d):
                src = os.path.join(d, f)
                if os.path.isfile(src):
                    os.symlink(src, os.path.join(c, f))
            copies.append(c)
        t0 = time.perf_counter()
        ps = [subprocess.Popen(["taskset", "-c", str(p % os.cpu_count()), refrun.ref_binary(scheme)], cwd=c,
                               stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for p, c in enumerate(copies)]
        rcs = [p.wait() for p in ps]
        runs[nt] = time.perf_counter() - t0
        if any(rcs):
            return None, f"reference CPU build failed with exit codes {sorted(set(rcs))}"
    dt = runs[warmup_steps + timed_steps] - runs[warmup_steps]
    if dt <= 0:
        return None, "reference CPU sample timing below its set-up noise (increase --steps)"
    pts = nx * ny * nz
    rate = procs * pts * timed_steps / max(dt, 1e-9) / 1e6
    sample = (f"reference CPU build ({scheme}, g++ {'-O3' if sc else '-O2'}, single-threaded as shipped), "
              f"{procs} concurrent processes pinned "
              f"one per core, each on the {nx}x{ny}x{nz} sub-grid of the workload (same generators), "
              f"{timed_steps} steps timed as wall({warmup_steps + timed_steps} steps) - wall({warmup_steps} steps)")
    out = {"value": rate, "unit": METRIC, "cores": procs, "kind": "reference", "sample": sample}
    if npml is not None:
        out["sample"] += f", {npml}-layer PML so that its PML-point share matches the 400x400x200 workload's"
        out["pml_point_fraction"] = {"sample": pml_point_fraction(nx, ny, nz, npml),
                                     "workload": pml_point_fraction(400, 400, 200, 12),
                                     "sample_with_12_layers": pml_point_fraction(nx, ny, nz, 12)}
    return out, None


def max_over_ranks(value, dist, device):
    """Largest per-rank value over all ranks (the value itself without a
    process group).  Timings of a multi-GPU run are the slowest rank's."""
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------- batches
def bench_batch(args, world, rank, local_rank):
    """``--workload batchN``: N independent CGFDM shots of uneven sizes
    (cgfdm.configs.batch_shots: 64-256 x 64-256 x 64-128, layered media,
    terrain up to 1 km, random moment tensors, 32 stations each) advanced
    together, one persistent stage launch per RK stage, 8 steps per graph
    replay.  Also times each shot alone for comparison.  One GPU."""
    import torch
    from cgfdm import Batch, Session, configs

    n = int(args.workload[len("batch"):] or 32)
    total = args.warmup + 2 * args.steps + 24  # batched steps, then the same number per shot alone
    root = os.path.join(WORK, f"{args.workload}_{total}")
    marker = os.path.join(root, ".done")
    if not os.path.exists(marker):
        if os.path.exists(root):
            shutil.rmtree(root)
        configs.batch_shots(root, n=n, steps=total)
        open(marker, "w").close()
    dirs = sorted(os.path.join(root, d) for d in os.listdir(root) if d.startswith("shot_"))
    sessions = [Session(d, options=session_options(args), device=local_rank) for d in dirs]
    pts = sum(s.info.nx * s.info.ny * s.info.nz for s in sessions)
    algo = sum(s.info.algo_bytes_per_step for s in sessions)
    b = Batch(sessions)
    b.run(args.warmup)
    # the default decomposition, then the autotuner's choice (timed below)
    ms_default = b.run_timed(8)
    # (FP16 storage: no autotuner, whose trials restore a device copy of the state)
    tuned = b.autotune(3) if args.storage == "fp32" else (0, None, ms_default / 8)
    tuned_tile = b.stage_tile()
    b.run(1)
    torch.cuda.synchronize(local_rank)
    with ClockSampler(local_rank) as clk:
        ms = b.run_timed(args.steps)
    b.close()
    # each shot alone, same number of steps
    alone_ms = 0.0
    for s in sessions:
        alone_ms += s.run_timed(args.steps)
    for s in sessions:
        s.close()
    # end to end: run directories on disk -> sessions -> batch -> traces on the host
    t0 = time.perf_counter()
    ss = [Session(d, device=local_rank) for d in dirs]
    b2 = Batch(ss)
    b2.run(args.steps)
    st_bytes = sum(s.stations().nbytes for s in ss)
    h2d = sum(s.info.h2d_bytes for s in ss)
    b2.close()
    for s in ss:
        s.close()
    e2e_s = time.perf_counter() - t0
    value = pts * args.steps / (ms * 1e-3) / 1e6
    hbm_peak, peak_kind = peaks()
    achieved = algo * args.steps / (ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "scheme": "CGFDM",
        "storage": ("fp32" if args.storage == "fp32" else
                    "fp16 stage/accumulator deltas (per-field scales) + fp32 step state; f32 arithmetic"),
        "config": {"workload": f"{n} CGFDM shots of uneven sizes (64-256 x 64-256 x 64-128, DH=100 m), layered "
                               "media, terrain <= 1 km, random moment tensors, 32 stations each, one persistent "
                               "stage launch per RK stage for all shots, 8-step CUDA graphs",
                   "points": pts, "shots": n,
                   "alone_Mpts_step_s": pts * args.steps / (alone_ms * 1e-3) / 1e6,
                   "autotuned": {"tile": f"32x{tuned_tile}", "kchunk": tuned[0], "ctas": tuned[1],
                                 "trial_ms_per_step": tuned[2],
                                 "default_ms_per_step": ms_default / 8},
                   "l2": "inputs larger than L2", "parallelism": "batch x1"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "peak_kind": peak_kind, "traffic": None,
                     "kernel": "k_cg_stage (batched; whole step incl. sources and stations)"},
        "e2e": {"value": pts * args.steps / e2e_s / 1e6, "unit": METRIC, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": st_bytes / args.steps, "seconds": e2e_s},
        "gpu_launches": int(args.steps * (4 + 2 * n)),
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- adjoint
ADJ_BYTES_PER_POINT_STAGE = 4 * (9 + 9 + 9 + 12 + 18 + 9 + 6)


def shots_of_rank(items, world, rank):
    """The shots a rank computes: every world-th one from its rank on
    (independent units; no exchange while they run)."""
    return list(items)[rank::world]


def sum_over_ranks(array, dist, device):
    """Sum of a gradient volume over all ranks (the array itself without a
    process group): the multi-shot gradient's one collective, an all-reduce
    of the three gradient volumes after every rank has finished its shots."""
    import numpy as np
    import torch

    if not dist:
        return array
    t = torch.from_numpy(np.ascontiguousarray(array, np.float32)).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def bench_adjoint(args, world, rank, local_rank):
    """``--workload adjoint[_STEPS[_NXxNYxNZ]]``: the misfit gradient with respect to
    Vp, Vs and rho (cgfdm_gradient) on the 192 x 192 x 128 layered model
    with a 2 km, +8 % Vs ball in the true medium (cgfdm.configs.adjoint_shots):
    four shots (2 Hz Ricker point sources), 64 surface stations, NT = 2000
    steps each (or STEPS; with a grid size, one shot of that size),
    checkpoints every --checkpoint-every steps (100).  The observed data
    are the true medium's seismograms; the gradient is taken at the starting
    medium (no ball) and summed over the shots.  Reports gradient throughput
    (shots x points x NT / seconds) and the adjoint/forward cost: wall time
    of the gradient over that of a forward run of the same shot (both from
    step 0, medium set, traces read back).  With N ranks (torchrun) every
    rank takes every N-th shot; the gradient volumes are then summed with one
    all-reduce (NCCL) and times are the slowest rank's.  --steps/--warmup
    do not apply (a shot is one unit)."""
    import numpy as np
    import torch
    from cgfdm import Session, configs

    parts = args.workload.split("_")
    NT = int(parts[1]) if len(parts) > 1 else 2000
    NX, NY, NZ = (int(v) for v in parts[2].split("x")) if len(parts) > 2 else (192, 192, 128)
    DH = 100.0
    n_shots = 4 if len(parts) <= 2 else 1
    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    root = os.path.join(WORK, f"adjoint_{NT}_{NX}x{NY}x{NZ}_{n_shots}")
    marker = os.path.join(root, ".done")
    if rank == 0 and not os.path.exists(marker):
        if os.path.exists(root):
            shutil.rmtree(root)
        configs.adjoint_shots(root, steps=NT, NX=NX, NY=NY, NZ=NZ, n_shots=n_shots)
        open(marker, "w").close()
    if dist:
        dist.barrier()
    all_dirs = sorted(os.path.join(root, d) for d in os.listdir(root) if d.startswith("shot_"))
    dirs = shots_of_rank(all_dirs, world, rank)
    true = configs.adjoint_layers(NX, NY, NZ, DH, True)
    start = configs.adjoint_layers(NX, NY, NZ, DH, False)
    K = args.checkpoint_every
    opts = json.dumps({"adjointStoreSegments": args.store_segments}) if args.store_segments else None
    t_fwd = t_grad = 0.0
    phases = np.zeros(3)
    grad_sum = None
    J_sum = 0.0
    dev_gb = 0.0
    with ClockSampler(local_rank) as clk:
        for d in dirs:
            s = Session(d, options=opts, device=local_rank)
            info = s.info
            s.set_medium(true)
            s.run(info.NT)
            obs = s.stations()[:, :, :3].copy()
            # forward run alone (second forward of the shot: warm)
            s.set_medium(start)
            torch.cuda.synchronize(local_rank)
            t0 = time.perf_counter()
            s.run(info.NT)
            s.stations()
            torch.cuda.synchronize(local_rank)
            t_fwd += time.perf_counter() - t0
            s.set_medium(start)
            torch.cuda.synchronize(local_rank)
            t0 = time.perf_counter()
            J, g = s.gradient(obs, K)
            torch.cuda.synchronize(local_rank)
            t_grad += time.perf_counter() - t0
            phases += np.array(s.gradient_profile())
            J_sum += J
            grad_sum = g if grad_sum is None else grad_sum + g
            dev_gb = info.device_bytes / 1e9
            s.close()
    # one collective: the gradient volumes summed over the ranks' shots;
    # times are the slowest rank's
    dev = f"cuda:{local_rank}"
    if dist:
        dist.barrier()
    grad_sum = sum_over_ranks(grad_sum if grad_sum is not None else np.zeros((3, NZ, NY, NX), np.float32), dist, dev)
    J_sum = float(sum_over_ranks(np.array([J_sum], np.float32), dist, dev)[0])
    t_fwd = max_over_ranks(t_fwd, dist, dev)
    t_grad = max_over_ranks(t_grad, dist, dev)
    n = len(all_dirs)
    steps_adj = max(1, len(dirs)) * NT
    adj_ms_step = phases[2] / steps_adj
    pts = NX * NY * NZ
    algo = ADJ_BYTES_PER_POINT_STAGE * 4 * pts
    achieved = algo / (adj_ms_step * 1e-3) / 1e9
    hbm_peak, peak_kind = peaks()
    # the gradient should see the ball: its Vs gradient there against elsewhere
    kk, jj, ii = np.meshgrid(np.arange(NZ), np.arange(NY), np.arange(NX), indexing="ij")
    zc = (NZ - 1) - 0.4 * NZ
    inside = np.sqrt((ii - (NX - 1) / 2) ** 2 + (jj - (NY - 1) / 2) ** 2 + (kk - zc) ** 2) * DH < 2000.0
    gvs = grad_sum[1]
    line = {
        "metric": METRIC, "value": n * pts * NT / t_grad / 1e6, "unit": METRIC, "n_gpus": world, "steps": NT,
        "warmup": 0, "ms_per_step": t_grad * 1e3 / steps_adj, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "scheme": "CGFDM",
        "config": {"workload": f"adjoint: CGFDM misfit gradient w.r.t. Vp, Vs, rho, {NX}x{NY}x{NZ}, DH=100 m, "
                               f"4 layers + half-space, true model with a 2 km-radius +8% Vs ball, {n} shot(s) "
                               f"(2 Hz Ricker point sources), 64 surface stations, checkpoint every {K} steps, FP32",
                   "points": pts, "shots": n, "NT": NT, "checkpoint_every": K,
                   "l2": "inputs larger than L2 (%.1f GB resident per session)" % dev_gb,
                   "parallelism": f"shots over {world} rank(s), gradient volumes all-reduced"},
        "adjoint_over_forward": t_grad / t_fwd,
        "forward_s": t_fwd, "gradient_s": t_grad,
        "phases_ms": {"forward_with_checkpoints": phases[0], "segment_reruns_storing_rhs": phases[1],
                      "adjoint_steps": phases[2]},
        "misfit": J_sum,
        "grad_vs_ball_over_outside": float(np.abs(gvs[inside]).mean() / max(np.abs(gvs[~inside]).mean(), 1e-300)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                     "traffic": (adj_traffic_per_point_stage() or 0) * 4 * pts or None,
                     "traffic_source": "ncu bytes per point and stage on adjoint_24_144x144x112 x points x 4 stages",
                     "kernel": "k_adj_pre + k_adj_gather (one adjoint step = 4 stages x 2 launches)",
                     "algo_bytes_per_step": algo, "mean_step_ms": adj_ms_step},
        "e2e": {"value": n * pts * NT / t_grad / 1e6, "unit": METRIC,
                "h2d_bytes_per_step": (start.nbytes + n * 0) / NT, "d2h_bytes_per_step": grad_sum.nbytes / NT / n,
                "path": "cgfdm_set_medium + cgfdm_gradient (host observed data in, host gradient out)"},
        "gpu_launches": int(n * NT * (6 + 6 + 9)),
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------- main
def bench_parts(args, world, rank, local_rank):
    """The workload decomposed into parts, all on this GPU: every phase of a
    step on every part, halos refreshed between phases (stored by the stage
    kernels with --exchange fused).  The parts synchronise with the host
    after every phase, so the time is wall clock around the timed steps
    (after a device synchronisation), against the same workload as one
    session, device-timed."""
    import torch

    from cgfdm import Session, domain

    if world != 1:
        print(json.dumps({"metric": METRIC, "unavailable": "--parts runs every part on one GPU; N = 1 only"}))
        return
    parts = tuple(int(x) for x in args.parts.split(","))
    total = args.warmup + args.steps + 8
    d = os.path.join(WORK, f"{args.workload}_{total}")
    make_workload(args.workload, total, d)
    s = Session(d, device=local_rank)
    pts = s.info.nx * s.info.ny * s.info.nz
    s.run(args.warmup)
    ms_one = s.run_timed(args.steps)
    s.close()
    dom = domain.LocalDomain(d, parts, device=local_rank, fused=args.exchange == "fused")
    dom.step(args.warmup)
    torch.cuda.synchronize(local_rank)
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        dom.step(args.steps)
        torch.cuda.synchronize(local_rank)
        wall = time.perf_counter() - t0
    nparts = len(dom.ps)
    dom.close()
    value = pts * args.steps / wall / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall * 1e3 / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "scheme": "CGFDM",
        "timing": "wall clock around the timed steps (the parts synchronise with the host after every phase)",
        "config": {"workload": workload_desc(args.workload), "points": pts, "parts": parts,
                   "exchange": args.exchange, "l2": "inputs larger than L2",
                   "parallelism": f"{nparts} parts on one GPU",
                   "one_session_Mpts_step_s": pts * args.steps / (ms_one * 1e-3) / 1e6},
        "gpu_launches": int(args.steps * nparts * (4 + 1)),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


FULL_STEPS = {"terrain_fault": 3000, "aweno_basin": 4000, "halfspace": 1000}


def session_options(args):
    o = {}
    if args.storage != "fp32":
        o["storage"] = args.storage
    if args.pipeline != "split":
        o["stagePipeline"] = args.pipeline
    if getattr(args, "tile", 0):
        o["stageTile"] = args.tile
    return json.dumps(o) if o else None


def bench_fp64_check(args, local_rank):
    """One JSON line: the benched path (FP32 or mixed storage) against the
    FP64 run over the workload's steps (seismogram and wavefield relative L2)."""
    steps = args.fp64_check
    if steps < 0:
        steps = args.full_steps or FULL_STEPS.get(args.workload, 1000)
    d = os.path.join(WORK, f"{args.workload}_{steps}")
    make_workload(args.workload, steps, d)
    e = fp64_error(d, steps, local_rank, session_options(args))
    print(json.dumps({"metric": "err_vs_fp64", "workload": workload_desc(args.workload), "storage": args.storage,
                      **e}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="terrain_fault")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--checkpoint-every", type=int, default=100, help="adjoint workload: checkpoint interval")
    ap.add_argument("--store-segments", type=int, default=0,
                    help="adjoint workload: cap on segments stored during the first forward (0: memory decides)")
    ap.add_argument("--parts", default="",
                    help="CGFDM workloads, one GPU: run the grid as PX,PY,PZ parts (domain decomposition)")
    ap.add_argument("--exchange", default="fused", choices=["fused", "explicit"],
                    help="with --parts: halos stored by the stage kernels, or packed and copied per phase")
    ap.add_argument("--fp64-check", type=int, default=0, metavar="STEPS",
                    help="only measure the FP32 run's error against the FP64 run over STEPS steps (-1: the "
                         "workload's full length) and print it as one JSON line")
    ap.add_argument("--full-steps", type=int, default=0,
                    help="with --fp64-check -1: the workload's full length (default: 3000 for terrain_fault, "
                         "4000 for aweno_basin, 1000 for halfspace)")
    ap.add_argument("--pipeline", default="split", choices=["ring", "split"],
                    help="CGFDM FP32 stage kernel: the current plane's halo box with interior column boxes for the "
                         "z window (default), or six full halo planes in a ring")
    ap.add_argument("--tile", type=int, default=0, choices=[0, 4, 8],
                    help="CGFDM: rows of the stage kernel's 32-column tiles (0: the session's default, 8 on the "
                         "FP32 split pipeline, 4 on the ring)")
    ap.add_argument("--kchunk", type=int, default=0,
                    help="CGFDM: z planes per work item of the stage kernel (0: the session's default)")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "fp16"],
                    help="wavefield storage of the CGFDM session: FP32, or FP16 stage and accumulator deltas "
                         "from the FP32 step state (mixed precision)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        procs = min(os.cpu_count() or 1, 32)
        timed = max(2, min(args.steps, 4))   # one step is within the set-up time's noise
        cb, why = cpu_reference_rate(args.workload, args.warmup if args.warmup <= 4 else 2, timed, procs)
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        line = {"metric": METRIC, "value": cb["value"], "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
                "steps": timed, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": workload_desc(args.workload),
                           "sample_grid": "x".join(map(str, SAMPLE_GRID_SC if is_scfdm(args.workload) else SAMPLE_GRID))},
                "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                                            "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch

    if args.fp64_check:
        return bench_fp64_check(args, local_rank)
    if args.parts:
        return bench_parts(args, world, rank, local_rank)
    if args.workload.startswith("batch"):
        return bench_batch(args, world, rank, local_rank)
    if args.workload.startswith("adjoint"):
        return bench_adjoint(args, world, rank, local_rank)

    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from cgfdm import Session

    total = args.warmup + args.steps + 8
    d = os.path.join(WORK, f"{args.workload}_{total}")
    if rank == 0:
        make_workload(args.workload, total, d)
    if dist:
        dist.barrier()

    # ---- device-timed leg: inputs resident on the GPU
    t_first = time.perf_counter()
    s = Session(d, options=session_options(args), device=local_rank)
    first_create_s = time.perf_counter() - t_first   # the process's first session (includes one-time costs)
    if args.kchunk:
        s.set_tiling(args.kchunk, s.tiling()[1])
    tiling = s.tiling() + (s.stage_tile(),) if not is_scfdm(args.workload) else None
    info = s.info
    pts = info.nx * info.ny * info.nz
    s.run(args.warmup)
    torch.cuda.synchronize(local_rank)
    if dist:
        dist.barrier()
    l0 = s.info.kernel_launches
    with ClockSampler(local_rank) as clk:
        ms = s.run_timed(args.steps)
    launches = s.info.kernel_launches - l0
    torch.cuda.synchronize(local_rank)
    if dist:
        dist.barrier()
    ms_max = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    stage_ms = s.profile_stages(8)
    algo_step = info.algo_bytes_per_step
    algo_launch = algo_step / info.stage_kernels_per_step
    s.close()

    # ---- end-to-end leg: run directory on disk -> C ABI -> stations on the host
    t0 = time.perf_counter()
    s2 = Session(d, options=session_options(args), device=local_rank)
    if args.kchunk:
        s2.set_tiling(args.kchunk, s2.tiling()[1])
    t1 = time.perf_counter()
    s2.run(args.steps)
    t2 = time.perf_counter()
    st = s2.stations()
    t3 = time.perf_counter()
    i2 = s2.info
    create_prof = s2.create_profile()
    t4 = time.perf_counter()
    s2.close()
    t5 = time.perf_counter()
    e2e_s = t5 - t0
    e2e_legs = {"create_s": t1 - t0, "run_s": t2 - t1, "stations_s": t3 - t2, "destroy_s": t5 - t4}
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local_rank}")

    value = world * pts * args.steps / (ms_max * 1e-3) / 1e6
    hbm_peak, peak_kind = peaks()
    achieved = algo_launch / (stage_ms * 1e-3) / 1e9
    tr = traffic_ratio()
    sc = is_scfdm(args.workload)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "storage": ("fp32" if args.storage == "fp32" else
                    "fp16 stage/accumulator deltas (per-field scales) + fp32 step state; f32 arithmetic"),
        "scheme": "SCFDM" if sc else "CGFDM",
        "config": {"workload": workload_desc(args.workload), "points": pts, "DT": info.DT,
                   "stage_tiling": ({"tile": f"32x{tiling[2]}", "kchunk": tiling[0], "ctas": tiling[1],
                                     "pipeline": "ring" if args.storage == "fp16" else args.pipeline}
                                    if tiling else None),
                   "l2": "inputs larger than L2 (model + wavefield %.1f GB resident)" % (info.device_bytes / 1e9),
                   "parallelism": f"replicas x{world}"},
        "hbm_gbs_algorithmic": algo_step * args.steps / (ms_max * 1e-3) / 1e9,
        "roofline": ({"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                      "frac": achieved / hbm_peak, "peak_kind": peak_kind,
                      "traffic": (tr * algo_launch if tr else None),
                      "traffic_source": "ncu ratio on terrain_fault_256x256x128 x algorithmic bytes of this launch",
                      "kernel": "k_cg_stage",
                      "algo_bytes_per_launch": algo_launch, "mean_launch_ms": stage_ms}
                     if not sc else
                     {"bound": "fp32", "unit": "TFLOP/s",
                      "achieved": SC_FLOP_PER_PT_STEP / 3 * pts / (stage_ms * 1e-3) / 1e12,
                      "peak": fp32_peak_tflops(), "peak_kind": "nominal (148 SMs x 128 lanes x 2 x max SM clock)",
                      "frac": SC_FLOP_PER_PT_STEP / 3 * pts / (stage_ms * 1e-3) / 1e12 / fp32_peak_tflops(),
                      "algo_flop_per_pt_step": SC_FLOP_PER_PT_STEP, "traffic": None,
                      "kernel": "k_sc_tile x3 (one TVD stage: x, y, z passes)",
                      "hbm_achieved_gbs": achieved, "hbm_frac": achieved / hbm_peak,
                      "algo_bytes_per_launch": algo_launch, "mean_launch_ms": stage_ms}),
        "e2e": {"value": world * pts * args.steps / e2e_s / 1e6, "unit": METRIC,
                "h2d_bytes_per_step": i2.h2d_bytes / args.steps, "d2h_bytes_per_step": st.nbytes / args.steps,
                "seconds": e2e_s, "path": "cgfdm_create(run dir) + cgfdm_run(K) + cgfdm_get_stations + destroy",
                "split_ms": create_prof, "legs": e2e_legs,
                "first_session_create_s": first_create_s},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    # the result's error against the FP64 run over the timed steps
    line["err_vs_fp64"] = fp64_error(d, args.steps, local_rank, session_options(args))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, why = cpu_reference_rate(args.workload, 2, 4, min(os.cpu_count() or 1, 32))
        line["cpu_baseline"] = cb if cb else {"unavailable": why}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
