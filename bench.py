#!/usr/bin/env python
"""Throughput benchmark of the B200 D3Q19 LBM + IBM time step.

Workload (default "suspension-128"): the dense power-law suspension as the
reference's own host expresses it -- 128^3 lattice (126^3 interior nodes, z
walls at +-0.05 lu/step, periodic x/y), 200 freely moving spheres of diameter
16 on the reference's jittered grid with its marker rule (1024 IBM markers
each), power-law fluid n = 0.6, k = 0.0105 with the reference's tau limits.
Both arms (--impl ours and --impl reference) run it from the same keywords and
initial state.  "dense-powerlaw-128" is the same lattice and sphere count with
512 markers per sphere placed by seeded random sequential addition (2 lu gap)
and tau clamped to [0.55, 2.0], which the reference's host cannot express; its
reference arm is the C restatement of the reference's algorithm on the same
initial state.  A step is one full time step (collide-stream with
boundaries, IBM, rigid bodies, particle contacts, zone rebuild every 10
steps).

Metric: MLUPS = interior nodes x steps / s / 1e6, summed over GPUs (each GPU
runs an independent replica: weak scaling, no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--storage fp32|fp16|bf16] [--two-buffers]

The distributions are kept in one buffer updated in place (the AA pattern,
d3q19_options.inplace = 1), which gives results bit-identical to the
reference's two buffers; --two-buffers measures that layout instead.

Other modes (--workload, one GPU, one JSON line each): powerlaw-128-fluid and
couette-sphere-64 (the same line for the fluid alone and the 64^3 single
sphere); batch-64 (64 uneven boxes in one lattice pool against each alone);
served-sweep (Poisson arrivals of shear-rheology solves through the pool's
serving loop against one at a time); served-preempt (the same on a pool
with a small HBM budget, with and without pre-emption); casson-precision
(FP32 / FP16 / BF16 storage against the FP64 build).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "dispersion-shear_d3q19-opencl_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, REPO)

# Algorithmic bytes per lattice node and step: 19 populations read + 19
# written, FP32 (4 B) or 16-bit shifted storage (2 B).
STORAGE = {"fp32": (0, 152, "f32"), "fp16": (1, 76, "f32 arithmetic, f16 shifted storage"),
           "bf16": (2, 76, "f32 arithmetic, bf16 shifted storage")}

WORKLOADS = {
    "dense-powerlaw-128": dict(
        iterations=10000, total_lattice_size=(128, 128, 128), boundary_conditions_xyz=(0, 0, 1), newtonian_tau=1.0,
        viscosity_model=2, viscosity_params=(0.0105, 0.6, 0.0, 0.0), use_constant_viscosity=0, tau_min=0.55,
        tau_max=2.0, velocity_bc_upper=(0.05, 0.0, 0.0), velocity_bc_lower=(-0.05, 0.0, 0.0), initial_f="constant",
        initial_vel=(0.0, 0.0, 0.0), num_particles=200, particle_diameter=16.0, ibm_points_per_particle=512,
        initial_particle_distribution=4, particle_seed=1, min_particle_gap=2.0, initial_particle_buffer=0.0,
        z_wall_particle_buffer=9.0, domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=10,
        particle_collision_params=2.0, video_freq=1000000, shear_stress_freq=1000000, console_print_freq=1000000),
}
# The same fluid without spheres (fluid kernel alone; a profiling aid).
WORKLOADS["powerlaw-128-fluid"] = dict(WORKLOADS["dense-powerlaw-128"], num_particles=0)
# 64^3 Couette flow past one fixed sphere of diameter 16 with 256 markers at
# the box centre, Newtonian tau = 0.8, walls +-0.02 (the reference's own
# CPU-runnable single-sphere case).
WORKLOADS["couette-sphere-64"] = dict(
    iterations=2000, total_lattice_size=(64, 64, 64), boundary_conditions_xyz=(0, 0, 1), newtonian_tau=0.8,
    viscosity_model=1, velocity_bc_upper=(0.02, 0.0, 0.0), velocity_bc_lower=(-0.02, 0.0, 0.0), initial_f="constant",
    initial_vel=(0.0, 0.0, 0.0), num_particles=1, particle_diameter=16.0, ibm_points_per_particle=256,
    fixed_particles=1, initial_particle_distribution=3, initial_particle_buffer=31.0, z_wall_particle_buffer=2.0,
    domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=10, video_freq=1000000, shear_stress_freq=1000000,
    console_print_freq=1000000)
DESCRIPTION = {
    "dense-powerlaw-128": "dense power-law suspension: 128^3 lattice, 200 spheres d=16 (512 markers, RSA seed 1, "
                          "gap 2), n=0.6 k=0.0105 tau in [0.55,2], walls +-0.05",
    "powerlaw-128-fluid": "power-law fluid alone: 128^3 lattice, n=0.6 k=0.0105 tau in [0.55,2], walls +-0.05",
    "couette-sphere-64": "Couette flow past one fixed sphere: 64^3 lattice, Newtonian tau 0.8, walls +-0.02, "
                         "d=16 with 256 markers at the centre",
}

# The same workload as the reference host can express it: its marker rule
# (1024 points for d=16), jittered-grid placement (distribution 2) instead of
# seeded RSA, no tau clamps, the build without USE_CONSTANT_VISCOSITY.
REFERENCE_KEYWORDS = {
    "dense-powerlaw-128": dict(
        total_lattice_size=(128, 128, 128), boundary_conditions_xyz=(0, 0, 1), newtonian_tau=1.0,
        viscosity_model=2, viscosity_params=(0.0105, 0.6, 0.0, 0.0), velocity_bc_upper=(0.05, 0.0, 0.0),
        velocity_bc_lower=(-0.05, 0.0, 0.0), initial_f="constant", initial_vel=(0.0, 0.0, 0.0), num_particles=200,
        particle_diameter=16.0, initial_particle_distribution=2, random_particle_shift=0.0,
        initial_particle_buffer=8.0, z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1),
        rebuild_neigh_list_freq=10, particle_collision_params=2.0, video_freq=1000000, shear_stress_freq=1000000,
        console_print_freq=1000000),
}


REFERENCE_KEYWORDS["powerlaw-128-fluid"] = dict(REFERENCE_KEYWORDS["dense-powerlaw-128"], num_particles=0)
# The dense suspension exactly as the reference's host expresses it -- its
# marker rule (1024 points for d = 16), jittered-grid placement, its tau
# limits -- run by both arms from the same keywords (the default line): the
# 128^3 lattice, 200 spheres of d = 16, power law n = 0.6, walls +-0.05.
REFERENCE_KEYWORDS["suspension-128"] = dict(REFERENCE_KEYWORDS["dense-powerlaw-128"], random_particle_shift=0.5,
                                            iterations=10000, use_constant_viscosity=0)
WORKLOADS["suspension-128"] = dict(REFERENCE_KEYWORDS["suspension-128"])
DESCRIPTION["suspension-128"] = ("dense power-law suspension as the reference expresses it: 128^3 lattice, 200 spheres "
                                 "d=16 on the reference's jittered grid (shift 0.5), 1024 markers each (the reference's "
                                 "rule), n=0.6 k=0.0105 (the reference's tau limits), walls +-0.05")
# The reference has no fixed spheres and derives 1024 markers for d = 16.
REFERENCE_KEYWORDS["couette-sphere-64"] = dict(
    total_lattice_size=(64, 64, 64), boundary_conditions_xyz=(0, 0, 1), newtonian_tau=0.8, viscosity_model=1,
    velocity_bc_upper=(0.02, 0.0, 0.0), velocity_bc_lower=(-0.02, 0.0, 0.0), initial_f="constant",
    initial_vel=(0.0, 0.0, 0.0), num_particles=1, particle_diameter=16.0, initial_particle_distribution=3,
    initial_particle_buffer=31.0, z_wall_particle_buffer=2.0, domain_decomposition=(1, 1, 1),
    rebuild_neigh_list_freq=10, video_freq=1000000, shear_stress_freq=1000000, console_print_freq=1000000)
# Which reference build runs the workload (with or without USE_CONSTANT_VISCOSITY).
REFERENCE_VARIABLE = {"dense-powerlaw-128": True, "powerlaw-128-fluid": True, "couette-sphere-64": False,
                      "suspension-128": True}
REFERENCE_NOTE = {
    "suspension-128": "the same keywords and initial state as the GPU arm (same_config)",
    "dense-powerlaw-128": "the 128^3 lattice with 200 d=16 spheres; reference marker rule (1024/sphere) and "
                          "jittered-grid placement",
    "powerlaw-128-fluid": "the 128^3 power-law lattice without spheres",
    "couette-sphere-64": "the 64^3 Couette lattice with one d=16 sphere (reference marker rule: 1024 markers; "
                         "the reference integrates the sphere)",
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed
    region (the GPU's physical index resolved through CUDA_VISIBLE_DEVICES)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.index = str(local_rank)
        if vis:
            ids = [v.strip() for v in vis.split(",") if v.strip()]
            if local_rank < len(ids):
                self.index = ids[local_rank]
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(workload, storage="fp32", inplace=False):
    """DRAM bytes per launch of the collide-stream kernel from the committed
    ncu summary (profiles/), or None."""
    suffix = ("" if storage == "fp32" else "_" + storage) + ("_inplace" if inplace else "")
    p = os.path.join(REPO, "profiles", f"fluid_step_kernel_{workload}{suffix}.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return d.get("dram_bytes_per_launch_full_size")
    except (OSError, ValueError):
        return None


FLUID_KERNELS = {"tile": 0, "tma": 1}


def setup(workload, device, storage="fp32", inplace=False, fluid_kernel="tile"):
    import numpy as np  # noqa: F401

    import d3q19_b200 as d3

    cfg = d3.parse_config(d3.keywords_text(WORKLOADS[workload]))
    hs = d3.HostState(cfg, data_dir=os.getcwd())
    hs.options.device = device
    hs.options.storage = STORAGE[storage][0]
    hs.options.inplace = int(inplace)
    hs.options.fluid_kernel = FLUID_KERNELS[fluid_kernel]
    sim = d3.Simulation.from_host_state(hs, device=device, storage=STORAGE[storage][0], inplace=int(inplace),
                                        fluid_kernel=FLUID_KERNELS[fluid_kernel])
    return d3, hs, sim


L2_BYTES = 126 * 2 ** 20


def l2_note(ip, bytes_per_node):
    """How the timed steps relate to L2: the two distribution buffers each
    step reads and writes against the 126 MB L2 (no flush is made)."""
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    fbytes = bytes_per_node * nc  # 19 populations read + 19 written
    if fbytes > L2_BYTES:
        return f"inputs larger than L2: the step streams {fbytes / 1e6:.0f} MB of distributions (L2 126 MB)"
    return (f"inputs smaller than L2 ({fbytes / 1e6:.0f} MB of distributions per step, L2 126 MB), no flush: "
            "an L2-resident small case, not the headline line")


def max_over_ranks(x, dist, device):
    """The largest x over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(world, interior, steps, ms_max):
    """Whole-job throughput of `world` independent replicas, each advancing
    `interior` nodes by `steps` steps, timed by the slowest rank."""
    return world * interior * steps / (ms_max * 1e-3) / 1e6


def launches(ip, rebuild, t0, k):
    """Kernels one step sequence launches: the fluid step, and with spheres
    the particle pass, the contact forces and (every rebuild steps) the zone
    rebuild."""
    n = 0
    for t in range(t0, t0 + k):
        n += 1
        if ip.NumParticles > 0:
            n += 2 + (1 if t % rebuild == 0 else 0)
    return n


def run_ours(args, rank, world, local_rank, dist):
    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    d3, hs, sim = setup(args.workload, local_rank, args.storage, args.inplace, args.fluid_kernel)
    kernel_name = {"tma": "fluid_tma_kernel", "tile": "fluid_step_kernel"}.get(sim.fluid_kernel, sim.fluid_kernel)
    bytes_per_node = STORAGE[args.storage][1]
    ip = hs.cfg.ip
    interior = (ip.LatticeSize[0] - 2) * (ip.LatticeSize[1] - 2) * (ip.LatticeSize[2] - 2)
    R = hs.cfg.hp.RebuildFreq
    stream = torch.cuda.ExternalStream(sim.stream_ptr, device=local_rank)
    t = 1
    sim.run(t, args.warmup)
    t += args.warmup
    sim.synchronize()

    # The CUDA graphs the timed steps replay are captured (not run) first.
    sim.prepare_run(t, args.steps)
    sim.synchronize()

    # Timed region: exactly K steps, barrier + synchronize on both sides.
    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(t, args.steps)
    e1.record(stream)
    sim.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    t += args.steps
    n_launch = launches(ip, R, t - args.steps, args.steps)
    ms_max = max_over_ranks(ms, dist, f"cuda:{local_rank}")

    # Per-launch device time of the collide-stream kernel (events around
    # each launch on the library's stream), for the roofline.
    kp = min(args.steps, 200)
    sim.profile(True)
    sim.run(t, kp)
    fluid_ms, nf, part_ms, npart = sim.profile_read()
    sim.profile(False)
    t += kp
    fluid_avg = fluid_ms / max(nf, 1)
    part_avg = part_ms / max(npart, 1)

    # End to end through the C ABI: pinned host buffers uploaded, K steps,
    # velocity and particle state read back.
    def pinned(a):
        buf = torch.empty(a.size, dtype=torch.float32 if a.dtype.kind == "f" else torch.int32, pin_memory=True)
        out = buf.numpy()
        out[:] = a
        return out

    hf, hu, htau = pinned(hs.f), pinned(hs.u), pinned(hs.tau)
    hk, hpf, hpff, hsp = pinned(hs.parKin), pinned(hs.parForce), pinned(hs.parFluidForce), pinned(hs.spherePoints)
    ru = pinned(np.zeros(3 * sim.nc, np.float32))
    rk = pinned(np.zeros(16 * sim.np, np.float32))
    rpff = pinned(np.zeros(8 * sim.np * sim.nfa, np.float32))
    hpm = pinned(d3.periodic_map(hs.cfg.ip))  # an input array, prepared on the host like the others
    sim2 = d3.Simulation(hs.cfg.ip, hs.cfg.fp, hs.options)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    sim2.write_lattice(hf, hu, htau)
    sim2.write_periodic_map(hpm)
    if sim2.np > 0:
        sim2.write_particles(hk, hpf, hpff, hsp)
        sim2.write_zones(hs.zoneNeighDat, hs.parsZone, hs.zoneMembers, hs.numParInZone, hs.threadMembers,
                         hs.numParInThread)
    sim2.run(1, args.steps)
    sim2.read_u(out=ru)  # straight into pinned host memory
    if sim2.np > 0:
        sim2.read_parkin(out=rk)
        sim2.read_parfluidforce(out=rpff)
    e2e_s = time.perf_counter() - w0
    e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local_rank}")
    h2d = hf.nbytes + hu.nbytes + htau.nbytes + hpm.nbytes + hk.nbytes + hpf.nbytes + hpff.nbytes + hsp.nbytes
    d2h = ru.nbytes + (rk.nbytes + rpff.nbytes if sim2.np > 0 else 0)
    sim2.close()
    sim.close()

    if rank != 0:
        return None
    peak, peak_kind = measured_peak()
    achieved = bytes_per_node * interior / (fluid_avg * 1e-3) / 1e9
    value = replica_mlups(world, interior, args.steps, ms_max)
    out = {
        "metric": "MLUPS", "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": STORAGE[args.storage][2],
        "data": ("synthetic (the reference's jittered-grid placement)" if args.workload == "suspension-128" else
                 "synthetic (seeded RSA placement)" if args.workload == "dense-powerlaw-128" else "synthetic"),
        "impl": "ours",
        "config": {"workload": args.workload, "description": DESCRIPTION[args.workload],
                   "lattice": list(ip.LatticeSize), "interior_nodes": interior, "spheres": ip.NumParticles,
                   "markers_per_sphere": ip.PointsPerParticle, "parallelism": f"replicas x{world}",
                   "l2": l2_note(ip, bytes_per_node),
                   "distribution_buffers": 1 if args.inplace else 2},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": ncu_traffic(args.workload, args.storage, args.inplace),
                     "kernel": kernel_name, "bytes_per_node": bytes_per_node,
                     "kernel_ms": round(fluid_avg, 5), "particle_kernel_ms": round(part_avg, 5),
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                     "fallback 6.65 TB/s",
                     "step_frac": round(value / world * 1e6 * bytes_per_node / 1e9 / peak, 4)},
        "e2e": {"value": round(replica_mlups(world, interior, args.steps, e2e_s * 1e3), 1), "unit": "MLUPS",
                "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                "note": "C-ABI calls from pinned host buffers: upload of the initial state, K steps, read-back "
                        "of u, sphere kinematics and forces"},
        "gpu_launches": n_launch,
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        if args.workload in PORT_WORKLOADS:
            out["cpu_baseline"] = port_baseline(args.workload)
            out["cpu_baseline"]["reference_program"] = cpu_baseline(args.workload)
        else:
            out["cpu_baseline"] = cpu_baseline(args.workload)
    return out


# ---------------------------------------------------------------------------
def _reference_run(workload, iters, threads):
    """Wall time of the reference's own program (built from its sources for
    the host cores, oracle/_ref) for `iters` steps of the workload."""
    from oracle import pyoracle as po

    kw = dict(REFERENCE_KEYWORDS[workload], iterations=iters)
    t0 = time.perf_counter()
    po.run_reference(kw, variable_viscosity=REFERENCE_VARIABLE[workload], serial=False, dump=False, threads=threads,
                     workdir=tempfile.mkdtemp(prefix="d3q19bench_"))
    return time.perf_counter() - t0


def cpu_baseline(workload, sample_steps=8):
    """CPU throughput of the reference on the box's host cores: the difference
    of two runs (1 and 1 + sample_steps steps) removes the set-up time."""
    from oracle import pyoracle as po

    threads = os.cpu_count() or 1
    kw = WORKLOADS[workload]
    N = kw["total_lattice_size"]
    interior = (N[0] - 2) * (N[1] - 2) * (N[2] - 2)
    if po.ref_available():
        ta = _reference_run(workload, 1, threads)
        tb = _reference_run(workload, 1 + sample_steps, threads)
        per = max(tb - ta, 1e-9) / sample_steps
        return {"value": round(interior / per / 1e6, 3), "unit": "MLUPS", "cores": threads, "kind": "reference",
                "sample": f"{sample_steps} steps of the reference's own program (GPU_program.cl "
                          f"{'without' if REFERENCE_VARIABLE[workload] else 'with'} USE_CONSTANT_VISCOSITY + "
                          "CPU_program.cl + D3Q19-OpenCL.c, mock OpenCL runtime, "
                          f"{threads} OpenMP threads) on {REFERENCE_NOTE[workload]}; per-step time from the "
                          f"difference of a 1-step and a {1 + sample_steps}-step run"}
    return {"value": None, "unit": "MLUPS", "cores": threads, "kind": "reference",
            "sample": "oracle/_ref not built on this machine"}


def port_baseline(workload, sample_steps=2):
    """CPU throughput of the reference's algorithm on exactly the GPU arm's
    initial state (lattice, sphere placement, markers): the C restatement
    oracle/d3q19_oracle.c, pinned bit for bit to the reference's own program
    on the golden vectors, run over the box's host cores (OpenMP over the
    collide-stream loop).  The restatement follows the reference's tau limits
    (no upper clamp), the GPU arm's configuration asks for tau in [0.55, 2]:
    the same work per node."""
    import numpy as np

    from oracle import pyoracle as po

    import d3q19_b200 as d3

    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    hs = d3.HostState(d3.parse_config(d3.keywords_text(WORKLOADS[workload])), data_dir=os.getcwd())
    ip, fp = hs.cfg.ip, hs.cfg.fp
    nc = ip.LatticeSize[0] * ip.LatticeSize[1] * ip.LatticeSize[2]
    oip, ofp = po.params_from_bytes(bytes(ip), bytes(fp))
    sm = d3.periodic_map(ip)
    arrays = dict(fA=hs.f.copy(), fB=hs.f.copy(), u=hs.u, tau_lb=hs.tau, strMap=sm, spherePoints=hs.spherePoints,
                  zoneNeighDat=hs.zoneNeighDat, numParInZone=hs.numParInZone, numParInThread=hs.numParInThread,
                  parsZone=hs.parsZone, zoneMembers=hs.zoneMembers, threadMembers=hs.threadMembers,
                  parKin=hs.parKin, parForce=hs.parForce, parFluidForce=hs.parFluidForce,
                  gpf=np.zeros(3 * max(ip.MaxSurfPointsPerNode, 1) * nc, np.float32),
                  countPoint=np.zeros(nc, np.int32))
    nth = hs.cfg.hp.DomainDecomp[0] * hs.cfg.hp.DomainDecomp[1] * hs.cfg.hp.DomainDecomp[2]
    st = po.OracleState(oip, ofp, arrays, nth, hs.cfg.hp.RebuildFreq, not hs.cfg.hp.UseConstantViscosity)
    st.step(1)  # first touch of the arrays
    t0 = time.perf_counter()
    st.run(2, sample_steps)
    per = (time.perf_counter() - t0) / sample_steps
    N = ip.LatticeSize
    interior = (N[0] - 2) * (N[1] - 2) * (N[2] - 2)
    return {"value": round(interior / per / 1e6, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{sample_steps} steps (after one untimed step) of the reference's algorithm restated in C "
                      f"(oracle/d3q19_oracle.c, bit-exact to the reference's own program on the golden vectors), "
                      f"{threads} OpenMP threads, on the GPU arm's initial state: {DESCRIPTION[workload]}"}


# Workloads whose reference arm is the restatement on the GPU arm's own state
# (the reference's host cannot place spheres by seeded random sequential
# addition or override its marker count).
PORT_WORKLOADS = {"dense-powerlaw-128"}


def run_reference_arm(args):
    if args.workload not in REFERENCE_KEYWORDS:
        return {"impl": "reference", "unavailable": f"{args.workload}: the reference runs one lattice per process and "
                                                    "has no pool or request loop"}
    if args.workload in PORT_WORKLOADS:
        b = port_baseline(args.workload, sample_steps=max(1, min(args.steps, 2)))
        b["reference_program"] = cpu_baseline(args.workload, sample_steps=max(1, min(args.steps, 8)))
    else:
        b = cpu_baseline(args.workload, sample_steps=max(1, min(args.steps, 8)))
    kw = WORKLOADS[args.workload]
    N = kw["total_lattice_size"]
    out = {"impl": "reference", "metric": "MLUPS", "value": b["value"], "unit": "MLUPS", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": (round((N[0] - 2) * (N[1] - 2) * (N[2] - 2) / (b["value"] * 1e6) * 1e3, 3)
                           if b["value"] else None),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "config": {"workload": args.workload, "description": DESCRIPTION[args.workload]},
           "cpu_baseline": b, "e2e": {"value": b["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}
    if b["value"] is None:
        out = {"impl": "reference", "unavailable": b["sample"]}
    return out


# ---------------------------------------------------------------------------
# The lattice pool: batched uneven boxes and the served sweep.
def batch_requests(n=64, seed=4):
    """64 independent boxes: edges from {32,48,64,96} per axis, 1-20 spheres
    of radius 4-8, power-law n in [0.4, 1], wall speed in [0.01, 0.05]."""
    import numpy as np

    from d3q19_b200 import serving as sv

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        edge = tuple(int(rng.choice([32, 48, 64, 96])) for _ in range(3))
        d = float(rng.uniform(8.0, 16.0))
        # 1-20 spheres, at most what fills a quarter of the slab their
        # centres may occupy (random sequential addition must place them).
        slab = (edge[0] - 2) * (edge[1] - 2) * max(edge[2] - 2 - d - 4, 0.0)
        nsph = min(int(rng.integers(1, 21)), int(0.25 * slab / (math.pi / 6 * d ** 3)))
        req = sv.ShearRequest(rid=i, edge=edge, phi=0.0, model="power_law", wall_speed=float(rng.uniform(0.01, 0.05)),
                              seed=int(rng.integers(1, 2 ** 31 - 1)), diameter=d, n_index=float(rng.uniform(0.4, 1.0)))
        kw = sv.solve_keywords(req)
        # Sphere count as drawn (not from a volume fraction); the slab must
        # hold the spheres' centres.
        kw.update(num_particles=nsph)
        if nsph > 0:
            kw.update(particle_diameter=d, initial_particle_distribution=4, particle_seed=req.seed,
                      min_particle_gap=0.0, initial_particle_buffer=0.0, z_wall_particle_buffer=d / 2 + 2,
                      particle_collision_params=2.0)
        out.append((req, kw))
    return out


def _time_pool(pool, steps, stream_ptr, torch):
    stream = torch.cuda.ExternalStream(stream_ptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pool.advance(steps)
    e1.record(stream)
    pool.synchronize()
    return e0.elapsed_time(e1)


def run_batch(args):
    """cfg: 64 uneven boxes advanced together (FP16 shifted storage, chunks
    of 1000 steps captured as graphs, grid sizes from the autotuner) against
    the same boxes one at a time in FP32."""
    import torch

    import d3q19_b200 as d3

    torch.cuda.set_device(0)
    items = batch_requests()
    states = [d3.HostState(d3.parse_config(d3.keywords_text(kw)), data_dir=os.getcwd()) for _, kw in items]
    nodes = sum((hs.cfg.ip.LatticeSize[0] - 2) * (hs.cfg.ip.LatticeSize[1] - 2) * (hs.cfg.ip.LatticeSize[2] - 2)
                for hs in states)
    chunk = 1000
    # Two buffers: with these small FP16 boxes they measured faster than the
    # in-place layout (17,573 against 16,593 MLUPS), unlike the served FP32 pools.
    pool = d3.Pool(storage=1, max_slots=len(states), hbm_budget=120 << 30, inplace=False)
    for hs in states:
        if pool.admit(hs) is None:
            raise RuntimeError("batch does not fit the pool")
    # The library's grid autotuner (d3q19_pool_autotune): each 200-step
    # advance of the live batch times the next candidate particle/contact
    # grid of the batch's work class until every candidate has run; the
    # fastest is kept (the fluid pass runs one CTA per tile).  The results do
    # not depend on the grid, so these are ordinary steps.
    d3.tune_clear()
    tuning_steps = 0
    while not pool.tune_state()["settled"]:
        pool.advance(200)
        tuning_steps += 200
    trials = pool.tune_trials()
    best = min(trials, key=lambda x: x[2])
    pool.advance(chunk)  # capture of the 1000-step chunk
    grid = pool.get_grid()[:2]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    ms = _time_pool(pool, chunk * max(1, args.steps // chunk), pool.stream_ptr, torch)
    steps = chunk * max(1, args.steps // chunk)
    pool.close()
    batched = nodes * steps / (ms * 1e-3) / 1e6
    # One at a time, FP32, graph-replayed runs of the same step count each.
    base_steps = 200
    t_alone = 0.0
    for hs in states:
        sim = d3.Simulation.from_host_state(hs, device=0, storage=0)
        sim.run(1, 64)
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.run(65, base_steps)
        e1.record(stream)
        sim.synchronize()
        t_alone += e0.elapsed_time(e1)
        sim.close()
    alone = nodes * base_steps / (t_alone * 1e-3) / 1e6
    return {"metric": "MLUPS (batched boxes)", "value": round(batched, 1), "unit": "MLUPS", "n_gpus": 1,
            "steps": steps, "higher_is_better": True, "dtype": "f32 arithmetic, f16 shifted storage",
            "data": "synthetic (seeded)", "impl": "ours",
            "config": {"workload": "batch-64", "boxes": len(states), "interior_nodes": nodes,
                       "description": "64 boxes, edges from {32,48,64,96} per axis, 1-20 spheres of radius 4-8, "
                                      "power-law n in [0.4,1], walls +-[0.01,0.05]; one launch per pass for all"},
            "autotune": {"particle_ctas_per_sm": best[1], "particle_ctas_per_sm_in_use": grid[1] // sms,
                         "fluid_grid": grid[0], "fluid": "one CTA per tile", "tuning_steps": tuning_steps,
                         "default_particle_ctas_per_sm": 4,
                         "trials_ns_per_tile_step": [[pp, round(t, 2)] for _, pp, t in trials],
                         "tile": "32x4x4"},
            "one_at_a_time_fp32": {"value": round(alone, 1), "unit": "MLUPS"},
            "speedup_vs_one_at_a_time_fp32": round(batched / alone, 2)}


def run_pool_mix(args):
    """cfg: the served sweep's first 48 requests resident in one FP32
    in-place pool at the default particle grid (no autotuner), advanced
    together: the batched kernels on a served mix, for profiling."""
    import torch

    import d3q19_b200 as d3
    from d3q19_b200 import serving as sv

    torch.cuda.set_device(0)
    reqs = sv.make_requests(48, 50.0, 2024, edges=(32, 64))
    pool = d3.Pool(storage=0, max_slots=64, hbm_budget=40 << 30, inplace=True, autotune=False)
    for r in reqs:
        if pool.admit(sv.host_state(r)) is None:
            raise RuntimeError("the mix does not fit the pool")
    nodes = sum((r.edge[0] - 2) ** 3 for r in reqs)
    # 32 x 4 x 4 tiles from the lattice origin, buffer layers included (as the kernels tile)
    tiles = sum(math.ceil(r.edge[0] / 32) * math.ceil(r.edge[1] / 4) * math.ceil(r.edge[2] / 4) for r in reqs)
    period = pool.period
    pool.advance(max(period, args.warmup // period * period))  # capture and warm-up
    steps = max(period, args.steps // period * period)
    pool.advance(steps)  # capture of the timed chunk length
    ms = _time_pool(pool, steps, pool.stream_ptr, torch)
    pool.close()
    return {"metric": "MLUPS (served mix in one pool)", "value": round(nodes * steps / (ms * 1e-3) / 1e6, 1),
            "unit": "MLUPS", "n_gpus": 1, "steps": steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded)", "impl": "ours",
            "config": {"workload": "pool-mix", "requests": len(reqs), "interior_nodes": nodes, "tiles": tiles,
                       "description": "the served sweep's first 48 requests (edges 32-64, phi 0-0.3, three laws) "
                                      "in one FP32 in-place pool, default grid"},
            "ns_per_tile_step": round(ms * 1e6 / (steps * tiles), 2)}


def warm_served_paths(storages, alone=True):
    """Untimed: a short burst through a pool of each storage (and, with
    alone, one solve on its own context), so that the timed runs do not pay
    the first use of the kernels, graphs and allocators."""
    import d3q19_b200 as d3
    from d3q19_b200 import serving as sv

    reqs = sv.make_requests(12, 0.0, 99, edges=(32, 64))
    for storage in storages:
        pool = d3.Pool(storage=storage, max_slots=64, hbm_budget=4 << 30, inplace=True)
        sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=2000).run(reqs)
        pool.close()
    if alone:
        sv.one_at_a_time(reqs[:2], storage=0, check_every=500, rel_tol=1e-4, max_steps=2000)


def run_served(args):
    """cfg: Poisson arrivals (50/s, seeded) of shear-rheology solves, cubic
    edge in [32, 64], volume fraction in [0, 0.3], Newtonian / power law /
    Casson, each until the mean shear stress changes < 1e-4 relative over 500
    steps (at most max_steps); a pool with continuous batching (FP32 storage;
    FP16 shifted storage reported beside it) against one-at-a-time FP32."""
    import numpy as np
    import torch

    import d3q19_b200 as d3
    from d3q19_b200 import serving as sv

    torch.cuda.set_device(0)
    reqs = sv.make_requests(args.requests, 50.0, 2024, edges=tuple(args.edges))
    max_steps = args.max_steps
    warm_served_paths((0, 1))
    runs = {}
    for storage in (0, 1):
        pool = d3.Pool(storage=storage, max_slots=256, hbm_budget=100 << 30, inplace=args.inplace)
        runs[storage] = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=max_steps,
                                  solo_nodes=args.solo_nodes or None).run(reqs)
        pool.close()
    # The autotuner's choices for the work classes the pools met (CTAs per SM
    # of the fluid and particle passes, ns per fluid tile step).
    tuned = [ln.split("\t") for ln in d3.tune_export().splitlines()]
    served, served16 = sv.summary(*runs[0]), sv.summary(*runs[1])
    base, bwall = sv.one_at_a_time(reqs, storage=0, check_every=500, rel_tol=1e-4, max_steps=max_steps)
    alone = sv.summary(base, bwall)
    by = {r.rid: r for r in base}

    def visc_diff(recs):
        d = [abs(r.eff_viscosity - by[r.rid].eff_viscosity) / max(abs(by[r.rid].eff_viscosity), 1e-30)
             for r in recs if not (r.failed or by[r.rid].failed)]
        return {"max": float(np.max(d)), "median": float(np.median(d))}

    recs = runs[0][0]
    return {"metric": "solves/s (served sweep)", "value": round(served["solves_per_s"], 3), "unit": "solves/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded Poisson arrivals)", "impl": "ours",
            "config": {"workload": "served-sweep", "requests": len(reqs), "arrival_rate_per_s": 50.0,
                       "edges": list(args.edges), "phi": [0.0, 0.3], "models": list(sv.MODELS),
                       "stop": "1e-4 over 500 steps",
                       "max_steps": max_steps, "pool_storage": "fp32",
                       "solo_nodes": args.solo_nodes or None,
                       "solo_requests": sum(1 for r in reqs if args.solo_nodes and
                                            math.prod(e - 2 for e in r.edge) >= args.solo_nodes),
                       "pool_layout": "in place" if args.inplace else "two buffers"},
            "autotune": [{"storage": int(t[2]), "inplace": int(t[3]), "class_tiles": f"<2^{t[4]}",
                          "fluid_ctas_per_sm": int(t[5]), "particle_ctas_per_sm": int(t[6]),
                          "ns_per_tile_step": float(t[7])} for t in tuned],
            "served": served, "served_fp16_pool": served16, "one_at_a_time_fp32": alone,
            "speedup_solves_per_s": round(served["solves_per_s"] / alone["solves_per_s"], 2),
            "speedup_fp16_pool": round(served16["solves_per_s"] / alone["solves_per_s"], 2),
            "per_request": [[r.rid, r.steps, by[r.rid].steps, round(r.latency, 3), round(by[r.rid].latency, 3)]
                            for r in sorted(recs, key=lambda r: r.rid)],
            "eff_viscosity_rel_diff_pool_vs_alone": visc_diff(recs),
            "eff_viscosity_rel_diff_fp16_pool_vs_alone": visc_diff(runs[1][0])}


def run_served_preempt(args):
    """cfg: the served sweep's Poisson arrivals (50/s, seeded) on an FP32 pool
    whose HBM budget (256 MB) holds a few members at a time, served twice: admission
    in arrival order only, and with pre-emption (a request that does not fit
    evicts the member with the most steps since its admission, once that is
    at least 2000; the evicted member's checkpoint waits in host memory and
    is re-admitted before later arrivals).  Reports throughput, latency and
    the measured cost of the evictions and re-admissions."""
    import numpy as np
    import torch

    import d3q19_b200 as d3
    from d3q19_b200 import serving as sv

    torch.cuda.set_device(0)
    reqs = sv.make_requests(args.requests, 50.0, 2025, edges=(32, 64))
    max_steps = 40000
    budget = 256 << 20
    warm_served_paths((0,), alone=False)
    out = {}
    for label, pre in (("arrival_order", None), ("preempt_2000", 2000)):
        pool = d3.Pool(storage=0, max_slots=64, hbm_budget=budget, inplace=args.inplace)
        cost = {"evict_s": 0.0, "readmit_s": 0.0, "bytes": 0, "n": 0}
        ev, re = pool.evict, pool.readmit

        def evict(slot, ev=ev, cost=cost):
            t = time.perf_counter()
            r = ev(slot)
            cost["evict_s"] += time.perf_counter() - t
            cost["bytes"] += int(r[0].nbytes)
            cost["n"] += 1
            return r

        def readmit(ck, re=re, cost=cost):
            t = time.perf_counter()
            r = re(ck)
            cost["readmit_s"] += time.perf_counter() - t
            return r

        pool.evict, pool.readmit = evict, readmit
        recs, wall = sv.Server(pool, check_every=500, rel_tol=1e-4, max_steps=max_steps, preempt_after=pre).run(reqs)
        pool.close()
        summ = sv.summary(recs, wall)
        summ["evictions"] = cost["n"]
        summ["checkpoint_mb_total"] = round(cost["bytes"] / 1e6, 1)
        summ["evict_s_total"] = round(cost["evict_s"], 3)
        summ["readmit_s_total"] = round(cost["readmit_s"], 3)
        summ["latency_by_rid"] = {r.rid: round(r.latency, 3) for r in recs}
        out[label] = summ
    a, b = out["arrival_order"], out["preempt_2000"]
    lat_a = np.array([a["latency_by_rid"][r.rid] for r in reqs])
    lat_b = np.array([b["latency_by_rid"][r.rid] for r in reqs])
    for v in out.values():
        del v["latency_by_rid"]
    return {"metric": "solves/s (served sweep, HBM-limited pool)", "value": round(b["solves_per_s"], 3),
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded Poisson arrivals)",
            "impl": "ours",
            "config": {"workload": "served-preempt", "requests": len(reqs), "arrival_rate_per_s": 50.0,
                       "edges": [32, 64], "phi": [0.0, 0.3], "models": list(sv.MODELS), "hbm_budget_mb": budget >> 20,
                       "stop": "1e-4 over 500 steps", "max_steps": max_steps},
            "runs": out,
            "requests_faster_with_preemption": int(np.sum(lat_b < lat_a)),
            "median_latency_ratio_preempt_over_arrival_order": round(float(np.median(lat_b / lat_a)), 3)}


def run_precision(args):
    """Casson suspension: 256x128x256 lattice, 1000 spheres of radius 6 (384
    markers each, seeded random placement), regularised Casson yield stress
    1e-4 and plastic tau 0.6, walls +-0.04; FP32, FP16 and BF16 shifted
    storage against the FP64 build after the same steps: errors of velocity,
    mean shear stress, effective viscosity and per-sphere force and torque."""
    import numpy as np
    import torch

    import d3q19_b200 as d3

    torch.cuda.set_device(0)
    kw = dict(iterations=args.steps, total_lattice_size=(256, 128, 256), boundary_conditions_xyz=(0, 0, 1),
              newtonian_tau=0.6, viscosity_model=4, viscosity_params=(1e-4, (0.6 - 0.5) / 3.0, 0.0, 0.0),
              use_constant_viscosity=0, casson_regularisation=1e-4, velocity_bc_upper=(0.04, 0.0, 0.0),
              velocity_bc_lower=(-0.04, 0.0, 0.0), initial_f="constant", initial_vel=(0.0, 0.0, 0.0),
              num_particles=1000, particle_diameter=12.0, ibm_points_per_particle=384,
              initial_particle_distribution=4, particle_seed=1, min_particle_gap=1.0, initial_particle_buffer=0.0,
              z_wall_particle_buffer=8.0, domain_decomposition=(1, 1, 1), rebuild_neigh_list_freq=10,
              particle_collision_params=2.0, video_freq=10 ** 9, shear_stress_freq=10 ** 9,
              console_print_freq=10 ** 9)
    hs = d3.HostState(d3.parse_config(d3.keywords_text(kw)), data_dir=os.getcwd())
    ip = hs.cfg.ip
    n = args.steps
    interior = (ip.LatticeSize[0] - 2) * (ip.LatticeSize[1] - 2) * (ip.LatticeSize[2] - 2)
    out = {}
    for label, over in (("fp64", dict(arithmetic=2)), ("fp32", {}), ("fp16", dict(storage=1)),
                        ("bf16", dict(storage=2))):
        sim = d3.Simulation.from_host_state(hs, device=0, **over)
        stream = torch.cuda.ExternalStream(sim.stream_ptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.run(1, n)
        e1.record(stream)
        sim.synchronize()
        ms = e0.elapsed_time(e1)
        np_ = ip.NumParticles
        pff = sim.read_parfluidforce().reshape(2, np_, ip.WorkGroupsPerParticle, 4).astype(np.float64).sum(axis=2)
        out[label] = dict(u=sim.read_u().astype(np.float64), stress=sim.mean_stress(), pff=pff[:, :, :3],
                          mlups=interior * n / (ms * 1e-3) / 1e6)
        sim.close()
    ref = out["fp64"]

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    table = {}
    for label in ("fp32", "fp16", "bf16"):
        o = out[label]
        table[label] = {"u_rel_l2": rel(o["u"], ref["u"]),
                        "mean_stress_rel": abs(o["stress"][0] - ref["stress"][0]) / abs(ref["stress"][0]),
                        "eff_viscosity_rel": abs(o["stress"][2] - ref["stress"][2]) / abs(ref["stress"][2]),
                        "sphere_force_rel_l2": rel(o["pff"][0], ref["pff"][0]),
                        "sphere_torque_rel_l2": rel(o["pff"][1], ref["pff"][1]),
                        "mlups": round(o["mlups"], 1)}
    return {"metric": "error vs FP64 build", "impl": "ours", "n_gpus": 1, "steps": n,
            "config": {"workload": "casson-256x128x256", "spheres": ip.NumParticles,
                       "markers_per_sphere": ip.PointsPerParticle,
                       "description": "regularised Casson (tau_Y 1e-4, plastic tau 0.6), 1000 spheres r=6, "
                                      "walls +-0.04"},
            "fp64_mlups": round(ref["mlups"], 1), "fp64_eff_viscosity": ref["stress"][2], "errors": table}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="suspension-128", choices=sorted(WORKLOADS) + ["batch-64",
                                                                                           "served-sweep",
                                                                                           "served-preempt",
                                                                                           "casson-precision",
                                                                                           "pool-mix"])
    ap.add_argument("--requests", type=int, default=128, help="served-sweep: number of requests")
    ap.add_argument("--edges", type=int, nargs=2, default=[32, 64], metavar=("LO", "HI"),
                    help="served-sweep: range of the cubic edges drawn")
    ap.add_argument("--max-steps", type=int, default=40000, help="served-sweep: step cap of a solve")
    ap.add_argument("--solo-nodes", type=int, default=1 << 20,
                    help="served-sweep: requests with at least this many interior nodes run on contexts of their "
                         "own beside the pool (0: every request joins the pool)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fluid-kernel", default="tile", choices=sorted(FLUID_KERNELS),
                    help="collide-stream kernel: tile (the per-tile kernel) or tma (the TMA-pipelined kernel "
                         "where the lattice allows it)")
    ap.add_argument("--two-buffers", action="store_true",
                    help="the reference's two distribution buffers instead of one updated in place (AA pattern); "
                         "the results are bit-identical either way")
    ap.add_argument("--storage", default="fp32", choices=sorted(STORAGE),
                    help="distribution storage: fp32 (the reference's), or 16-bit shifted")
    args = ap.parse_args()
    args.inplace = not args.two_buffers
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_arm(args)), flush=True)
        return
    if args.workload in ("batch-64", "served-sweep", "served-preempt", "casson-precision", "pool-mix"):
        if rank == 0:
            run = {"batch-64": run_batch, "served-sweep": run_served, "served-preempt": run_served_preempt,
                   "casson-precision": run_precision, "pool-mix": run_pool_mix}
            print(json.dumps(run[args.workload](args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    try:
        out = run_ours(args, rank, world, local_rank, dist)
    finally:
        if dist:
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
