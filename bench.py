#!/usr/bin/env python
"""MPD-RDME throughput on the crowded-cell workload (B200).

One bench step = 40 MPD timesteps (x, y, z sweeps, reaction, overflow
handling) of the 128x128x256 crowded cell (10 nm, 8 site types with 20 %
obstacles, 200 species, 500 first- and second-order reactions, 1M particles,
IntLattice 16 slots, tau = 10 us), a segment of that model's 5,000-timestep
trajectory.  Inputs are seeded and synthetic (lattice_microbes_b200.configs.
config2).  --workload rodcell runs the 64x64x128 rod-cell model (ByteLattice
8 slots, configs.config1) the same way, 500 timesteps per bench step;
--workload batch / cme / serve run the batched, CME-ensemble and serving
forms; --workload trajectory runs the rod-cell model as a trajectory written
to a `.lm` file (species counts and a device lattice frame every 100
timesteps through the file's writer thread).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 is launched through torch.distributed.run: every rank runs its own
replicate (its own seed) on its own GPU with no data exchange (replicas only);
the value is all ranks' site-steps over the slowest rank's device time.

--impl reference times the reference's own CPU RDME solver on the host
cores: lm::rdme::NextSubvolumeSolver compiled from the reference sources
(oracle/_ref), one trajectory of the same workload per host core as
ReplicateRunner runs replicates, each bench step one stretch of simulated
time timed by the trajectory's own species-count records; its site-steps are
sites x simulated time / tau.  The default run reports the same figure as
cpu_baseline, and beside it the reference's MPD device functions compiled
for the host (the reference has no CPU MPD solver of its own).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-steps/s"
L2_FLUSH_BYTES = 256 << 20    # larger than the 126 MB L2

# Single-lattice workloads.  S slots of b bytes per site: the reference
# schedule moves B_sweep = 2 S b + 1 bytes per site per sweep and
# B_step = 7 S b + 4 per site-step (three sweeps + the reaction read).
WORKLOADS = {
    "bimolecular": dict(
        desc="bimolecular A + B <-> C, 32x32x32 ByteLattice-8, 1 site type, 1000 A + 1000 B, "
             "10,000 timesteps of 50 us per step",
        config="config0", S=8, b=1, tau=50e-6, dtype="u8", timesteps_per_step=10000, ref_timesteps=1000,
        nsm_seg=0.25, nsm_segments=8, ref_mpd_timesteps=600,
        l2="flushed between timed steps (256 MB write); working set 0.3 MB is L2-resident within a step"),
    "rodcell": dict(
        desc="rod-cell 64x64x128 ByteLattice-8, 3 site types, 5 species, 8 reactions, 5400 particles",
        config="config1", S=8, b=1, tau=25e-6, dtype="u8", timesteps_per_step=500, ref_timesteps=1000,
        nsm_seg=0.005, nsm_segments=8, ref_mpd_timesteps=60,
        l2="flushed between timed steps (256 MB write); working set 9 MB is L2-resident within a step"),
    "crowded": dict(
        desc="crowded cell 128x128x256 IntLattice-16, 8 site types (20% obstacles), 200 species, "
             "500 reactions, 1M particles",
        config="config2", S=16, b=4, tau=10e-6, dtype="u32", timesteps_per_step=40, ref_timesteps=100,
        nsm_seg=1e-6, nsm_segments=20, ref_mpd_timesteps=2,
        l2="inputs larger than L2: 537 MB of particle buffers + 4 MB site types per timestep"),
}


# The largest single-GPU configuration: the crowded cell.
DEFAULT_WORKLOAD = "crowded"


def make_spec(workload, seed):
    from lattice_microbes_b200 import configs
    return getattr(configs, WORKLOADS[workload]["config"])(seed=seed)


def b_sweep(w):
    return 2 * w["S"] * w["b"] + 1


def b_step(w):
    return 7 * w["S"] * w["b"] + 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--timesteps-per-step", type=int, default=0, help="0 = the workload's default")
    ap.add_argument("--cpu-sample-timesteps", type=int, default=0,
                    help="timesteps per core of the reference MPD functions on the host (0 = auto)")
    ap.add_argument("--cpu-sample-time", type=float, default=0.0,
                    help="simulated seconds per timed stretch of the reference NextSubvolumeSolver (0 = auto)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference kernels on the GPU (e.g. under a profiler)")
    ap.add_argument("--e2e-depth", type=int, default=3,
                    help="solves in flight in the end-to-end measurement (lattices it rotates over)")
    ap.add_argument("--schedule", choices=["auto", "fused", "phases", "cluster", "grid"], default="auto")
    ap.add_argument("--workload", choices=["crowded", "rodcell", "bimolecular", "batch", "cme", "serve", "trajectory",
                                           "pair"],
                    default=DEFAULT_WORKLOAD,
                    help="crowded: one 128x128x256 IntLattice-16 (default); rodcell: one 64x64x128 ByteLattice-8; "
                         "bimolecular: the plain 32x32x32 A + B <-> C run, 10,000 timesteps per step; "
                         "batch: 256 bimolecular replicates of "
                         "uneven size in one launch per timestep; cme: 65,536 two-state gene replicates "
                         "(direct method) to t = 3600 s; serve: a Poisson stream of solve requests; trajectory: "
                         "the rod cell with its records written to a .lm file")
    ap.add_argument("--replicates", type=int, default=0, help="batch: 256, cme: 65536 (0 = default)")
    ap.add_argument("--requests", type=int, default=1000,
                    help="serve: requests of the stream to replay (the whole 1000-request stream takes about 30 "
                         "minutes for both arms; fewer replay its head)")
    return ap.parse_args()


# --------------------------------------------------------------------------
# CPU side: the reference's code on the host cores
# --------------------------------------------------------------------------

class stdout_to_stderr:
    """Sends what the reference's code prints on standard output (its
    Print::printf warnings) to standard error while it runs, at the file
    descriptor level, so that standard output holds only the JSON line.
    Worker processes started inside inherit the redirection."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def host_cores():
    """Host threads this process may run on."""
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_worker(args):
    """One replicate of the reference MPD device functions on one core (spawned)."""
    workload, seed, timesteps = args
    sys.path.insert(0, ROOT)
    from tests.cases import oracle_tables
    from tests.oracle_lib import reference_run
    spec = make_spec(workload, seed)
    t = oracle_tables(spec)
    t0 = time.perf_counter()
    r = reference_run(t, spec.lattice, spec.sites, 1000 + seed, 0, timesteps)
    dt = time.perf_counter() - t0
    if r is None:
        return None
    return dt, int(r[1]), spec.nsites


def cpu_reference_sample(workload, timesteps, cores):
    """Reference MPD device functions, `cores` replicates in parallel;
    returns (site-steps/s, sample)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_cpu_worker, [(workload, s, timesteps) for s in range(cores)])
    if any(r is None for r in res):
        return None, "reference checker not built (oracle/_ref)"
    wall = max(r[0] for r in res)
    value = res[0][2] * timesteps * cores / wall
    sample = ("%d replicates x %d timesteps of the %s workload, one per core, reference device "
              "functions compiled for the host; %.1f s wall" % (cores, timesteps, workload, wall))
    return value, sample


def _byte_lattice(spec):
    """The spec's particles in a ByteLattice with the same slot count (the
    reference NextSubvolumeSolver runs ByteLattices only; ids <= 255)."""
    import numpy as np
    from lattice_microbes_b200 import configs
    if spec.bytes_per_slot == 1:
        return spec
    N = spec.nsites
    slots = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat = configs.empty_lattice(spec.X, spec.Y, spec.Z, spec.slots, 1)
    for k in range(spec.slots):
        lat[(k // 4) * N:(k // 4 + 1) * N] |= slots[:, k].astype(np.uint32) << np.uint32(8 * (k % 4))
    spec.lattice, spec.bytes_per_slot = lat, 1
    return spec


def _nsm_worker(args):
    """One replicate of the reference NextSubvolumeSolver on one core
    (spawned): one trajectory of `segments` stretches of `seg_time` simulated
    seconds, with a species-count record at the end of each.  The records'
    wall-clock stamps time the stretches; the solver's set-up (lattice, queue,
    every subvolume's propensities) comes before the first record and is not
    timed."""
    workload, seed, seg_time, segments = args
    sys.path.insert(0, ROOT)
    from tests import ref_cpu_lib
    if not ref_cpu_lib.available():
        return None
    spec = _byte_lattice(make_spec(workload, seed))
    ref_cpu_lib.nsm_run(spec, 1000 + seed, seed + 1, seg_time * segments, seg_time)
    walls = ref_cpu_lib.record_walls()
    if len(walls) < segments + 1:
        return None
    return [float(x) for x in walls[:segments + 1]], spec.nsites


def cpu_nsm_sample(workload, seg_time, segments, skip, cores):
    """Reference NextSubvolumeSolver, `cores` replicates of the workload in
    parallel, each one trajectory of `segments` stretches of `seg_time`
    simulated seconds, the first `skip` stretches untimed.  Returns
    (site-steps/s, sample, per-stretch site-steps/s) with site-steps = sites x
    simulated time / tau over the slowest core's wall time."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_nsm_worker, [(workload, s, seg_time, segments) for s in range(cores)])
    if any(r is None for r in res):
        return None, "reference CPU solvers not built (oracle/_ref)", []
    tau = WORKLOADS[workload]["tau"]
    N = res[0][1]
    timed = segments - skip
    wall = max(r[0][segments] - r[0][skip] for r in res)
    value = N * (timed * seg_time / tau) * cores / wall
    per = [N * (seg_time / tau) * cores / max(r[0][k + 1] - r[0][k] for r in res) for k in range(skip, segments)]
    sample = ("%d replicates of the %s workload, one per core, each one trajectory of %d stretches of %.4g s of "
              "simulated time (%.4g MPD-timestep equivalents each), the first %d untimed; reference "
              "NextSubvolumeSolver built from its sources; %.1f s wall over the timed stretches, the solver's "
              "set-up excluded" % (cores, workload, segments, seg_time, seg_time / tau, skip, wall))
    return value, sample, per


# --------------------------------------------------------------------------
# Clocks during the timed region
# --------------------------------------------------------------------------

class ClockSampler:
    """SM clocks, power and clock-event reasons of `device` during a timed
    region: read through NVML every 20 ms on a background thread (reads
    only; no setting is touched), or from nvidia-smi's 200 ms log when NVML
    is not available."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None
        self.thread = None
        self.samples = []

    def _nvml_start(self):
        import threading
        import pynvml as nv
        nv.nvmlInit()
        try:
            import torch
            index = torch.cuda._get_nvml_device_index(self.device)
        except Exception:
            index = self.device
        h = nv.nvmlDeviceGetHandleByIndex(index)
        self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        self.stop_flag = threading.Event()

        def run():
            while not self.stop_flag.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, [k for k, v in bits.items() if r & v]))
                except Exception:
                    pass
                self.stop_flag.wait(0.02)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def start(self):
        try:
            self._nvml_start()
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            sm = [float(v) for v, _ in self.samples]
            if sm:
                out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = float(self.max_mhz)
            out["reasons"] = sorted({k for _, ks in self.samples for k in ks})
            out["samples"] = len(sm)
            out["source"] = "nvml, 20 ms"
            return out
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(self.REASONS):
                if r[5 + k].strip() == "Active":
                    reasons.add(nm)
        if sm:
            out["sm_mhz"] = statistics.median(sm)
        if mx:
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        out["source"] = "nvidia-smi, 200 ms"
        return out


def measured_peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic_per_launch(workload, kernel):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu
    summary (profiles/traffic.json), if any."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        e = d.get(workload) or {}
        return e.get("kernel_dram_bytes_per_launch") if e.get("kernel", "").startswith(kernel) else None
    except Exception:
        return None


# --------------------------------------------------------------------------
# Our arm
# --------------------------------------------------------------------------

def run_ours(a):
    import numpy as np
    import torch

    from lattice_microbes_b200.replicas import Ranks, aggregate_rate
    ranks = Ranks()
    world, rank, local = ranks.world, ranks.rank, ranks.local
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    ranks.init("nccl")

    # CPU baseline first (spawned workers, before any GPU work on this rank).
    w = WORKLOADS[a.workload]
    cpu = None
    cpu_mpd = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = host_cores()
        with stdout_to_stderr():
            val, sample, _ = cpu_nsm_sample(a.workload, a.cpu_sample_time or w["nsm_seg"], w["nsm_segments"] + 1,
                                            1, cores)
        if val is not None:
            cpu = {"value": val, "unit": METRIC, "cores": cores, "kind": "reference", "sample": sample}
        with stdout_to_stderr():
            val, sample = cpu_reference_sample(a.workload, a.cpu_sample_timesteps or w["ref_mpd_timesteps"],
                                               cores)
        if val is not None:
            cpu_mpd = {"value": val, "unit": METRIC, "cores": cores, "sample": sample}

    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.solver import Context, Lattice, Model, kernel_launches

    T = a.timesteps_per_step or w["timesteps_per_step"]
    spec = make_spec(a.workload, 1 + rank)
    N = spec.nsites
    B_SWEEP, B_STEP = b_sweep(w), b_step(w)
    ctx = Context(device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", device))
    model = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice, spec.sites)
    seed = ranks.seed(2024)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    # The reference's own kernels (compiled for sm_100a from its sources) on
    # this GPU, with its per-timestep host flow: the GPU bar to beat.
    ref_gpu = None
    if rank == 0 and not a.no_reference_gpu:
        try:
            from tests.cases import oracle_tables
            from tests.oracle_lib import reference_gpu_time
            nref = w["ref_timesteps"]
            with stdout_to_stderr():
                r = reference_gpu_time(oracle_tables(spec), spec.lattice, spec.sites, seed, 0, nref)
            if r is not None and r[0] == 0:
                ref_gpu = {"value": N * nref / (r[1] / 1e3), "unit": METRIC, "timesteps": nref,
                           "what": "reference device functions built for sm_100a, reference host loop "
                                   "(4 launches + stream sync + overflow check per timestep)"}
        except Exception as e:  # checker absent: report why
            ref_gpu = {"unavailable": str(e)[:200]}

    from lattice_microbes_b200 import _lib as LL
    tuned = None
    if a.schedule == "phases":
        lat.set_schedule(LL.LMB_SCHEDULE_PHASES)
    elif a.schedule == "cluster":
        lat.set_schedule(LL.LMB_SCHEDULE_CLUSTER)
    elif a.schedule == "grid":
        lat.set_schedule(LL.LMB_SCHEDULE_GRID)
    elif a.schedule == "fused" or a.no_autotune:
        lat.set_schedule(LL.LMB_SCHEDULE_FUSED)
    else:
        tuned = lat.autotune(model, seed, 0, 100)
    sched = lat.schedule()
    sched_name = {LL.LMB_SCHEDULE_FUSED: "fused Ty=%d Tz=%d" % (sched[1], sched[2]),
                  LL.LMB_SCHEDULE_CLUSTER: "cluster (whole lattice in one thread-block cluster, one launch per run)",
                  LL.LMB_SCHEDULE_GRID: "grid Ty=%d Tz=%d (every fused tile resident at once, one launch per run)"
                                        % (sched[1], sched[2]),
                  }.get(sched[0], "phases")

    step = 0
    for _ in range(a.warmup):
        lat.run(model, seed, step, T)
        step += T

    # ---- device-timed throughput (inputs resident in HBM) ----
    clocks = ClockSampler(device)
    times = []
    ranks.barrier()
    torch.cuda.synchronize(device)
    launches0 = kernel_launches()
    clocks.start()
    with torch.cuda.stream(stream):
        for _ in range(a.steps):
            flush.fill_(1.0)  # L2 flush between timed steps, outside the events
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            lat.run_async(model, seed, step, T)
            e1.record(stream)
            lat.wait()
            times.append(e0.elapsed_time(e1))
            step += T
    torch.cuda.synchronize(device)
    clock_info = clocks.stop()
    launches = kernel_launches() - launches0
    ranks.barrier()
    ms_total = ranks.max(sum(times), device)
    value = aggregate_rate(N * T * a.steps, ms_total, world)

    # ---- per-kernel device times (roofline of the dominant kernel) ----
    st, phase_ms, phase_n = lat.run_profiled(model, seed, step, T)
    step += T
    # The profiled run brackets every launch with events (no graph replay), so
    # its absolute times run long; only its shares are used, applied to the
    # device-timed, graph-replayed bench step: per-launch times below sum to
    # ms_per_step.
    names = ["sweep_x", "sweep_y", "sweep_z", "reaction", "overflow", "fused_step"]
    total_ms = float(phase_ms.sum())
    step_ms = ms_total / a.steps                  # T timesteps, as the profiled run
    phases = {names[k]: {"launches": int(phase_n[k]),
                         "ms_per_launch": step_ms * float(phase_ms[k]) / total_ms / int(phase_n[k]),
                         "share": float(phase_ms[k]) / total_ms,
                         "profiled_ms_per_launch": float(phase_ms[k]) / int(phase_n[k])}
              for k in range(6) if phase_n[k] > 0}
    peak, peak_kind = measured_peak_hbm()
    sweep_fraction = None
    if phase_n[5] > 0:
        kern = ("cluster_run_kernel (every timestep of the run in one launch; per timestep)"
                if sched[0] == LL.LMB_SCHEDULE_CLUSTER else
                "fused_grid_kernel (every timestep of the run in one launch; per timestep)"
                if sched[0] == LL.LMB_SCHEDULE_GRID else
                "fused_step_kernel (x, y, z sweeps + reaction + overflow, one timestep)")
        launch_ms = phases["fused_step"]["ms_per_launch"]
        alg_bytes = N * B_STEP                 # site-steps per launch x per-site-step bytes
        own_bytes = N * B_SWEEP                # its own dataflow: read slots + site type, write slots
    else:
        kern = "sweep_pp_kernel (x, y, z hop sweeps by particle)"
        sweep_share = float(phase_ms[:3].sum()) / total_ms
        launch_ms = step_ms * sweep_share / max(1, int(phase_n[:3].sum()))
        alg_bytes = N * B_SWEEP
        # With plane bounds a sweep moves only the planes that can hold
        # particles: its own dataflow is the ncu DRAM traffic, when recorded.
        own_bytes = ncu_traffic_per_launch(a.workload, "sweep") or alg_bytes
        sweep_fraction = alg_bytes / (launch_ms / 1e3) / 1e9 / peak
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9
    # ---- end to end through the public API with host buffers ----
    # Every step is one solve: its input lattice and site types copied from
    # pinned host memory, T timesteps, the final lattice copied back into
    # pinned host memory (lmb_run_native_async).  The solves rotate over
    # `depth` lattices on as many contexts (streams), each step's solve
    # queued while the ones before run, so that the copies of some solves
    # overlap the timesteps of others (a lattice's own upload waits for its
    # previous download on its stream); the clock runs from the first call
    # to the last solve's end (wall clock).
    depth = max(1, a.e2e_depth)
    words = spec.words * N
    h_lat = torch.from_numpy(spec.lattice.copy()).pin_memory()
    h_sites = torch.from_numpy(spec.sites.copy()).pin_memory()
    h_out = [torch.empty(words, dtype=torch.int32).pin_memory() for _ in range(depth)]
    extra = []
    ring = [lat]
    for _ in range(depth - 1):
        c_ = Context(device)
        l_ = Lattice(c_, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
        l_.set_schedule(*sched)
        l_.set_native(spec.lattice, spec.sites)
        extra.append((c_, l_))
        ring.append(l_)
    for k in range(depth):  # graphs captured and buffers touched before the clock starts
        ring[k].run_native_async(model, seed, 0, T, h_lat.data_ptr(), h_sites.data_ptr(), h_out[k].data_ptr())
        ring[k].wait()
    torch.cuda.synchronize(device)
    ranks.barrier()
    t0 = time.perf_counter()
    for k in range(a.steps):
        if k >= depth:
            ring[k % depth].wait()
        ring[k % depth].run_native_async(model, seed, 0, T, h_lat.data_ptr(), h_sites.data_ptr(),
                                         h_out[k % depth].data_ptr())
    for k in range(min(depth, a.steps)):
        ring[(a.steps - 1 - k) % depth].wait()
    e2e_total = ranks.max((time.perf_counter() - t0) * 1e3, device)
    e2e_value = aggregate_rate(N * T * a.steps, e2e_total, world)
    for c_, l_ in extra:
        l_.close()
        c_.close()

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": METRIC,
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": ms_total / a.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": w["dtype"],
            "data": "synthetic (seeded, lattice_microbes_b200.configs.%s)" % w["config"],
            "config": {
                "workload": w["desc"],
                "timesteps_per_step": T,
                "sites": N,
                "parallelism": "replicas" if world > 1 else "single",
                "schedule": sched_name,
                "autotune_ms": None if tuned is None else tuned[3],
                "l2": w["l2"],
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peak,
                "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": ncu_traffic_per_launch(a.workload, "fused_step_kernel" if phase_n[5] > 0 else "sweep"),
                "kernel": kern,
                "ms_per_launch": launch_ms,
                "algorithmic_bytes_per_launch": alg_bytes,
                "own_dataflow_bytes_per_launch": own_bytes,
                "own_dataflow_frac": own_bytes / (launch_ms / 1e3) / 1e9 / peak,
                "peak_kind": peak_kind,
                "note": (("achieved = N x B_step (reference-schedule bytes of a site-step) per fused launch / "
                          "launch time; own_dataflow_frac counts the fused kernel's single read and write of the "
                          "lattice" if phase_n[5] > 0 else
                          "achieved = N x B_sweep (reference-schedule bytes of a site's sweep) per sweep launch / "
                          "sweep launch time; the sweeps keep per-segment plane bounds and move only the word "
                          "planes that can hold particles, so own_dataflow_frac (ncu DRAM bytes per launch) is far "
                          "below it and the sweeps are bound by instruction issue and latency, not HBM") +
                         "; launch times are the device-timed step x the kernel's share of device time in an "
                         "event-bracketed run" + {"rodcell": "; working set 9 MB is L2-resident",
                                                 "bimolecular": "; working set 0.3 MB is L2-resident"}.get(
                                                     a.workload, "")),
                "phases": phases,
                "sweep_fraction": sweep_fraction,
                "step_fraction_reference_schedule": value * B_STEP / (peak * 1e9),
            },
            "e2e": {
                "value": e2e_value,
                "unit": METRIC,
                "h2d_bytes_per_step": int(words * 4 + N),
                "d2h_bytes_per_step": int(words * 4),
                "what": "one solve per step through lmb_run_native_async (input lattice and site types from "
                        "pinned host memory, %d timesteps, final lattice to pinned host memory), solves "
                        "rotating over %d lattices on as many streams so that copies overlap timesteps; "
                        "wall clock" % (T, depth),
                "solves_in_flight": depth,
            },
            "gpu_launches": int(launches),
            "clocks": clock_info,
            "cpu_baseline": cpu,
            "reference_mpd_on_host_cores": cpu_mpd,
            "reference_kernels_b200": ref_gpu,
            "run_stats": {"overflows": int(st.overflows), "reactions_per_step": int(st.reactions)},
        }
        print(json.dumps(line), flush=True)
    lat.close()
    model.close()
    ctx.close()
    ranks.finish()


def run_reference(a):
    """The reference's CPU RDME solver on the host cores, same workload and
    metric as our arm: one NextSubvolumeSolver trajectory per core, each
    bench step one stretch of simulated time (min(W, 1) untimed stretch
    first), timed by the trajectory's own records."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wname = a.workload if a.workload in WORKLOADS else DEFAULT_WORKLOAD
    w = WORKLOADS[wname]
    cores = host_cores()
    seg = a.cpu_sample_time or w["nsm_seg"]
    skip = min(a.warmup, 1)
    with stdout_to_stderr():
        value, sample, per = cpu_nsm_sample(wname, seg, a.steps + skip, skip, cores)
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return
    spec_sites = make_spec(wname, 1).nsites
    T = a.timesteps_per_step or w["timesteps_per_step"]
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": spec_sites * T / value * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": w["dtype"],
        "data": "synthetic (seeded, lattice_microbes_b200.configs.%s)" % w["config"],
        "config": {"workload": w["desc"], "timesteps_per_step": T, "sites": spec_sites,
                   "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": cores, "kind": "reference",
                         "sample": sample},
        "per_step_values": per,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch(a):
    """Batched replicates: config-0 chemistry (A + B <-> C, 32 nm, tau = 50 us)
    on cubic lattices with edges drawn from {16, 24, 32, 48, 64}, all advanced
    by one launch per timestep with tile shapes chosen per edge by the batch
    autotuner.  Metric: replicates/s, a replicate being one 10,000-timestep
    trajectory.  Compared with the plain solver running the same replicates
    one after another, each with the schedule its own autotuner picks for its
    edge, over the same timesteps."""
    import torch

    from lattice_microbes_b200 import _lib as LL
    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.solver import Batch, Context, Lattice, Model, compose_seed, kernel_launches

    torch.cuda.set_device(0)
    T = a.timesteps_per_step or 200
    edges = configs.batch_edges(seed=7, count=a.replicates or 256)
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    lats, models, specs = [], [], []
    for k, e in enumerate(edges):
        spec = configs.config0(seed=k + 1, edge=e)
        m = Model.from_spec(ctx, spec)
        lat = Lattice(ctx, e, e, e, 8, 1)
        lat.set_native(spec.lattice, spec.sites)
        lats.append(lat)
        models.append(m)
        specs.append(spec)
    seeds = [compose_seed(2024, k) for k in range(len(lats))]
    sites_total = sum(e ** 3 for e in edges)
    batch = Batch(ctx, lats, models)
    t0 = time.perf_counter()
    batch.autotune(seeds, 0, 16)
    tune_s = time.perf_counter() - t0
    plan = {}
    for e, (ty, tz) in zip(edges, batch.plan()):
        plan[str(e)] = "%dx%d" % (ty, tz)
    step = 0
    for _ in range(a.warmup):
        batch.run(seeds, step, T)
        step += T
    times = []
    launches0 = kernel_launches()
    clocks = ClockSampler(0)
    clocks.start()
    # An NVTX range marks the timed launches for a profiler's filter.
    rng = torch.cuda.nvtx.range_start("batch timed")
    with torch.cuda.stream(stream):
        for _ in range(a.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.run_async(seeds, step, T)
            e1.record(stream)
            batch.wait()
            times.append(e0.elapsed_time(e1))
            step += T
    torch.cuda.nvtx.range_end(rng)
    clock_info = clocks.stop()
    launches = kernel_launches() - launches0
    ms_step = sum(times) / a.steps / T                       # per timestep, all replicates
    rep_per_s = len(lats) / (10000 * ms_step / 1e3)

    # Plain solver, one replicate after another on the same stream: each edge's
    # schedule from the single-lattice autotuner, every replicate run for the
    # same T timesteps (one untimed pass first: graph capture).
    sched = {}
    for e in sorted(set(edges)):
        k = edges.index(e)
        s_, ty, tz, _ = lats[k].autotune(models[k], seeds[k], step, 32)
        sched[e] = (s_, ty, tz)
    for lat, e in zip(lats, edges):
        lat.set_schedule(*sched[e])
    for lat, m, sd in zip(lats, models, seeds):
        lat.run(m, sd, step, T)
    step += T
    with torch.cuda.stream(stream):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for lat, m, sd in zip(lats, models, seeds):
            lat.run_async(m, sd, step, T)
        e1.record(stream)
        for lat in lats:
            lat.wait()
    seq_ms_step = e0.elapsed_time(e1) / T
    seq_rep_per_s = len(lats) / (10000 * seq_ms_step / 1e3)
    line = {
        "metric": "replicates/s",
        "value": rep_per_s,
        "unit": "replicates/s",
        "n_gpus": 1,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": sum(times) / a.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic (seeded bimolecular replicates, lattice_microbes_b200.configs.config0)",
        "config": {"workload": "batch of %d bimolecular replicates, edges {16,24,32,48,64}, %d sites"
                               % (len(lats), sites_total),
                   "timesteps_per_step": T, "trajectory_timesteps": 10000,
                   "batch_plan_by_edge": plan, "autotune_s": tune_s},
        "site_steps_per_s": sites_total / (ms_step / 1e3),
        "sequential_plain": {"value": seq_rep_per_s, "unit": "replicates/s",
                             "what": "all %d replicates, one after another, %d timesteps each" % (len(lats), T),
                             "schedule_by_edge": {str(e): ("fused %dx%d" % (v[1], v[2]) if v[0] == LL.LMB_SCHEDULE_FUSED else
                                                           "cluster" if v[0] == LL.LMB_SCHEDULE_CLUSTER else
                                                           "grid %dx%d" % (v[1], v[2]) if v[0] == LL.LMB_SCHEDULE_GRID
                                                           else "phases")
                                                  for e, v in sched.items()}},
        "speedup_vs_sequential": rep_per_s / seq_rep_per_s,
        "gpu_launches": int(launches),
        "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)
    batch.close()
    for lat, m in zip(lats, models):
        lat.close()
        m.close()
    ctx.close()


def _gd_worker(args):
    """Reference GillespieDSolver replicates on one core (spawned)."""
    first, count = args
    sys.path.insert(0, ROOT)
    from lattice_microbes_b200 import configs
    from tests import ref_cpu_lib
    if not ref_cpu_lib.available():
        return None
    m = configs.two_state_gene()
    t0 = time.perf_counter()
    for k in range(first, first + count):
        ref_cpu_lib.gillespie_run(m.ns, m.rtype, m.K, m.S, m.D, m.init, 77, k + 1, m.max_time, m.write_interval)
    return time.perf_counter() - t0


def cpu_gillespie_sample(per_core, cores):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_gd_worker, [(c * per_core, per_core) for c in range(cores)])
    if any(r is None for r in res):
        return None, "reference CPU solvers not built (oracle/_ref)"
    wall = max(res)
    value = per_core * cores / wall
    return value, ("%d replicates per core on %d cores of the two-state gene model to t = 3600 s, reference "
                   "GillespieDSolver built from its sources; %.1f s wall" % (per_core, cores, wall))


def run_cme(a):
    """GillespieD CME ensemble: 65,536 replicates of the two-state gene model
    (configs.two_state_gene) to t = 3600 s, counts every 600 s, one GPU
    thread per replicate.  Metric: replicates/s (trajectories to 3600 s)."""
    import numpy as np
    import torch

    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.solver import CMEEnsemble, Context, kernel_launches

    reps = a.replicates or 65536
    cores = host_cores()
    cpu = None
    if not a.no_cpu_baseline:
        with stdout_to_stderr():
            v, sample = cpu_gillespie_sample(1500, cores)
        if v is not None:
            cpu = {"value": v, "unit": "replicates/s", "cores": cores, "kind": "reference", "sample": sample}
    torch.cuda.set_device(0)
    ctx = Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    m = configs.two_state_gene()
    ens = CMEEnsemble(ctx, m, reps)
    for k in range(a.warmup):
        ens.run(1000 + k, m.max_time, m.write_interval)
    times, events = [], 0
    launches0 = kernel_launches()
    clocks = ClockSampler(0)
    clocks.start()
    with torch.cuda.stream(stream):
        for k in range(a.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            ens.begin(k + 1, m.max_time, m.write_interval)
            e0.record(stream)
            ens.advance_async(m.max_time)
            e1.record(stream)
            torch.cuda.synchronize(0)
            times.append(e0.elapsed_time(e1))
            events += ens.stats()[0]
    clock_info = clocks.stop()
    launches = kernel_launches() - launches0
    ms = sum(times) / a.steps
    value = reps / (ms / 1e3)
    # End to end through the public API: initial counts in, records out.
    init = np.tile(m.init, (reps, 1)).astype(np.uint32)
    e2e = []
    for k in range(a.steps):
        t0 = time.perf_counter()
        ens.set_initial_counts(init)
        ens.run(k + 1, m.max_time, m.write_interval)
        out = ens.counts()
        e2e.append(time.perf_counter() - t0)
    entries = ens.entries()
    ens.close()
    ctx.close()
    line = {
        "metric": "replicates/s",
        "value": value,
        "unit": "replicates/s",
        "n_gpus": 1,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int32 counts, f32 propensities, f64 time",
        "data": "synthetic (two-state gene model, lattice_microbes_b200.configs.two_state_gene)",
        "config": {"workload": "GillespieD CME ensemble, %d replicates of the two-state gene model to t = 3600 s, "
                               "counts every 600 s" % reps,
                   "l2": "state and records (%d MB) are L2-resident; the kernel is issue-bound" %
                         max(1, reps * (entries * 4 * 4 + 64) >> 20)},
        "events_per_s": events / a.steps / (ms / 1e3),
        "e2e": {"value": reps / (sum(e2e) / a.steps), "unit": "replicates/s",
                "h2d_bytes_per_step": int(init.nbytes), "d2h_bytes_per_step": int(out.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clock_info,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_serve(a):
    """Serving: the first --requests requests of a seeded Poisson stream
    (50 req/s; edges 16..128, 2..50 species, 0.5..2 particles per site,
    1k..20k timesteps; configs.serve_stream) replayed at their arrival times
    into the solve server (continuous batching, 150 GB budget, ByteLattice
    16 slots).  Compared with sequential plain runs: the same requests solved
    one at a time in arrival order (lmb_run each), each timed over the same
    per-request work as a served solve (set-up, upload, run, counts and
    lattice back, release), their latencies computed from the same arrival
    times."""
    import numpy as np
    import torch

    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.solver import Context, Lattice, Model, Server, compose_seed, kernel_launches

    torch.cuda.set_device(0)
    stream_reqs = configs.serve_stream(seed=4, count=a.requests)
    specs = []
    for r in stream_reqs:
        sp = configs.serve_problem(r)
        specs.append(_to_byte16(sp))
    seeds = [compose_seed(2024, r.index) for r in stream_reqs]
    site_steps = sum(float(s.nsites) * r.timesteps for s, r in zip(specs, stream_reqs))
    ctx = Context(0)
    # Warm-up: one small solve through the server.
    srv = Server(ctx, slots=16, bytes_per_slot=1, hbm_budget_bytes=150 << 30, max_active=256, chunk_timesteps=256)
    for k in range(a.warmup):
        srv.submit(10 ** 6 + k, specs[0], 1, 64)
    while True:
        act, q = srv.step()
        while srv.pop_result(with_lattice=False) is not None:
            pass
        if act == 0 and q == 0:
            break
    launches0 = kernel_launches()
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    submitted, done = 0, {}
    while len(done) < len(stream_reqs):
        now = time.perf_counter() - t0
        while submitted < len(stream_reqs) and stream_reqs[submitted].arrival <= now:
            r = stream_reqs[submitted]
            srv.submit(r.index, specs[submitted], seeds[submitted], r.timesteps)
            submitted += 1
        act, q = srv.step()
        while True:
            res = srv.pop_result(with_lattice=False)
            if res is None:
                break
            info = res[0]
            done[info.id] = (time.perf_counter() - t0, info.stats.status)
        if act == 0 and q == 0 and submitted < len(stream_reqs):
            time.sleep(max(0.0, stream_reqs[submitted].arrival - (time.perf_counter() - t0)))
    makespan = time.perf_counter() - t0
    clock_info = clocks.stop()
    launches = kernel_launches() - launches0
    st = srv.status()
    srv.close()
    lat = np.array([done[r.index][0] - r.arrival for r in stream_reqs])
    failed = sum(1 for v in done.values() if v[1] != 0)

    # Sequential plain solver: one solve at a time, arrival order.
    solo_s = []
    from lattice_microbes_b200 import _lib as LL
    for sp, r, sd in zip(specs, stream_reqs, seeds):
        # The same work per request as the server does for a solve: model
        # and lattice set-up (per-phase schedule for a large dense solve, as
        # the server gives it), upload, the run, the species counts and the
        # lattice copied back, device memory freed.
        torch.cuda.synchronize(0)
        s0 = time.perf_counter()
        m = Model.from_spec(ctx, sp)
        L2 = Lattice(ctx, sp.X, sp.Y, sp.Z, 16, 1)
        if sp.nsites >= (1 << 17) and r.density >= 0.05:
            L2.set_schedule(LL.LMB_SCHEDULE_PHASES)
        L2.set_native(sp.lattice, sp.sites)
        L2.run(m, sd, 0, r.timesteps)
        L2.species_counts(sp.ns)
        L2.get_native()
        L2.close()
        m.close()
        solo_s.append(time.perf_counter() - s0)
    finish, seq_lat = 0.0, []
    for r, d in zip(stream_reqs, solo_s):
        finish = max(finish, r.arrival) + d
        seq_lat.append(finish - r.arrival)
    seq_lat = np.array(seq_lat)
    ctx.close()
    line = {
        "metric": "solves/s",
        "value": len(stream_reqs) / makespan,
        "unit": "solves/s",
        "n_gpus": 1,
        "steps": 1,
        "warmup": a.warmup,
        "ms_per_step": makespan * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic (seeded Poisson request stream, lattice_microbes_b200.configs.serve_stream)",
        "config": {"workload": "serving: first %d requests of a 50 req/s Poisson stream, edges 16..128, 2..50 "
                               "species, 0.5..2 particles/site, 1k..20k timesteps, ByteLattice-16, 150 GB budget, "
                               "256 slots, 256-timestep chunks" % len(stream_reqs),
                   "site_steps": site_steps},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "mean": float(lat.mean())},
        "site_steps_per_s": site_steps / makespan,
        "peak_resident": {"solves": int(st.peak_active), "bytes": int(st.peak_bytes)},
        "failed": failed,
        "sequential_plain": {"solves_per_s": len(stream_reqs) / finish,
                             "latency_s": {"p50": float(np.percentile(seq_lat, 50)),
                                           "p99": float(np.percentile(seq_lat, 99))},
                             "site_steps_per_s": site_steps / sum(solo_s)},
        "speedup_vs_sequential": (len(stream_reqs) / makespan) / (len(stream_reqs) / finish),
        "e2e": {"value": len(stream_reqs) / makespan, "unit": "solves/s",
                "h2d_bytes_per_step": int(sum(s.lattice.nbytes + s.sites.nbytes for s in specs)),
                # Each retired solve's lattice and species counts come back.
                "d2h_bytes_per_step": int(sum(s.lattice.nbytes + 8 * (s.ns + 1) for s in specs))},
        "gpu_launches": int(launches),
        "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)


def run_pair(a):
    """Two large dense serving solves side by side against one after another:
    the measurement behind the served form's bound.  Each solve is a
    serving request of the largest kind (edge 128, ByteLattice-16, 2
    particles per site, 30 species) on the per-phase schedule the server
    gives large dense solves, T timesteps.  Side by side: two contexts (two
    streams), both runs enqueued before either is waited for, as the
    server's two solo streams run them.  One after another: the same two runs,
    the second enqueued after the first has finished.  Both arms are timed
    from the first enqueue to the last completion (best of --steps), with each
    stream's CUDA-event time beside them."""
    import torch

    from lattice_microbes_b200 import _lib as LL
    from lattice_microbes_b200 import configs
    from lattice_microbes_b200.solver import Context, Lattice, Model, compose_seed

    torch.cuda.set_device(0)
    T = a.timesteps_per_step or 200
    reqs = [configs.ServeRequest(index=k, arrival=0.0, edge=128, ns=30, density=2.0, timesteps=T, seed=900 + k)
            for k in range(2)]
    specs = [_to_byte16(configs.serve_problem(r)) for r in reqs]
    ctxs = [Context(0), Context(0)]
    models, lats = [], []
    for c, sp in zip(ctxs, specs):
        m = Model.from_spec(c, sp)
        lat = Lattice(c, sp.X, sp.Y, sp.Z, 16, 1)
        lat.set_schedule(LL.LMB_SCHEDULE_PHASES)
        lat.set_native(sp.lattice, sp.sites)
        models.append(m)
        lats.append(lat)
    seeds = [compose_seed(77, k) for k in range(2)]
    streams = [torch.cuda.ExternalStream(c.stream, device=torch.device("cuda", 0)) for c in ctxs]
    step = 0
    for _ in range(max(1, a.warmup)):
        for lat, m, sd in zip(lats, models, seeds):
            lat.run(m, sd, step, T)
        step += T

    def timed(side_by_side):
        nonlocal step
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2)]
        torch.cuda.synchronize(0)
        t0 = time.perf_counter()
        for k in range(2):
            with torch.cuda.stream(streams[k]):
                ev[k][0].record(streams[k])
                lats[k].run_async(models[k], seeds[k], step, T)
                ev[k][1].record(streams[k])
            if not side_by_side:
                lats[k].wait()
        for k in range(2):
            if side_by_side:
                lats[k].wait()
        wall = time.perf_counter() - t0
        step += T
        per = [e0.elapsed_time(e1) for e0, e1 in ev]
        return wall, per

    seq = [timed(False) for _ in range(a.steps)]
    par = [timed(True) for _ in range(a.steps)]
    seq_ms = min(w * 1e3 for w, _ in seq)
    par_ms = min(w * 1e3 for w, _ in par)
    sites = specs[0].nsites
    line = {
        "metric": "site-steps/s",
        "value": 2 * sites * T / (par_ms / 1e3),
        "unit": "site-steps/s",
        "n_gpus": 1,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": par_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8",
        "data": "synthetic (two seeded serving requests, lattice_microbes_b200.configs.serve_problem)",
        "config": {"workload": "two 128^3 ByteLattice-16 serving solves, 2 particles per site, 30 species, "
                               "per-phase schedule, %d timesteps each" % T},
        "one_after_another": {"ms": seq_ms, "site_steps_per_s": 2 * sites * T / (seq_ms / 1e3),
                              "ms_per_solve": [p for p in seq[-1][1]]},
        "side_by_side": {"ms_wall": par_ms, "ms_per_stream": par[-1][1]},
        "gain": seq_ms / par_ms,
    }
    print(json.dumps(line), flush=True)
    for lat, m in zip(lats, models):
        lat.close()
        m.close()
    for c in ctxs:
        c.close()


def run_trajectory(a):
    """The rod-cell model as a trajectory with output: each bench step is 500
    timesteps in runs of 100, after each run the species counts (taken inside
    the run) and a lattice frame go to a `.lm` file (lmb_lmfile_append_lattice_device: GPU transpose,
    copy to pinned memory, gzip-1 16^3 chunks on the writer thread), and the
    timed region ends when the file is flushed.  The same loop without the
    file is timed beside it; both are wall-clock (host calls included)."""
    import numpy as np
    import torch

    from lattice_microbes_b200.lmfile import LMFile, LMFileWriter
    from lattice_microbes_b200.replicas import Ranks
    from lattice_microbes_b200.solver import Context, Lattice, Model, kernel_launches
    ranks = Ranks()
    if ranks.rank != 0:
        return
    w = WORKLOADS["rodcell"]
    spec = make_spec("rodcell", 1)
    N, T, every = spec.nsites, a.timesteps_per_step or 500, 100
    ctx = Context(0)
    model = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat.set_native(spec.lattice, spec.sites)
    tuned = lat.autotune(model, 7, 0, 100)
    tmp = tempfile.mkdtemp()

    def loop(writer, first, steps):
        # With output: each run takes the species totals in its own work
        # (lmb_run_counts_async); without: the runs alone.
        t = first
        for _ in range(steps):
            for _ in range(T // every):
                if writer is not None:
                    _, _, c = lat.run_counts(model, 7, t, every, spec.ns)
                    t += every
                    writer.append_species_counts(0, [t * spec.tau], np.asarray(c[1:], np.int32)[None, :])
                    writer.append_lattice_device(0, t * spec.tau, lat)
                else:
                    lat.run(model, 7, t, every)
                    t += every
        if writer is not None:
            writer.flush()
        return t

    path = os.path.join(tmp, "traj.lm")
    wr = LMFileWriter(path)
    t = loop(wr, 0, a.warmup)
    clocks = ClockSampler(0)
    torch.cuda.synchronize()
    launches0 = kernel_launches()
    clocks.start()
    t0 = time.perf_counter()
    t = loop(wr, t, a.steps)
    wall = time.perf_counter() - t0
    clock_info = clocks.stop()
    launches = kernel_launches() - launches0
    frames, nbytes = wr.stats()
    wr.close()
    with LMFile(path) as f:
        nframes = len(f.lattice_times(0))
        last = f.lattice(0, nframes - 1)
    ref_last = np.asarray(lat.get_row_major()[0])
    assert np.array_equal(last, ref_last), "last frame in the file differs from the device lattice"
    size = os.path.getsize(path)
    os.unlink(path)
    t1 = time.perf_counter()
    loop(None, t, a.steps)
    wall_plain = time.perf_counter() - t1
    rate = N * T * a.steps / wall
    fr = a.steps * T // every
    raw = N * spec.slots * spec.bytes_per_slot
    line = {
        "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": wall / a.steps * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": w["dtype"], "data": "synthetic (seeded, lattice_microbes_b200.configs.config1)",
        "config": {"workload": "rod-cell trajectory to a .lm file: " + w["desc"], "timesteps_per_step": T,
                   "frame_every": every, "sites": N, "parallelism": "single", "schedule": "fused Ty=%d Tz=%d" % (tuned[1], tuned[2]) if tuned[0] == 0 else "phases",
                   "timing": "wall clock, host calls and the file flush included"},
        "output": {"frames": fr, "frames_per_s": fr / wall, "raw_bytes_per_frame": raw,
                   "gzip_bytes_per_frame": nbytes / max(frames, 1), "file_bytes": size,
                   "raw_GB_per_s": fr * raw / wall / 1e9},
        "without_output": {"value": N * T * a.steps / wall_plain, "unit": METRIC,
                           "ms_per_step": wall_plain / a.steps * 1e3},
        "output_cost_frac": 1.0 - wall_plain / wall,
        "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": (T // every) * (raw + 8 * (spec.ns + 1))},
        "gpu_launches": launches, "clocks": clock_info,
    }
    lat.close()
    model.close()
    ctx.close()
    print(json.dumps(line))


def _to_byte16(spec):
    """The request's particles in a 16-slot ByteLattice (the serving layout)."""
    import numpy as np
    from lattice_microbes_b200 import configs
    N = spec.nsites
    slots = configs.native_to_slots(spec.lattice, spec.X, spec.Y, spec.Z, spec.slots, spec.bytes_per_slot)
    lat = configs.empty_lattice(spec.X, spec.Y, spec.Z, 16, 1)
    for k in range(spec.slots):
        lat[(k // 4) * N:(k // 4 + 1) * N] |= slots[:, k].astype(np.uint32) << np.uint32(8 * (k % 4))
    spec.lattice, spec.slots = lat, 16
    return spec


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "cme":
        run_cme(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "pair":
        run_pair(args)
    elif args.workload == "trajectory":
        run_trajectory(args)
    else:
        run_ours(args)
