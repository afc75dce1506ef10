"""Benchmark: vertex-steps/s of the deformable-ring hot path on B200.

Workload (default, the metric's configuration): 1024 rings, nv 32/45
bidisperse 1:1.4 (39,424 vertices), smooth vertex-segment Lennard-Jones (rc
2.5 sigma, epsilon 1), calA0 1.05, packing fraction 0.85, shape constants ea
1e5, el 20, eb 10, NVE velocity Verlet at dt 0.002 from ring velocities drawn
at T 0.01.  The relaxed packing is the seeded synthetic state in
bench_state/smooth_lj_1024.npz (written by bench_state/make_state.py: rings
placed without overlap at phi 0.40, FIRE-compressed to 0.85); the thermal
velocities are drawn on the host from numpy's default_rng(1000 + rank), the
same draw in both arms, so the reference arm runs the same state without the
GPU library.

One bench step = ``--md-steps`` NVE steps (default 1000) through one
``DPM2D.NVELoop`` call, neighbour-list rebuilds included as they fall due.
``value`` = vertices x MD steps x bench steps / device time (max over ranks)
for ``--precision`` (default fp64, the reference's arithmetic); the other
precision (mixed: FP32 far pair units, FP64 near-contact units and
everything else) is timed the same way from the same start state under
``precision_comparison``, with the force error of the mixed path against
FP64 on thermal states and both paths' NVE energy drift.  ``e2e`` (both
precisions) adds, every bench step, the upload of positions and velocities
from pinned host memory and the download of positions, velocities and the
potential energy through the public API.  ``scale_up`` runs the same
dynamics on 65,536 rings (a periodic 8 x 8 tiling of the packing, 2.52M
vertices) for both precisions.

Multi-GPU (``--gpus N``): one independent replica per rank (weak scaling, no
collective on the data path); the batched-systems measurement splits its
systems into contiguous vertex-balanced blocks, one per rank.  Run directly
with ``--gpus N`` the script launches its N ranks itself
(torch.distributed.run); under a launcher WORLD_SIZE must equal N.  Rank 0
prints the line.  ``--impl reference`` times the reference's own kernels
compiled as host code (oracle/_ref) on the host cores, and the reference's
own CUDA build on the same state.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "vertex-steps/s at 1 B200: mixed vs plain FP64 at <=1e-6 force err; HBM GB/s frac"
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64 (vector), nominal
UNIT = "vertex-steps/s"
STATE = os.path.join(ROOT, "bench_state", "smooth_lj_1024.npz")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--md-steps", type=int, default=1000)
    ap.add_argument("--state", default=STATE, help="prepared packing (npz); empty: prepare --rings rings on the GPU")
    ap.add_argument("--rings", type=int, default=1024, help="ring count when no --state is given")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-systems FIRE / compression measurement")
    ap.add_argument("--batch-systems", type=int, default=256)
    ap.add_argument("--no-rigid", action="store_true", help="skip the rigid-ellipse measurement")
    ap.add_argument("--rigid-steps", type=int, default=2000)
    ap.add_argument("--no-diff", action="store_true", help="skip the derivative measurement")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-scale-up", action="store_true", help="skip the 65,536-ring measurement")
    ap.add_argument("--scale-tiles", type=int, default=8, help="scale-up: k x k copies of the packing")
    ap.add_argument("--scale-steps", type=int, default=200, help="scale-up: MD steps per timed repetition")
    ap.add_argument("--save-state", default=None, help="write the prepared state (npz) after preparation")
    ap.add_argument("--profile-jam", action="store_true",
                    help="only the device compression of the jamming measurement, inside a profiler range "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--jam-systems", type=int, default=8,
                    help="systems of the compression-to-jamming measurement (each also runs through its own context)")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="only time the fused step kernel (few launches; for ncu captures)")
    ap.add_argument("--profile-build", action="store_true",
                    help="only run full neighbour-list builds of the prepared state (for ncu captures)")
    ap.add_argument("--profile-tiles", type=int, default=1,
                    help="with --profile-kernel: profile k x k periodic copies of the packing")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per vertex of the fused kernel (0: library default)")
    ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64"],
                    help="arithmetic of the headline run (the other one is timed for comparison)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the other precision's run and the accuracy / energy-drift runs")
    ap.add_argument("--drift-steps", type=int, default=100000,
                    help="NVE steps of each precision's energy-drift run (untimed)")
    ap.add_argument("--plan-only", action="store_true",
                    help="print each rank's block of batched systems and exit (no device work)")
    return ap.parse_args(argv)


# ------------------------------------------------------------ shared input
def load_state(path: str) -> dict:
    """The prepared packing as host arrays (numpy only; no library needed)."""
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def thermal_velocities(nv_list, T: float, seed: int) -> np.ndarray:
    """Ring velocities N(0, sqrt(T)) per component from default_rng(seed),
    copied to every vertex of the ring (both arms use this draw)."""
    nv_list = np.asarray(nv_list)
    rng = np.random.default_rng(seed)
    return np.repeat(rng.normal(0.0, np.sqrt(T), size=(len(nv_list), 2)), nv_list, axis=0).reshape(-1)


def workload_string(c: dict, rings: int, vertices: int) -> str:
    return (f"{rings} deformable rings nv 32/45 (1:1.4), {vertices} vertices, smooth vertex-segment LJ rc "
            f"{c['LJcutoff']:g}, calA0 1.05, phi 0.85, ea {c['ea']:g} el {c['el']:g} eb {c['eb']:g}, NVE dt "
            f"{c['dt']:g}, T {c['T']:g} velocities from default_rng(1000)")


def packing_of(state: dict, vel: np.ndarray):
    from cudaring_b200 import synth

    n = len(state["nv_list"])
    return synth.Packing(nv_list=state["nv_list"], pos=state["pos"].copy(), vel=vel, rad=state["rad"],
                         l0=state["l0"], theta0=state["theta0"], a0=state["a0"], box=state["box"],
                         centres=np.zeros((n, 2)))


# ------------------------------------------------------------ ranks
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def launch_ranks(args) -> int:
    """``bench.py --gpus N`` run directly: start its N ranks under
    torch.distributed.run (one process per GPU) and pass their output on."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.abspath(__file__),
           *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def init_group(world: int):
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))


def close_group(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


from cudaring_b200.replicas import gather_per_system, max_over_ranks, shard_systems, sum_over_ranks  # noqa: E402


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


BATCH_SEED = 20261207


def batch_block(num_systems: int, world: int, rank: int):
    """This rank's contiguous, vertex-balanced block of the batched systems."""
    from cudaring_b200.compress import batch_packings

    pks = batch_packings(num_systems, seed=BATCH_SEED)
    sizes = [p.num_vertices for p in pks]
    return pks, shard_systems(sizes, world, rank)


def print_plan(args, world: int, rank: int):
    """The ranks' blocks of batched systems (host logic only, any backend)."""
    _, blk = batch_block(args.batch_systems, world, rank)
    plan = gather_per_system([(rank, blk.start, blk.stop)], world)
    if rank == 0:
        print(json.dumps({"plan": [list(x) for x in plan], "world": world, "systems": args.batch_systems}),
              flush=True)


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: wait for its first sample,
            # then keep only the samples taken from here on (the timed region)
            t_end = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < t_end and self.proc.poll() is None:
                time.sleep(0.005)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def committed_traffic(precision: str) -> dict | None:
    """DRAM bytes per launch of the step kernel from a committed ncu capture."""
    path = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f).get(precision)
    return None


# ------------------------------------------------------------ CPU baseline
def cpu_reference_rate(state: dict, vel: np.ndarray, c: dict, threads: int, target_seconds: float = 12.0,
                       rebuild_every: float | None = None) -> dict:
    """Reference kernels compiled as host code (oracle/_ref): one neighbour build
    plus NVE steps on the same state and velocities; vertex-steps/s with the
    build amortised over the rebuild interval measured on the GPU run."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle

    kind = "reference" if oracle.ref_available() else "port"
    if kind != "reference":
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": "oracle/_ref not built; CPU baseline skipped"}
    R, nv = setup_reference(state, vel, c)
    cut = R.ref_set_displacement_cutoff(0.5, 2 * state["rad"].mean())
    t0 = time.perf_counter()
    R.ref_calc_neighbor_list(cut)
    t_build = time.perf_counter() - t0
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    # time-bounded sample: single NVE steps until the budget is spent, so a
    # rebuild (an O(Nv^2) scan in the reference) that falls due is included
    upd0 = R.ref_update_count()
    nsteps, t_steps = 0, 0.0
    while nsteps < 2 or (t_steps < target_seconds and nsteps < 5000):
        t0 = time.perf_counter()
        R.ref_nve_loop(1)
        t_steps += time.perf_counter() - t0
        nsteps += 1
    upd = R.ref_update_count() - upd0
    # steps without a rebuild in the sample: charge the list build at the
    # rebuild rate measured on the GPU run of the same dynamics
    t_plain = t_steps if upd else t_steps + (nsteps / rebuild_every) * t_build if rebuild_every else t_steps
    rate = nv * nsteps / t_plain
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": (f"{nsteps} NVE steps of the same {nv}-vertex state on {threads} threads "
                       f"({t_steps:.1f} s, {upd} rebuilds in sample; one O(Nv^2) list build takes {t_build:.1f} s"
                       + (f"; rebuilds charged at the GPU run's rate of one per {rebuild_every:.0f} steps"
                          if (upd == 0 and rebuild_every) else "") + ")")}


def setup_reference(state: dict, vel: np.ndarray, c: dict):
    """oracle/_ref (the reference's kernels as host code) holding the state."""
    import oracle

    R = oracle.ref()
    nvl = np.asarray(state["nv_list"], dtype=np.int64)
    pos = np.ascontiguousarray(state["pos"], dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    rad, l0, a0 = (np.ascontiguousarray(state[k], dtype=np.float64) for k in ("rad", "l0", "a0"))
    th0 = np.ascontiguousarray(state["theta0"], dtype=np.float64)
    box = state["box"]
    R.ref_create(len(nvl), nvl)
    R.ref_set_box(float(box[0]), float(box[1]))
    R.ref_set_types(1, 1, 0, 0)
    R.ref_set_energy_costs(c["ea"], c["el"], c["eb"], c["ec"])
    R.ref_set_lj_cutoff(c["LJcutoff"])
    R.ref_set_time_step(c["dt"])
    R.ref_set_state(pos.ctypes.data, vel.ctypes.data, rad.ctypes.data, l0.ctypes.data, th0.ctypes.data,
                    a0.ctypes.data)
    setup_reference.keep = (pos, vel, rad, l0, th0, a0, nvl)  # arrays the library reads stay alive
    return R, int(nvl.sum())


# ------------------------------------------------------------------- main
PREC_DTYPE = {"mixed": "f64 state + f32 far pair units (near-contact units f64)", "fp64": "f64"}


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args)
    world, rank, local = dist_setup()
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
    if args.profile_jam:
        print(json.dumps(jamming_measurement(args.jam_systems, profile_only=True)), flush=True)
        return 0
    if args.plan_only:
        init_group(world)
        print_plan(args, world, rank)
        close_group(world)
        return 0
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)

    import torch

    from cudaring_b200 import DPM2D, synth, workloads

    torch.cuda.set_device(local)
    init_group(world)
    t_prep = time.perf_counter()
    if args.state:
        state = load_state(args.state)
        c = synth.workload_config("smooth_lj", len(state["nv_list"]))
        prep_info = {"fire_iterations": int(state["fire_iterations"]), "state": os.path.relpath(args.state, ROOT)}
    else:
        d0, info = workloads.prepared_deformable("smooth_lj", args.rings, seed=20261203 + rank)
        state = {"nv_list": d0.numVertexInParticleList, "pos": d0.getVertexPositions(), "rad": d0.getVertexRadii(),
                 "l0": d0.getRestLengths(), "theta0": d0.getRestAngles(), "a0": d0.getRestAreas(),
                 "box": d0.getBoxSize()}
        d0.close()
        c = info["config"]
        prep_info = {"fire_iterations": info["fire_iterations"], "state": "prepared in this run"}
        if args.save_state:
            np.savez_compressed(args.save_state, fire_iterations=info["fire_iterations"], **state)
    vel0 = thermal_velocities(state["nv_list"], c["T"], 1000 + rank)
    kw = {k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff", "dt")}
    d = DPM2D.from_packing(packing_of(state, vel0), **kw)
    cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
    d.calcNeighborList(cut)
    d.resetLastPositions()
    d.calcForceEnergy()
    nv, npr = d.numVertices, d.numParticles
    if args.lanes:
        d.setLanes(args.lanes)
    elif not args.profile_kernel:
        d.autotune(30)  # untimed: picks lanes per vertex by timing the fused kernel
    lanes = d.getLanes()
    if args.profile_build:
        # forced one-launch builds of the list (the rebuild a step sequence
        # runs when the displacement check fires)
        for _ in range(3):
            d.calcNeighborList(cut)
        ms = []
        for _ in range(5):
            t0 = time.perf_counter()
            d.calcNeighborList(cut)
            torch.cuda.synchronize()
            ms.append((time.perf_counter() - t0) * 1e3)
        print(json.dumps({"profile_build_wall_ms": min(ms), "vertices": nv,
                          "list_size": d.getNeighborListSize()}), flush=True)
        d.close()
        close_group(world)
        return 0
    if args.profile_kernel:
        if args.profile_tiles > 1:
            big = workloads.tile_system(d, args.profile_tiles, c)
            d.close()
            d = big
            nv = d.numVertices
            if args.lanes:
                d.setLanes(args.lanes)
            lanes = d.getLanes()
        d.setPrecision(args.precision)
        ms = d.profileStepKernel(3)
        print(json.dumps({"profile_kernel_ms": ms, "vertices": nv, "lanes": lanes,
                          "precision": args.precision}), flush=True)
        d.close()
        close_group(world)
        return 0
    d.setTimeStep(c["dt"])
    d.initNVE(c["T"], readState=True)
    x0, v0 = d.getVertexPositions(), d.getVertexVelocities()
    t_prep = time.perf_counter() - t_prep

    import ctypes

    sp = ctypes.c_void_p()
    d._call("cr_get_stream", ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    M = args.md_steps
    peaks = measured_peaks()
    bytes_per_step = 88 * nv + 8 * npr

    def l2_flush():
        with torch.cuda.stream(stream):
            flush.fill_(1.0)

    def restart(precision):
        d.setPrecision(precision)
        d.setVertexPositions(x0)
        d.setVertexVelocities(v0)
        d.calcNeighborList(cut)
        d.calcForceEnergy()
        d.initNVE(0.0, readState=True)

    def timed_run(precision):
        restart(precision)
        # warm-up (also captures and instantiates the CUDA graphs)
        for _ in range(args.warmup):
            d.NVELoop(M)
            l2_flush()
        torch.cuda.synchronize()
        x_warm = d.getVertexPositions()
        upd0, launches0, e0 = d.getUpdateCount(), d.getLaunchCount(), d.getEnergy()
        barrier(world)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            ev0.record(stream)
            for _ in range(args.steps):
                d.NVELoop(M)
                l2_flush()
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier(world)
        ms_total = max_over_ranks(ev0.elapsed_time(ev1), world)
        return {"ms_total": ms_total, "value": nv * M * args.steps * world / (ms_total / 1e3),
                "launches": d.getLaunchCount() - launches0, "updates": d.getUpdateCount() - upd0,
                "energy_change_rel": abs(d.getEnergy() - e0) / abs(e0) if e0 else None,
                "clocks": clocks.summary(), "x_warm": x_warm, "x_end": d.getVertexPositions()}

    def e2e_run(precision):
        """Through the public API with host buffers: every bench step uploads
        positions and velocities from pinned memory, runs NVELoop(M) and reads
        back positions, velocities and the potential energy."""
        restart(precision)
        hpos = torch.empty(2 * nv, dtype=torch.float64, pin_memory=True).numpy()
        hvel = torch.empty(2 * nv, dtype=torch.float64, pin_memory=True).numpy()
        hpos[:] = x0
        hvel[:] = v0
        d.NVELoop(M)  # warm-up of this precision's graphs
        n_e2e = max(1, min(args.steps, 5))
        barrier(world)
        torch.cuda.synchronize()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        for _ in range(n_e2e):
            d.setVertexPositions(hpos)
            d.setVertexVelocities(hvel)
            d.NVELoop(M)
            d.getVertexPositions(out=hpos)
            d.getVertexVelocities(out=hvel)
            _ = d.getPotentialEnergy()
        eb.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(ea.elapsed_time(eb), world)
        return {"value": nv * M * n_e2e * world / (ms_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 2 * 16 * nv, "d2h_bytes_per_step": 2 * 16 * nv + 8,
                "precision": precision, "bench_steps": n_e2e}

    def kernel_alone(precision):
        d.setPrecision(precision)
        ms_launch = ctypes.c_double()
        d._call("cr_profile_step_kernel", 200, ctypes.byref(ms_launch))
        return ms_launch.value

    prim = args.precision
    other = "fp64" if prim == "mixed" else "mixed"
    run = timed_run(prim)
    value = run["value"]
    e2e = None if args.no_e2e else e2e_run(prim)

    # roofline of the dominant kernel.  The middle steps of each NVELoop run in
    # the multi-step kernel (up to 64 steps per launch, grid barriers between
    # steps), so the unit is one step: algorithmic bytes per step over the
    # device time per step of the timed region (CUDA events on the library's
    # stream; rebuild launches included).  The single-step kernel timed alone
    # (back-to-back launches) is reported beside it.
    ms_launch = kernel_alone(prim)
    step_s = run["ms_total"] * 1e-3 / (args.steps * M)
    achieved = bytes_per_step / step_s / 1e9
    traffic = committed_traffic(prim)
    iso = bytes_per_step / (ms_launch * 1e-3) / 1e9
    # secondary roof: the FP64 pipe.  Flop model of one step: ~120 flops per
    # vertex for the shape terms and ~35 per listed pair and role (two smooth
    # units per list entry), over B200's nominal FP64 rate
    d.setVertexPositions(x0)
    d.calcNeighborList(cut)
    pairs = float(d.getMaxNeighborList().sum())
    flops_per_step = 120.0 * nv + 2 * 35.0 * pairs
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": traffic.get("bytes_per_launch") if traffic else None,
                "kernel": f"k_tile_steps<LJ, smooth, {prim}> (multi-step) + k_nbr_fused rebuilds",
                "us_per_step": step_s * 1e6, "algorithmic_bytes_per_step": bytes_per_step,
                "traffic_note": "DRAM bytes of one single-step launch of the same step body (ncu, cold L2)",
                "single_step_kernel": {"kernel": f"k_tile<LJ, smooth, step, {prim}>", "ms_per_launch": ms_launch,
                                       "achieved": iso, "frac": iso / peaks["hbm_gbs"]},
                "secondary": {"bound": "fp64 pipe", "unit": "TFLOP/s",
                              "flops_per_step_model": flops_per_step,
                              "achieved": flops_per_step / step_s / 1e12, "peak": FP64_NOMINAL_TFLOPS,
                              "peak_source": "nominal (B200 FP64, not measured on this pool)",
                              "frac": flops_per_step / step_s / 1e12 / FP64_NOMINAL_TFLOPS,
                              "ncu_fp64_pipe_active_pct": traffic.get("fp64_pipe_active_pct") if traffic else None}}

    comparison = None
    if not args.no_compare:
        orun = timed_run(other)
        oms = kernel_alone(other)
        o_step_s = orun["ms_total"] * 1e-3 / (args.steps * M)
        comparison = {other: {"value": orun["value"], "ms_per_step": orun["ms_total"] / args.steps,
                              "us_per_md_step": o_step_s * 1e6,
                              "roofline_frac": bytes_per_step / o_step_s / 1e9 / peaks["hbm_gbs"],
                              "single_step_kernel_ms_per_launch": oms,
                              "gpu_launches": orun["launches"], "rebuilds": orun["updates"],
                              "clocks": orun["clocks"],
                              "e2e": None if args.no_e2e else e2e_run(other)}}
        fp64_value = orun["value"] if prim == "mixed" else value
        mixed_value = value if prim == "mixed" else orun["value"]
        comparison["mixed_over_fp64"] = mixed_value / fp64_value
        comparison["accuracy"] = precision_accuracy(d, cut, [run["x_warm"], run["x_end"]], v0, args.drift_steps,
                                                    restart)

    scale = None
    if not args.no_scale_up:
        d.setVertexPositions(x0)  # tile the prepared packing itself
        scale = scale_up_measurement(d, c, args, world, peaks)

    batch = None if args.no_batch else batched_fire_measurement(args.batch_systems, world, rank)
    jam = None if (args.no_batch or rank != 0) else jamming_measurement(args.jam_systems)

    rigid = None
    if rank == 0 and not args.no_rigid:
        rigid = rigid_ellipse_measurement(args.rigid_steps)

    deriv = None
    if rank == 0 and not args.no_diff:
        deriv = derivative_measurement()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        steps_per_rebuild = (M * args.steps / run["updates"]) if run["updates"] else None
        cpu = cpu_reference_rate(state, vel0, c, os.cpu_count() or 1, rebuild_every=steps_per_rebuild)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run["ms_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": PREC_DTYPE[prim],
            "data": "synthetic: seeded rings placed at phi 0.40, FIRE-compressed to 0.85 (bench_state), "
                    "T=0.01 ring velocities from default_rng(1000 + rank)",
            "config": {"workload": workload_string(c, npr, nv), "precision": prim, "rings": npr, "vertices": nv,
                       "md_steps_per_bench_step": M, "l2": "flushed between bench steps (256 MB write)",
                       "parallelism": f"replicas x{world}", "state": prep_info["state"],
                       "neighbour_rebuilds_in_timed_region": run["updates"],
                       "energy_change_rel_timed_region": run["energy_change_rel"],
                       "prep_seconds": t_prep, "fire_iterations_prep": prep_info["fire_iterations"],
                       "lanes_per_vertex": lanes},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": run["launches"],
            "clocks": run["clocks"], "precision_comparison": comparison, "scale_up": scale,
            "batched_systems": batch, "compression_to_jamming": jam, "rigid_ellipses": rigid, "derivatives": deriv,
        }
        print(json.dumps(line), flush=True)
    d.close()
    close_group(world)
    return 0


def scale_up_measurement(d, c: dict, args, world: int, peaks: dict) -> dict:
    """The same dynamics on k x k periodic copies of the packing (65,536 rings,
    2.52M vertices at k = 8; a periodic image tiling is itself a packing at
    the same phi), thermal velocities of every ring drawn anew: vertex-steps/s
    and the HBM fraction of the algorithmic bytes for both precisions.  One
    warm-up repetition, then three timed repetitions of ``--scale-steps``
    steps; the 250 MB working set is larger than L2."""
    import ctypes

    import torch

    from cudaring_b200 import workloads

    k = args.scale_tiles
    d.setPrecision("fp64")
    big = workloads.tile_system(d, k, c)
    nv, npr = big.numVertices, big.numParticles
    big.setVertexVelocities(thermal_velocities(big.numVertexInParticleList, c["T"], 2000))
    big.setTimeStep(c["dt"])
    cut = big.setDisplacementCutoff(0.5, 2.0 * big.getMeanVertexRadius())
    x0, v0 = big.getVertexPositions(), big.getVertexVelocities()
    sp = ctypes.c_void_p()
    big._call("cr_get_stream", ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    out = {"workload": f"{k}x{k} periodic copies of the benchmark packing: {npr} rings, {nv} vertices",
           "unit": UNIT, "md_steps": args.scale_steps, "repetitions": 3,
           "algorithmic_bytes_per_step": 88 * nv + 8 * npr, "lanes_per_vertex": big.getLanes()}
    for prec in ("fp64", "mixed"):
        big.setPrecision(prec)
        big.setVertexPositions(x0)
        big.setVertexVelocities(v0)
        big.calcNeighborList(cut)
        big.calcForceEnergy()
        big.initNVE(0.0, readState=True)
        big.NVELoop(args.scale_steps)
        upd0 = big.getUpdateCount()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            big.NVELoop(args.scale_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        step_s = ms * 1e-3 / (3 * args.scale_steps)
        ach = (88 * nv + 8 * npr) / step_s / 1e9
        out[prec] = {"value": nv * 3 * args.scale_steps * world / (ms * 1e-3), "us_per_step": step_s * 1e6,
                     "hbm_achieved_gbs": ach, "hbm_frac": ach / peaks["hbm_gbs"],
                     "rebuilds": big.getUpdateCount() - upd0}
    big.close()
    return out


def batched_fire_measurement(num_systems: int, world: int, rank: int, fire_iters: int = 2000,
                             loop_systems: int = 8) -> dict:
    """Many independent systems in one launch per op (cr_batch_*): the FIRE
    throughput of the batch against the per-system single-context loop on the
    same states, plus a bounded sample of the compression protocol.

    Workload: ``num_systems`` deformable-ring packings, ring counts uniform in
    [16, 512], bidisperse 1:1.4 with nv 16/22, calA0 uniform in [1.0, 1.2],
    harmonic repulsion, brought to packing fraction 0.60 (untimed).  Timed:
    FIRE to max |F| <= 1e-10 / sigma (at most ``fire_iters`` iterations) on
    every system, as vertex-iterations per second; the per-system loop runs
    the same minimisation on ``loop_systems`` of them one at a time (rank 0).
    With several ranks each takes a contiguous vertex-balanced block of the
    systems; vertex-iterations are summed and the time is the slowest rank's."""
    import torch

    from cudaring_b200 import DPM2D
    from cudaring_b200.batch import Batch
    from cudaring_b200.compress import prepare_batch

    t0 = time.perf_counter()
    all_pks, blk = batch_block(num_systems, world, rank)
    pks = [all_pks[s] for s in blk]
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    b = Batch.from_packings(pks, **kw)
    prepare_batch(b, 0.60, step=0.03, tol0=1e-6, max_fire_iters=5000)
    lanes = b.autotune(10)
    t_prep = time.perf_counter() - t0
    nvs = np.array([p.num_vertices for p in pks])
    nv_all = int(sum(p.num_vertices for p in all_pks))
    pos, rad, l0, a0 = b.getVertexPositions(), b.getVertexRadii(), b.getRestLengths(), b.getRestAreas()
    out = {"workload": f"{num_systems} systems, {nv_all} vertices, rings U[16,512] nv 16/22, harmonic, "
                       f"phi 0.60, FIRE to 1e-10/sigma (<= {fire_iters} iterations)",
           "unit": "vertex-iterations/s", "lanes_per_vertex": lanes, "tile_shape": list(b.getTileShape()),
           "prep_seconds": t_prep,
           "ranks": world, "rank0_block": [blk.start, blk.stop]}
    for prec in ("fp64", "mixed"):
        b.setVertexPositions(pos)
        b.setVertexVelocities(np.zeros_like(pos))
        b.setPrecision(prec)
        sig = b.getMeanParticleSizes()
        b.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-2, 1e-1, 0.2], 20, dt=1e-2 * sig)
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its, fmax = b.fireMinimize(1e-10 / sig, fire_iters)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0, world)
        vi = sum_over_ranks(float((its * nvs).sum()), world)
        per = gather_per_system([(int(i), bool(f <= 1e-10 / s)) for i, f, s in zip(its, fmax, sig)], world)
        out[prec] = {"value": vi / dt, "seconds": dt, "iterations_mean": float(np.mean([p[0] for p in per])),
                     "converged_systems": int(sum(p[1] for p in per))}
    # the per-system loop: the same minimisation through single contexts
    if rank == 0:
        vi, tt = 0.0, 0.0
        for s in range(min(loop_systems, len(pks))):
            pk = pks[s]
            pk.pos = pos[b.system_slice(s)].copy()
            pk.rad = rad[b.system_slice(s, dim=1)].copy()
            pk.l0 = l0[b.system_slice(s, dim=1)].copy()
            pk.a0 = a0[b.system_slice(s, per="ring", dim=1)].copy()
            pk.vel = np.zeros_like(pk.pos)
            d = DPM2D.from_packing(pk, **kw)
            d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * d.getMeanVertexRadius()))
            d.calcForceEnergy()
            sg = d.getMeanParticleSize()
            d.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-2 * sg, 1e-1 * sg, 0.2], 20, 0, d.numVertices)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            it, _ = d.minimizeFIRE(1e-10 / sg, fire_iters)
            torch.cuda.synchronize()
            tt += time.perf_counter() - t0
            vi += it * d.numVertices
            d.close()
        out["per_system_loop_fp64"] = {"value": vi / tt, "systems": min(loop_systems, len(pks)),
                                       "sample": "the first systems of rank 0's block, one single-system context each"}
        out["batch_over_loop_fp64"] = out["fp64"]["value"] / world / out["per_system_loop_fp64"]["value"]
    # compression protocol sample (compressFIRE.cpp:101-205) from phi 0.60
    b.setVertexPositions(pos)
    b.setVertexVelocities(np.zeros_like(pos))
    b.setPrecision("fp64")
    barrier(world)
    t0 = time.perf_counter()
    res = b.compress(dphi=1e-3, min_dphi=1e-6, fire_dt=1e-2, tol0=1e-10, max_fire_iters=20000, max_steps=3)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, world)
    vi = sum_over_ranks(float((res["fire_iterations"] * nvs).sum()), world)
    phis = gather_per_system([float(x) for x in res["phi"]], world)
    out["compression_sample"] = {"steps": 3, "dphi": 1e-3, "seconds": dt, "value": vi / dt,
                                 "phi_mean": float(np.mean(phis))}
    b.close()
    return out


def jamming_measurement(num_systems: int = 8, profile_only: bool = False) -> dict:
    """Compression to jamming of a small batch, three ways: the protocol as
    one graph launch on the device (cr_batch_compress), the same protocol
    driven from the host between steps and FIRE chunks
    (cr_batch_compress_stepwise; the same states are required), and every
    system through its own single-system context (compress.compress_system).
    Rank 0 only: a secondary measurement."""
    import torch

    from cudaring_b200 import DPM2D, synth
    from cudaring_b200.batch import Batch
    from cudaring_b200.compress import batch_packings, compress_system, prepare_batch

    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    pks = batch_packings(num_systems, seed=17, rings=(16, 32))
    b = Batch.from_packings(pks, **kw)
    prepare_batch(b, phi0=0.70)
    pos, rad, l0, a0 = b.getVertexPositions(), b.getVertexRadii(), b.getRestLengths(), b.getRestAreas()
    prm = dict(dphi=2e-2, min_dphi=2e-3, fire_dt=1e-2, tol0=1e-6, max_fire_iters=20000, max_steps=40)
    out = {"workload": f"{num_systems} systems, rings U[16,32] nv 16/22, harmonic, from phi 0.70: dphi 0.02 halved "
                       "on overshoot down to 0.002, FIRE to 1e-6/sigma, at most 40 steps",
           "vertices": int(sum(p.num_vertices for p in pks))}
    if profile_only:
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        t0 = time.perf_counter()
        r = b.compress(**prm)
        torch.cuda.synchronize()
        out["device"] = {"seconds": time.perf_counter() - t0, "fire_iterations": int(r["fire_iterations"].sum()),
                         "launches": b.getLaunchCount()}
        torch.cuda.profiler.stop()
        b.close()
        return out
    res = {}
    for mode in ("device", "stepwise", "one_launch_per_op"):
        b.setVertexPositions(pos)
        b.setVertexVelocities(np.zeros_like(pos))
        b.setVertexRadii(rad)
        b.setRestLengths(l0)
        b.setRestAreas(a0)
        b.setPersistent(mode != "one_launch_per_op")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = b.compress(stepwise=mode == "stepwise", **prm)
        torch.cuda.synchronize()
        res[mode] = (time.perf_counter() - t0, r)
    b.close()
    t_op, r_op = res["one_launch_per_op"]
    t_dev, r_dev = res["device"]
    t_host, r_host = res["stepwise"]
    same = all(np.array_equal(r_dev[k], r_host[k]) for k in ("phi", "steps", "state", "fire_iterations"))
    out["device"] = {"seconds": t_dev, "phi": [round(float(x), 5) for x in r_dev["phi"]],
                     "steps": [int(x) for x in r_dev["steps"]], "state": [int(x) for x in r_dev["state"]],
                     "fire_iterations": int(r_dev["fire_iterations"].sum())}
    out["stepwise"] = {"seconds": t_host, "same_states_as_device": bool(same)}
    out["device_one_launch_per_op"] = {
        "seconds": t_op, "note": "the same graph with the persistent FIRE kernel off",
        "same_states_as_device": bool(all(np.array_equal(r_dev[k], r_op[k])
                                          for k in ("phi", "steps", "state", "fire_iterations")))}
    # every system through its own context, from the same prepared state
    vo = np.cumsum([0] + [p.num_vertices for p in pks])
    ro = np.cumsum([0] + [p.num_particles for p in pks])
    t0 = time.perf_counter()
    phis = []
    for s, pk in enumerate(pks):
        one_pk = synth.Packing(nv_list=pk.nv_list, pos=pos[2 * vo[s]:2 * vo[s + 1]], vel=np.zeros(2 * pk.num_vertices),
                               rad=rad[vo[s]:vo[s + 1]], l0=l0[vo[s]:vo[s + 1]], theta0=pk.theta0,
                               a0=a0[ro[s]:ro[s + 1]], box=pk.box, centres=pk.centres)
        d = DPM2D.from_packing(one_pk, **kw)
        d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
        phis.append(round(float(compress_system(d, **prm)["phi"]), 5))
        d.close()
    torch.cuda.synchronize()
    t_loop = time.perf_counter() - t0
    out["per_system_loop"] = {"seconds": t_loop, "systems": num_systems, "phi": phis,
                              "note": "the FIRE sums reduce in another order, so decisions at the 2 tol margin can "
                                      "flip and the paths to jamming part"}
    out["device_over_stepwise"] = t_host / t_dev
    out["persistent_speedup"] = t_op / t_dev
    out["device_over_loop"] = t_loop / t_dev
    return out


def derivative_measurement() -> dict:
    """The differentiation workload: 256 rings of 32
    vertices, harmonic, phi 0.88, FIRE-minimised to max |F| <= 1e-12; wall
    times of the minimised-state gradients of U and P along (ea, el, eb, calA0)
    (two conjugate-gradient Hessian solves to 1e-10), of Hessian-vector
    products on device buffers, and of d(U + K)/d(x0, v0) through 200 NVE
    steps (dt 0.002) with checkpoints every 20 steps."""
    import torch

    from cudaring_b200 import diff, workloads

    t0 = time.perf_counter()
    d, info = workloads.prepared_deformable("dense_harmonic")
    c = info["config"]
    sig = d.getMeanParticleSize()
    d.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-3 * sig, 1e-2 * sig, 0.2], 20, 0, d.numVertices)
    fire_it, fmax = d.minimizeFIRE(1e-12, 1000000)
    prep = time.perf_counter() - t0
    nv = d.numVertices
    calA0 = float(np.mean(c["calA0"])) if np.ndim(c["calA0"]) else float(c["calA0"])
    t1 = time.perf_counter()
    g = diff.minimized_gradients(d, calA0, tol=1e-10)  # block-Jacobi preconditioned CG
    t_grad = time.perf_counter() - t1
    d.setCGPreconditioner("none")
    t1 = time.perf_counter()
    g0 = diff.minimized_gradients(d, calA0, tol=1e-10)
    t_grad0 = time.perf_counter() - t1
    d.setCGPreconditioner("block_jacobi")
    # dP carries the adjoint term (dU's vanishes with the force at the minimum)
    agree = max(abs(g["dP"][k] - g0["dP"][k]) / max(abs(g0["dP"][k]), 1e-300) for k in g0["dP"])
    v = torch.randn(2 * nv, dtype=torch.float64, device="cuda")
    hv = torch.empty_like(v)
    for _ in range(5):
        d.hvpDevice(v.data_ptr(), hv.data_ptr())
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    reps = 200
    for _ in range(reps):
        d.hvpDevice(v.data_ptr(), hv.data_ptr())
    torch.cuda.synchronize()
    t_hvp = (time.perf_counter() - t2) / reps
    x0 = d.getVertexPositions()
    v0 = np.random.default_rng(3).normal(0.0, 0.01, size=x0.shape)
    t3 = time.perf_counter()
    J, gx, gv = diff.nve_gradient(d, x0, v0, 200, 0.002, checkpoint=20)
    t_nve = time.perf_counter() - t3
    out = {"workload": f"{d.numParticles} rings nv 32 ({nv} vertices), harmonic, phi {info['phi']:.3f}, "
                       f"FIRE to max |F| {fmax:.1e} ({fire_it} iterations)",
           "prep_seconds": prep,
           "minimized_gradients": {"seconds": t_grad, "cg_iterations": {k: it_rr[0] for k, it_rr in g["cg"].items()},
                                   "preconditioner": "block-Jacobi (2 x 2 vertex blocks)",
                                   "unpreconditioned": {"seconds": t_grad0,
                                                        "cg_iterations": {k: it_rr[0] for k, it_rr in g0["cg"].items()},
                                                        "max_rel_diff_dP": agree},
                                   "dU": g["dU"], "dP": g["dP"]},
           "hvp": {"ms_per_product": t_hvp * 1e3, "vertex_products_per_s": nv / t_hvp},
           "nve_gradient": {"seconds": t_nve, "steps": 200, "checkpoint": 20, "J": J}}
    d.close()
    return out


def rigid_ellipse_measurement(steps: int) -> dict:
    """Rigid bumpy ellipses (4096 rings of 24 vertices, WCA, rigid phi 0.65):
    rigid Langevin at T 0.1, gamma 1, and the same with active self-propulsion
    (f0 = v0 gamma = 0.1, taup = 1 / Dr = 100), dt 0.001, FP64 and mixed.
    vertex-steps/s over ``steps`` steps timed with CUDA events on the
    context's stream after a warm-up, neighbour rebuilds included."""
    import ctypes

    import torch

    from cudaring_b200 import workloads
    from cudaring_b200.dpm2d import simControl

    d, info = workloads.prepared_ellipses()
    c = info["config"]
    sp = ctypes.c_void_p()
    d._call("cr_get_stream", ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    nv = d.numVertices
    out = {"workload": f"{d.numParticles} rigid ellipses x 24 vertices ({nv} vertices), aspect U[1.2, 2.0], WCA, "
                       f"rigid phi {info['phi']:.3f}, dt {c['dt']}", "unit": "vertex-steps/s", "steps": steps,
           "prep_seconds": info["prep_seconds"], "lanes_per_vertex": d.getLanes()}
    for prec in ("fp64", "mixed"):
        d.setPrecision(prec)
        res = {}
        for mode in ("langevin", "active"):
            d.setParticleType(simControl.particleEnum.active if mode == "active" else simControl.particleEnum.passive)
            d.setSelfPropulsionParams(c["driving"] if mode == "active" else 0.0, c["taup"])
            d.initRigidLangevin(c["T"], c["gamma"], readState=True)
            d.rigidLangevinLoop(max(100, steps // 10))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            u0 = d.getUpdateCount()
            torch.cuda.synchronize()
            e0.record(stream)
            d.rigidLangevinLoop(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            res[mode] = {"value": nv * steps / (ms / 1e3), "ms_per_step": ms / steps,
                         "rebuilds": d.getUpdateCount() - u0}
        out[prec] = res
    d.setParticleType(simControl.particleEnum.passive)
    d.close()
    return out


def precision_accuracy(d, cut, states, v0, drift_steps, restart) -> dict:
    """Force / energy error of the mixed path against FP64 on thermal states,
    and the NVE energy error of both precisions over ``drift_steps`` steps
    from the same start state."""
    errs, maxabs, eerr = [], [], []
    for x in states:
        d.setVertexPositions(x)
        d.calcNeighborList(cut)
        d.setPrecision("fp64")
        d.calcForceEnergy()
        f64, e64 = d.getVertexForces(), d.getPotentialEnergy()
        d.setPrecision("mixed")
        d.calcForceEnergy()
        fmx, emx = d.getVertexForces(), d.getPotentialEnergy()
        errs.append(float(np.linalg.norm(fmx - f64) / np.linalg.norm(f64)))
        maxabs.append(float(np.abs(fmx - f64).max()))
        eerr.append(abs(emx - e64) / abs(e64))
    drift = {"steps": drift_steps}
    chunk = 1000
    for prec in ("fp64", "mixed"):
        restart(prec)
        e0 = d.getEnergy()
        es = []
        for _ in range(max(1, drift_steps // chunk)):
            d.NVELoop(chunk)
            es.append(d.getEnergy())
        es = np.array(es)
        t = np.arange(1, len(es) + 1) * chunk
        slope = float(np.polyfit(t, (es - e0) / abs(e0), 1)[0]) if len(es) > 1 else None
        drift[prec] = {"max_rel": float(np.abs(es - e0).max() / abs(e0)), "slope_rel_per_step": slope}
    drift["mixed_over_fp64_max_rel"] = drift["mixed"]["max_rel"] / drift["fp64"]["max_rel"]
    return {"force_err_l2_rel": errs, "force_err_max_abs": maxabs, "potential_energy_rel_err": eerr,
            "states": "thermal states: the start and the end of the timed run", "energy_drift": drift}


def run_reference_arm(args, world, rank):
    """The reference's own kernels as host code (oracle/_ref, all host threads)
    on the benchmark state and velocities, loaded with numpy: this arm maps
    neither libcudaring.so nor any kernel of this repository."""
    if rank != 0:
        return 0
    import oracle
    from cudaring_b200 import synth

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcrref.so was not built "
                                                              "(needs the reference checkout at build time)"}))
        return 0
    if not args.state or not os.path.exists(args.state):
        print(json.dumps({"impl": "reference", "unavailable": "the prepared benchmark state (--state) is missing"}))
        return 0
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    state = load_state(args.state)
    npr = len(state["nv_list"])
    c = synth.workload_config("smooth_lj", npr)
    vel = thermal_velocities(state["nv_list"], c["T"], 1000)
    R, nv = setup_reference(state, vel, c)
    cut = R.ref_set_displacement_cutoff(0.5, 2 * state["rad"].mean())
    t0 = time.perf_counter()
    R.ref_calc_neighbor_list(cut)
    t_build = time.perf_counter() - t0
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    # each bench step: single NVE steps until ~5 s have passed (rebuilds,
    # O(Nv^2) scans in the reference, included as they fall due)
    for _ in range(max(1, args.warmup)):
        R.ref_nve_loop(1)
    per_budget = 5.0
    total_steps, t = 0, 0.0
    for _ in range(args.steps):
        t_step, n = 0.0, 0
        while n < 1 or t_step < per_budget:
            t0 = time.perf_counter()
            R.ref_nve_loop(1)
            t_step += time.perf_counter() - t0
            n += 1
        total_steps += n
        t += t_step
    per = total_steps / max(1, args.steps)
    upd = R.ref_update_count()
    value = nv * total_steps / t
    gpu_build = reference_cuda_build(state, vel, c)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded rings placed at phi 0.40, FIRE-compressed to 0.85 (bench_state), "
                    "T=0.01 ring velocities from default_rng(1000 + rank)",
            "config": {"workload": workload_string(c, npr, nv), "precision": "fp64", "rings": npr, "vertices": nv,
                       "md_steps_per_bench_step": per, "state": os.path.relpath(args.state, ROOT),
                       "rebuilds_in_sample": upd, "list_build_seconds": t_build},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{total_steps} NVE steps in {t:.1f} s, reference kernels as host code, "
                                       f"{threads} OpenMP threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_cuda_build": gpu_build}
    print(json.dumps(line), flush=True)
    return 0


def reference_cuda_build(state: dict, vel: np.ndarray, c: dict, warmup: int = 100, steps: int = 2000) -> dict | None:
    """The reference's own CUDA build (oracle/_ref/ref_gpu_nve, compiled from
    its sources) on the same state and thermal velocities, read from the
    reference's on-disk packing format; timed with CUDA events inside it."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_nve")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_gpu_nve was not built (needs the reference checkout at build time)"}
    import tempfile

    from cudaring_b200 import packing_io

    nv = int(np.sum(state["nv_list"]))
    with tempfile.TemporaryDirectory() as tmp:
        packing_io.save_packing_arrays(tmp, packing_of(state, vel), digits=17)
        try:
            r = subprocess.run([exe, tmp, str(len(state["nv_list"])), str(warmup), str(steps), repr(c["dt"]),
                                repr(c["ea"]), repr(c["el"]), repr(c["eb"]), "lj", "smooth", repr(c["LJcutoff"])],
                               capture_output=True, text=True, timeout=600)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference CUDA build did not finish within 600 s"}
    if r.returncode != 0 or not r.stdout.strip():
        return {"unavailable": f"reference CUDA build exited {r.returncode}: {r.stderr.strip()[-200:]}"}
    info = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": info["vertex_steps_per_s"], "unit": UNIT, "ms_per_step": info["ms_per_step"],
            "steps": info["steps"], "warmup": info["warmup"], "rebuilds": info["updates"],
            "sample": f"farceri/cudaRing DPM2D compiled for sm_100a, NVELoop() x {steps} after {warmup} warm-up "
                      f"steps on the same {nv}-vertex state and velocities, CUDA-event timed"}


if __name__ == "__main__":
    sys.exit(main())
