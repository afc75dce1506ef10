"""Benchmark: vertex-steps/s of the deformable-ring hot path on B200.

Workload (default): 1024 rings, nv 32/45 bidisperse 1:1.4 (39,424 vertices),
smooth vertex-segment Lennard-Jones (rc 2.5 sigma, epsilon 1), calA0 1.05,
packing fraction 0.85, shape constants ea 1e5, el 20, eb 10, NVE velocity
Verlet at dt 0.002 with ring velocities drawn at T 0.01.  Inputs are synthetic
and seeded: rings placed without overlap at phi 0.40, compressed to 0.85 with
FIRE (cudaring_b200.workloads), then given thermal velocities; none of that is
timed.

One bench step = ``--md-steps`` NVE steps (default 1000) through one
``DPM2D.NVELoop`` call, neighbour-list rebuilds included as they fall due.
``value`` = vertices x MD steps x bench steps / device time (max over ranks)
for ``--precision`` (default mixed: FP32 pair terms, everything else FP64);
the other precision is timed the same way from the same start state and
reported under ``precision_comparison`` with the force error of the mixed
path against FP64 and both paths' NVE energy drift over ``--drift-steps``.
``e2e`` adds, every bench step, the upload of positions and velocities from
pinned host memory and the download of positions, velocities and the
potential energy through the public API.

Multi-GPU: one independent replica per rank (weak scaling, no collective on
the data path); rank 0 prints the line.  ``--impl reference`` times the
reference's own kernels compiled as host code (oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "vertex-steps/s at 1 B200: mixed vs plain FP64 at <=1e-6 force err; HBM GB/s frac"
UNIT = "vertex-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--md-steps", type=int, default=1000)
    ap.add_argument("--rings", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-systems FIRE / compression measurement")
    ap.add_argument("--batch-systems", type=int, default=256)
    ap.add_argument("--no-rigid", action="store_true", help="skip the rigid-ellipse measurement")
    ap.add_argument("--rigid-steps", type=int, default=2000)
    ap.add_argument("--no-diff", action="store_true", help="skip the derivative measurement")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--save-state", default=None, help="write the prepared state (npz) after preparation")
    ap.add_argument("--load-state", default=None, help="start from a state written by --save-state")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="only time the fused step kernel (few launches; for ncu captures)")
    ap.add_argument("--profile-build", action="store_true",
                    help="only run full neighbour-list builds of the prepared state (for ncu captures)")
    ap.add_argument("--lanes", type=int, default=0, help="lanes per vertex of the fused kernel (0: library default)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="arithmetic of the timed run (the other one is timed for comparison)")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the other precision's run and the accuracy / energy-drift runs")
    ap.add_argument("--drift-steps", type=int, default=100000,
                    help="NVE steps of each precision's energy-drift run (untimed)")
    return ap.parse_args()


def prepared_state(args, rank):
    """The prepared workload: built with FIRE compression, or loaded from --load-state."""
    from cudaring_b200 import DPM2D, synth, workloads

    if args.load_state:
        z = np.load(args.load_state)
        c = synth.workload_config("smooth_lj", len(z["nv_list"]))
        pk = synth.Packing(nv_list=z["nv_list"], pos=z["pos"], vel=z["vel"], rad=z["rad"], l0=z["l0"],
                           theta0=z["theta0"], a0=z["a0"], box=z["box"], centres=np.zeros((len(z["nv_list"]), 2)))
        kw = {k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff", "dt")}
        d = DPM2D.from_packing(pk, **kw)
        cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
        d.calcNeighborList(cut)
        d.resetLastPositions()
        d.calcForceEnergy()
        info = {"config": c, "fire_iterations": int(z["fire_iterations"]), "phi": d.getPreferredPhi()}
    elif args.rings > 1024 and args.rings % 1024 == 0 and int(round((args.rings // 1024) ** 0.5)) ** 2 * 1024 == args.rings:
        # large systems: the prepared 1024-ring packing replicated k x k times
        # (a periodic image tiling is itself a packing at the same phi); the
        # thermal velocities drawn afterwards decorrelate the copies
        d0, info = workloads.prepared_deformable("smooth_lj", 1024, seed=20261203 + rank)
        k = int(round((args.rings // 1024) ** 0.5))
        d = workloads.tile_system(d0, k, info["config"])
        d0.close()
        info = dict(info, tiled=f"{k}x{k} copies of the 1024-ring packing")
    else:
        d, info = workloads.prepared_deformable("smooth_lj", args.rings, seed=20261203 + rank)
    if args.save_state and not args.load_state:
        nvl = d.numVertexInParticleList
        np.savez(args.save_state, nv_list=nvl, pos=d.getVertexPositions(), vel=d.getVertexVelocities(),
                 rad=d.getVertexRadii(), l0=d.getRestLengths(), a0=d.getRestAreas(), theta0=d.getRestAngles(),
                 box=d.getBoxSize(), fire_iterations=info["fire_iterations"])
    if args.lanes:
        d.setLanes(args.lanes)
    elif not args.profile_kernel:
        d.autotune(30)  # untimed: picks lanes per vertex by timing the fused kernel
    info["lanes"] = d.getLanes()
    return d, info


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


from cudaring_b200.replicas import max_over_ranks  # noqa: E402  (device time of the slowest rank)


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------ CPU baseline
def cpu_reference_rate(d, c: dict, threads: int, target_seconds: float = 12.0,
                       rebuild_every: float | None = None) -> dict:
    """Reference kernels compiled as host code (oracle/_ref): one neighbour build
    plus NVE steps on the same prepared state; vertex-steps/s with the build
    amortised over the rebuild interval measured on the GPU run."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import oracle

    kind = "reference" if oracle.ref_available() else "port"
    if kind != "reference":
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "port",
                "sample": "oracle/_ref not built; CPU baseline skipped"}
    R = oracle.ref()
    pos, vel = d.getVertexPositions(), d.getVertexVelocities()
    rad, l0, a0 = d.getVertexRadii(), d.getRestLengths(), d.getRestAreas()
    th0 = np.full(d.numVertices, 0.0)
    nvl = d.numVertexInParticleList
    th0 = np.repeat(2 * np.pi / nvl, nvl).astype(np.float64)
    box = d.getBoxSize()
    R.ref_create(len(nvl), nvl)
    R.ref_set_box(float(box[0]), float(box[1]))
    R.ref_set_types(1, 1, 0, 0)
    R.ref_set_energy_costs(c["ea"], c["el"], c["eb"], c["ec"])
    R.ref_set_lj_cutoff(c["LJcutoff"])
    R.ref_set_time_step(c["dt"])
    R.ref_set_state(pos.ctypes.data, vel.ctypes.data, rad.ctypes.data, l0.ctypes.data, th0.ctypes.data,
                    a0.ctypes.data)
    cut = R.ref_set_displacement_cutoff(0.5, 2 * rad.mean())
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
    rate = d.numVertices * nsteps / t_plain
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": (f"{nsteps} NVE steps of the same {d.numVertices}-vertex state on {threads} threads "
                       f"({t_steps:.1f} s, {upd} rebuilds in sample; one O(Nv^2) list build takes {t_build:.1f} s"
                       + (f"; rebuilds charged at the GPU run's rate of one per {rebuild_every:.0f} steps"
                          if (upd == 0 and rebuild_every) else "") + ")")}


# ------------------------------------------------------------------- main
PREC_DTYPE = {"mixed": "f64 state + f32 pair terms", "fp64": "f64"}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference_arm(args, world, rank)

    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    t_prep = time.perf_counter()
    d, info = prepared_state(args, rank)
    nv, npr = d.numVertices, d.numParticles
    if args.profile_build:
        # forced one-launch builds of the list (the rebuild a step sequence
        # runs when the displacement check fires), timed with CUDA events
        import torch

        cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
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
        return
    if args.profile_kernel:
        d.setPrecision(args.precision)
        ms = d.profileStepKernel(3)
        print(json.dumps({"profile_kernel_ms": ms, "vertices": nv, "lanes": d.getLanes(),
                          "precision": args.precision}), flush=True)
        d.close()
        return
    c = info["config"]
    d.setTimeStep(c["dt"])
    d.setSeed(1000 + rank)
    d.initNVE(c["T"], readState=False)
    cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
    # the thermal start state that every run below begins from
    x0, v0 = d.getVertexPositions(), d.getVertexVelocities()
    t_prep = time.perf_counter() - t_prep

    import ctypes

    sp = ctypes.c_void_p()
    d._call("cr_get_stream", ctypes.byref(sp))
    stream = torch.cuda.ExternalStream(sp.value)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    M = args.md_steps

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
                "clocks": clocks.summary(), "x_warm": x_warm}

    def kernel_roofline(precision):
        d.setPrecision(precision)
        ms_launch = ctypes.c_double()
        d._call("cr_profile_step_kernel", 200, ctypes.byref(ms_launch))
        bytes_per_launch = 88 * nv + 8 * npr
        achieved = bytes_per_launch / (ms_launch.value * 1e-3) / 1e9
        return ms_launch.value, bytes_per_launch, achieved

    prim = args.precision
    run = timed_run(prim)
    value = run["value"]
    x_end = d.getVertexPositions()

    # e2e through the public API with host buffers (same precision)
    e2e = None
    if not args.no_e2e:
        hpos = torch.empty(2 * nv, dtype=torch.float64, pin_memory=True).numpy()
        hvel = torch.empty(2 * nv, dtype=torch.float64, pin_memory=True).numpy()
        hpos[:] = d.getVertexPositions()
        hvel[:] = d.getVertexVelocities()
        n_e2e = max(1, min(args.steps, 5))
        barrier(world)
        torch.cuda.synchronize()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record(stream)
        for _ in range(n_e2e):
            d.setVertexPositions(hpos)
            d.setVertexVelocities(hvel)
            d.NVELoop(M)
            hpos[:] = d.getVertexPositions()
            hvel[:] = d.getVertexVelocities()
            _ = d.getPotentialEnergy()
        eb.record(stream)
        torch.cuda.synchronize()
        ms_e2e = max_over_ranks(ea.elapsed_time(eb), world)
        e2e = {"value": nv * M * n_e2e * world / (ms_e2e / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 2 * 16 * nv, "d2h_bytes_per_step": 2 * 16 * nv + 8}

    # roofline of the dominant kernel.  The middle steps of each NVELoop run in
    # the multi-step kernel (up to 64 steps per launch, grid barriers between
    # steps), so the unit is one step: algorithmic bytes per step over the
    # device time per step of the timed region (CUDA events on the library's
    # stream; rebuild launches included).  The single-step kernel timed alone
    # (back-to-back launches) is reported beside it.
    ms_launch, bytes_per_launch, iso_achieved = kernel_roofline(prim)
    step_s = run["ms_total"] * 1e-3 / (args.steps * M)
    achieved = bytes_per_launch / step_s / 1e9
    peaks = measured_peaks()
    traffic = committed_traffic(prim)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": traffic.get("bytes_per_launch") if traffic else None,
                "kernel": f"k_tile_steps<LJ, smooth, {prim}> (multi-step) + k_nbr_fused rebuilds",
                "us_per_step": step_s * 1e6, "algorithmic_bytes_per_step": bytes_per_launch,
                "traffic_note": "DRAM bytes of one single-step launch of the same step body (ncu, cold L2)",
                "single_step_kernel": {"kernel": f"k_tile<LJ, smooth, step, {prim}>", "ms_per_launch": ms_launch,
                                       "achieved": iso_achieved, "frac": iso_achieved / peaks["hbm_gbs"]}}

    comparison = None
    if not args.no_compare:
        other = "fp64" if prim == "mixed" else "mixed"
        orun = timed_run(other)
        oms, _, oach = kernel_roofline(other)
        o_step_s = orun["ms_total"] * 1e-3 / (args.steps * M)
        comparison = {other: {"value": orun["value"], "ms_per_step": orun["ms_total"] / args.steps,
                              "us_per_md_step": o_step_s * 1e6,
                              "roofline_frac": bytes_per_launch / o_step_s / 1e9 / peaks["hbm_gbs"],
                              "single_step_kernel_ms_per_launch": oms,
                              "gpu_launches": orun["launches"], "clocks": orun["clocks"]}}
        fp64_value = orun["value"] if prim == "mixed" else value
        mixed_value = value if prim == "mixed" else orun["value"]
        comparison["mixed_over_fp64"] = mixed_value / fp64_value
        comparison["accuracy"] = precision_accuracy(d, cut, [run["x_warm"], x_end], v0, args.drift_steps, restart)

    batch = None
    if rank == 0 and not args.no_batch:
        batch = batched_fire_measurement(args.batch_systems)

    rigid = None
    if rank == 0 and not args.no_rigid:
        rigid = rigid_ellipse_measurement(args.rigid_steps)

    deriv = None
    if rank == 0 and not args.no_diff:
        deriv = derivative_measurement()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        steps_per_rebuild = (M * args.steps / run["updates"]) if run["updates"] else None
        cpu = cpu_reference_rate(d, c, os.cpu_count() or 1, rebuild_every=steps_per_rebuild)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run["ms_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": PREC_DTYPE[prim],
            "data": "synthetic: seeded rings placed at phi 0.40, FIRE-compressed to 0.85, T=0.01 velocities",
            "config": {"workload": f"{npr} deformable rings nv 32/45 (1:1.4), {nv} vertices, smooth vertex-segment "
                                   f"LJ rc 2.5, calA0 1.05, phi 0.85, ea {c['ea']:g} el {c['el']:g} "
                                   f"eb {c['eb']:g}, NVE dt 0.002, precision {prim}",
                       "precision": prim, "rings": npr, "vertices": nv, "md_steps_per_bench_step": M,
                       "l2": "flushed between bench steps (256 MB write)", "parallelism": f"replicas x{world}",
                       "neighbour_rebuilds_in_timed_region": run["updates"],
                       "energy_change_rel_timed_region": run["energy_change_rel"],
                       "prep_seconds": t_prep, "fire_iterations_prep": info["fire_iterations"],
                       "lanes_per_vertex": info["lanes"]},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": run["launches"],
            "clocks": run["clocks"], "precision_comparison": comparison, "batched_systems": batch,
            "rigid_ellipses": rigid, "derivatives": deriv,
        }
        print(json.dumps(line), flush=True)
    d.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


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
    t1 = time.perf_counter()
    g = diff.minimized_gradients(d, float(np.mean(c["calA0"])) if np.ndim(c["calA0"]) else float(c["calA0"]),
                                 tol=1e-10)
    t_grad = time.perf_counter() - t1
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


def batched_fire_measurement(num_systems: int, fire_iters: int = 2000, loop_systems: int = 8) -> dict:
    """Many independent systems in one launch per op (cr_batch_*): the FIRE
    throughput of the batch against the per-system single-context loop on the
    same states, plus a bounded sample of the compression protocol.

    Workload: ``num_systems`` deformable-ring packings, ring counts uniform in
    [16, 512], bidisperse 1:1.4 with nv 16/22, calA0 uniform in [1.0, 1.2],
    harmonic repulsion, brought to packing fraction 0.60 (untimed).  Timed:
    FIRE to max |F| <= 1e-10 / sigma (at most ``fire_iters`` iterations) on
    every system, as vertex-iterations per second; the per-system loop runs
    the same minimisation on ``loop_systems`` of them one at a time."""
    import torch

    from cudaring_b200 import DPM2D
    from cudaring_b200.batch import Batch
    from cudaring_b200.compress import batch_packings, prepare_batch

    t0 = time.perf_counter()
    pks = batch_packings(num_systems, seed=20261207)
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    b = Batch.from_packings(pks, **kw)
    prepare_batch(b, 0.60, step=0.03, tol0=1e-6, max_fire_iters=5000)
    lanes = b.autotune(10)
    t_prep = time.perf_counter() - t0
    nvs = np.array([p.num_vertices for p in pks])
    pos, rad, l0, a0 = b.getVertexPositions(), b.getVertexRadii(), b.getRestLengths(), b.getRestAreas()
    out = {"workload": f"{num_systems} systems, {int(nvs.sum())} vertices, rings U[16,512] nv 16/22, harmonic, "
                       f"phi 0.60, FIRE to 1e-10/sigma (<= {fire_iters} iterations)",
           "unit": "vertex-iterations/s", "lanes_per_vertex": lanes, "prep_seconds": t_prep}
    for prec in ("fp64", "mixed"):
        b.setVertexPositions(pos)
        b.setVertexVelocities(np.zeros_like(pos))
        b.setPrecision(prec)
        sig = b.getMeanParticleSizes()
        b.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-2, 1e-1, 0.2], 20, dt=1e-2 * sig)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        its, fmax = b.fireMinimize(1e-10 / sig, fire_iters)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[prec] = {"value": float((its * nvs).sum()) / dt, "seconds": dt, "iterations_mean": float(its.mean()),
                     "converged_systems": int((fmax <= 1e-10 / sig).sum())}
    # the per-system loop: the same minimisation through single contexts
    vi, tt = 0.0, 0.0
    for s in range(min(loop_systems, num_systems)):
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
    out["per_system_loop_fp64"] = {"value": vi / tt, "systems": min(loop_systems, num_systems),
                                   "sample": "the first systems of the batch, one single-system context each"}
    out["batch_over_loop_fp64"] = out["fp64"]["value"] / out["per_system_loop_fp64"]["value"]
    # compression protocol sample (compressFIRE.cpp:101-205) from phi 0.60
    b.setVertexPositions(pos)
    b.setVertexVelocities(np.zeros_like(pos))
    b.setPrecision("fp64")
    t0 = time.perf_counter()
    res = b.compress(dphi=1e-3, min_dphi=1e-6, fire_dt=1e-2, tol0=1e-10, max_fire_iters=20000, max_steps=3)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    out["compression_sample"] = {"steps": 3, "dphi": 1e-3, "seconds": dt,
                                 "value": float((res["fire_iterations"] * nvs).sum()) / dt,
                                 "phi_mean": float(res["phi"].mean())}
    b.close()
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
    if rank != 0:
        return
    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcrref.so was not built "
                                                              "(needs the reference checkout at build time)"}))
        return
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    # same prepared state, built on the GPU when one is present, else on the CPU port
    from cudaring_b200 import workloads

    d, info = workloads.prepared_deformable("smooth_lj", args.rings, seed=20261203)
    c = info["config"]
    R = oracle.ref()
    nvl = d.numVertexInParticleList
    pos, rad, l0, a0 = d.getVertexPositions(), d.getVertexRadii(), d.getRestLengths(), d.getRestAreas()
    rng = np.random.default_rng(1000)
    vel = np.repeat(rng.normal(0.0, np.sqrt(c["T"]), size=(len(nvl), 2)), nvl, axis=0).reshape(-1)
    th0 = np.repeat(2 * np.pi / nvl, nvl).astype(np.float64)
    box = d.getBoxSize()
    R.ref_create(len(nvl), nvl)
    R.ref_set_box(float(box[0]), float(box[1]))
    R.ref_set_types(1, 1, 0, 0)
    R.ref_set_energy_costs(c["ea"], c["el"], c["eb"], c["ec"])
    R.ref_set_lj_cutoff(c["LJcutoff"])
    R.ref_set_time_step(c["dt"])
    R.ref_set_state(pos.ctypes.data, vel.ctypes.data, rad.ctypes.data, l0.ctypes.data, th0.ctypes.data, a0.ctypes.data)
    cut = R.ref_set_displacement_cutoff(0.5, 2 * rad.mean())
    t0 = time.perf_counter()
    R.ref_calc_neighbor_list(cut)
    t_build = time.perf_counter() - t0
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    # each bench step: single NVE steps until ~5 s have passed (rebuilds,
    # O(Nv^2) scans in the reference, included as they fall due)
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
    value = d.numVertices * total_steps / t
    gpu_build = reference_cuda_build(d, c, vel)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (same prepared state as the ours arm)",
            "config": {"workload": f"{d.numParticles} deformable rings, {d.numVertices} vertices, smooth LJ, phi 0.85,"
                                   f" NVE dt 0.002", "md_steps_per_bench_step": per,
                       "rebuilds_in_sample": upd, "list_build_seconds": t_build},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{total_steps} NVE steps in {t:.1f} s, reference kernels as host code, "
                                       f"{threads} OpenMP threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_cuda_build": gpu_build}
    print(json.dumps(line), flush=True)
    d.close()


def reference_cuda_build(d, c: dict, vel: np.ndarray, warmup: int = 100, steps: int = 2000) -> dict | None:
    """The reference's own CUDA build (oracle/_ref/ref_gpu_nve, compiled from
    its sources) on the same prepared state and thermal velocities, read from
    the reference's on-disk packing format; timed with CUDA events inside it."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_nve")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_gpu_nve was not built (needs the reference checkout at build time)"}
    import tempfile

    from cudaring_b200 import packing_io, synth

    nvl = d.numVertexInParticleList
    pk = synth.Packing(nv_list=nvl, pos=d.getVertexPositions(), vel=vel, rad=d.getVertexRadii(), l0=d.getRestLengths(),
                       theta0=d.getRestAngles(), a0=d.getRestAreas(), box=d.getBoxSize(),
                       centres=np.zeros((len(nvl), 2)))
    with tempfile.TemporaryDirectory() as tmp:
        packing_io.save_packing_arrays(tmp, pk, digits=17)
        try:
            r = subprocess.run([exe, tmp, str(len(nvl)), str(warmup), str(steps), repr(c["dt"]), repr(c["ea"]),
                                repr(c["el"]), repr(c["eb"]), "lj", "smooth", repr(c["LJcutoff"])],
                               capture_output=True, text=True, timeout=600)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference CUDA build did not finish within 600 s"}
    if r.returncode != 0 or not r.stdout.strip():
        return {"unavailable": f"reference CUDA build exited {r.returncode}: {r.stderr.strip()[-200:]}"}
    info = json.loads(r.stdout.strip().splitlines()[-1])
    return {"value": info["vertex_steps_per_s"], "unit": UNIT, "ms_per_step": info["ms_per_step"],
            "steps": info["steps"], "warmup": info["warmup"], "rebuilds": info["updates"],
            "sample": f"farceri/cudaRing DPM2D compiled for sm_100a, NVELoop() x {steps} after {warmup} warm-up "
                      f"steps on the same {d.numVertices}-vertex state, CUDA-event timed"}


if __name__ == "__main__":
    main()
