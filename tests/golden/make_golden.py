"""Generates the golden fixtures in tests/golden/ from the reference itself.

The outputs are computed by oracle/_ref/libcrref.so -- farceri/cudaRing's own
kernels (include/cudaKernel.cuh) compiled as host code by oracle/build_ref.sh
-- on seeded inputs built with cudaring_b200.synth.  Inputs and outputs are
stored together, so the tests do not depend on the generator staying
bit-identical.  Run from the repository root, where the reference checkout
is available:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from cudaring_b200 import synth  # noqa: E402
from oracle.integrators import philox_noise  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# Force/energy/neighbour cases: (name, rings, potential, interaction, placement, phi, extra)
FORCE_CASES = [
    ("harmonic_vv_bidisperse", dict(workload="bidisperse_harmonic"), "harmonic", "vertexVertex", "uniform", 0.70, {}),
    ("harmonic_smooth", dict(workload="smooth_lj", n=48), "harmonic", "vertexSmooth", "uniform", 0.80, {}),
    ("lj_smooth", dict(workload="smooth_lj", n=64), "lennardJones", "vertexSmooth", "rsa", 0.40, {}),
    ("lj_vv", dict(workload="smooth_lj", n=64), "lennardJones", "vertexVertex", "rsa", 0.40, {}),
    ("wca_vv", dict(nv=24, n=64), "wca", "vertexVertex", "rsa", 0.40, {}),
    ("wca_smooth", dict(nv=24, n=64), "wca", "vertexSmooth", "rsa", 0.40, {}),
    ("adhesive_vv", dict(workload="bidisperse_harmonic"), "adhesive", "vertexVertex", "uniform", 0.70, dict(l1=0.1, l2=0.3)),
    ("adhesive_smooth", dict(workload="bidisperse_harmonic"), "adhesive", "vertexSmooth", "uniform", 0.70, dict(l1=0.1, l2=0.3)),
    ("fene_vv", dict(workload="bidisperse_harmonic"), "harmonic", "vertexVertex", "uniform", 0.70, dict(monomer=1, stiff=1.0, ext=1.5)),
]

FIELDS = {"pos": 0, "vel": 1, "force": 2, "energy": 3, "p_energy": 4, "area": 5, "perimeter": 6,
          "theta": 7, "length": 8, "ppos": 9}


def packing_for(spec, phi, placement, seed):
    if "workload" in spec:
        c = synth.workload_config(spec["workload"], spec.get("n"))
        nv, a0, calA0 = c["nv"], c["a0"], c["calA0"]
    else:
        n = spec["n"]
        nv, a0, calA0 = [spec["nv"]] * n, [1.0] * (n // 2) + [1.4 ** 2] * (n - n // 2), 1.0
    return synth.make_packing(nv, a0, calA0, phi, seed=seed, placement=placement)


def setup_ref(pk, potential, interaction, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj=2.5, l1=0.0, l2=0.0, monomer=0,
              stiff=0.0, ext=0.0):
    R = oracle.ref()
    R.ref_create(pk.num_particles, pk.nv_list)
    R.ref_set_box(float(pk.box[0]), float(pk.box[1]))
    R.ref_set_types(oracle.POTENTIALS[potential], oracle.INTERACTIONS[interaction], monomer, 0)
    R.ref_set_energy_costs(ea, el, eb, ec)
    R.ref_set_lj_cutoff(lj)
    R.ref_set_attraction(l1, l2)
    R.ref_set_fene(stiff, ext)
    R.ref_set_state(pk.pos.ctypes.data, pk.vel.ctypes.data, pk.rad.ctypes.data, pk.l0.ctypes.data,
                    pk.theta0.ctypes.data, pk.a0.ctypes.data)
    cut = R.ref_set_displacement_cutoff(0.5, 2 * pk.rad.mean())
    return R, cut


def grab(R, pk, names):
    out = {}
    sizes = dict(pos=2 * pk.num_vertices, vel=2 * pk.num_vertices, force=2 * pk.num_vertices,
                 energy=pk.num_vertices, p_energy=pk.num_particles, area=pk.num_particles,
                 perimeter=pk.num_particles, theta=pk.num_vertices, length=pk.num_vertices, ppos=2 * pk.num_particles)
    for n in names:
        a = np.zeros(sizes[n])
        R.ref_get(FIELDS[n], a)
        out["out_" + n] = a
    return out


def inputs(pk, **params):
    d = {"nv_list": pk.nv_list, "pos": pk.pos, "vel": pk.vel, "rad": pk.rad, "l0": pk.l0, "theta0": pk.theta0,
         "a0": pk.a0, "box": pk.box}
    for k, v in params.items():
        d["param_" + k] = np.asarray(v)
    return d


def force_cases():
    for idx, (name, spec, pot, inter, placement, phi, extra) in enumerate(FORCE_CASES):
        pk = packing_for(spec, phi, placement, seed=20261203 + 100 + idx)
        kw = dict(l1=extra.get("l1", 0.0), l2=extra.get("l2", 0.0), monomer=extra.get("monomer", 0),
                  stiff=extra.get("stiff", 0.0), ext=extra.get("ext", 0.0))
        R, cut = setup_ref(pk, pot, inter, **kw)
        R.ref_calc_neighbor_list(cut)
        ls = R.ref_neighbor_list_size()
        nbr = np.zeros(pk.num_vertices * max(ls, 1), np.int64)
        cnt = np.zeros(pk.num_vertices, np.int64)
        R.ref_get_neighbors(nbr)
        R.ref_get_max_neighbor_list(cnt)
        R.ref_calc_force_energy()
        d = inputs(pk, potential=oracle.POTENTIALS[pot], interaction=oracle.INTERACTIONS[inter], ea=1.0, el=1.0,
                   eb=0.01, ec=1.0, lj_cutoff=2.5, cut_distance=cut, **kw)
        d.update(grab(R, pk, ["force", "energy", "p_energy", "area", "perimeter", "theta", "length", "ppos"]))
        d["out_neighbors"] = nbr[: pk.num_vertices * ls]
        d["out_max_neighbor_list"] = cnt
        d["out_list_size"] = np.asarray(ls)
        d["out_potential_energy"] = np.asarray(R.ref_potential_energy())
        np.savez_compressed(os.path.join(OUT, f"force_{name}.npz"), **d)
        print(f"force_{name}: nv={pk.num_vertices} listSize={ls} maxF={np.abs(d['out_force']).max():.3e}")


def traj_cases():
    # NVE on the 32-ring bidisperse harmonic geometry with ring-rigid velocities large enough to trigger rebuilds.
    pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 200)
    rng = np.random.default_rng(7)
    pk.vel = np.repeat(rng.normal(0.0, 0.3, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    dt, nsteps = 0.005, 200
    R, cut = setup_ref(pk, "harmonic", "vertexVertex")
    R.ref_set_time_step(dt)
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    R.ref_nve_loop(nsteps)
    d = inputs(pk, potential=0, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt,
               nsteps=nsteps, cut_distance=cut)
    d.update(grab(R, pk, ["pos", "vel", "force", "energy"]))
    d["out_update_count"] = np.asarray(R.ref_update_count())
    d["out_potential_energy"] = np.asarray(R.ref_potential_energy())
    d["out_kinetic_energy"] = np.asarray(R.ref_kinetic_energy())
    np.savez_compressed(os.path.join(OUT, "traj_nve_harmonic_vv.npz"), **d)
    print(f"traj_nve_harmonic_vv: updates={int(d['out_update_count'])}")

    # NVE, smooth LJ, 64 rings.
    pk = packing_for(dict(workload="smooth_lj", n=64), 0.40, "rsa", seed=20261203 + 201)
    pk.vel = np.repeat(rng.normal(0.0, 0.3, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    dt, nsteps = 0.002, 150
    R, cut = setup_ref(pk, "lennardJones", "vertexSmooth")
    R.ref_set_time_step(dt)
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    R.ref_nve_loop(nsteps)
    d = inputs(pk, potential=1, interaction=1, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt,
               nsteps=nsteps, cut_distance=cut)
    d.update(grab(R, pk, ["pos", "vel", "force", "energy", "p_energy"]))
    d["out_update_count"] = np.asarray(R.ref_update_count())
    d["out_potential_energy"] = np.asarray(R.ref_potential_energy())
    np.savez_compressed(os.path.join(OUT, "traj_nve_lj_smooth.npz"), **d)
    print(f"traj_nve_lj_smooth: updates={int(d['out_update_count'])}")

    # FIRE on the 32-ring bidisperse harmonic geometry.
    pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 202)
    R, cut = setup_ref(pk, "harmonic", "vertexVertex")
    dt = 0.01
    params = np.array([0.2, 0.5, 1.1, 0.99, dt, 10 * dt, 0.2])
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    R.ref_fire_init(params, 20, 0)
    nsteps = 300
    R.ref_fire_loop(nsteps)
    st = np.zeros(3)
    R.ref_fire_state(st)
    d = inputs(pk, potential=0, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, nsteps=nsteps,
               fire=params, cut_distance=cut)
    d.update(grab(R, pk, ["pos", "vel", "force", "energy"]))
    d["out_fire_state"] = st
    d["out_max_unbalanced_force"] = np.asarray(R.ref_max_unbalanced_force())
    d["out_potential_energy"] = np.asarray(R.ref_potential_energy())
    np.savez_compressed(os.path.join(OUT, "traj_fire_harmonic_vv.npz"), **d)
    print(f"traj_fire_harmonic_vv: maxF={float(d['out_max_unbalanced_force']):.3e} state={st}")

    # Langevin with the library's Philox noise (seed, streams 2s) injected.
    pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 203)
    pk.vel = np.repeat(rng.normal(0.0, 0.1, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    dt, nsteps, T, gamma, seed = 0.005, 60, 0.01, 1.0, 12345
    R, cut = setup_ref(pk, "harmonic", "vertexVertex")
    R.ref_set_time_step(dt)
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    xi = np.concatenate([philox_noise(seed, 2 * s, pk.num_particles).reshape(-1) for s in range(nsteps)])
    noise_amp = np.sqrt(2.0 * T * gamma / dt)
    R.ref_langevin_loop(nsteps, gamma, noise_amp, xi.ctypes.data, 0.0, None)
    d = inputs(pk, potential=0, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt,
               nsteps=nsteps, T=T, gamma=gamma, seed=seed, cut_distance=cut)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    np.savez_compressed(os.path.join(OUT, "traj_langevin_harmonic_vv.npz"), **d)
    print("traj_langevin_harmonic_vv: done")


RIGID_FIELDS = {"torque": 11, "p_force": 12, "p_torque": 13, "p_angle": 14, "moi": 15, "p_vel": 16,
                "p_angvel": 17}


def stochastic_cases():
    # BAOAB, Brownian, driven Brownian and active Langevin with the library's
    # Philox draws (seed, stream 2s for the thermostat of step s, 2s+1 for the
    # self-propulsion angle) injected into the reference kernels.
    seed = 4242
    pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 204)
    rng = np.random.default_rng(5)
    vel = np.repeat(rng.normal(0.0, 0.1, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    npart = pk.num_particles
    dt, T, gamma, nsteps = 0.005, 0.01, 1.0, 60

    def fresh():
        pk.vel = vel.copy()
        R, cut = setup_ref(pk, "harmonic", "vertexVertex")
        R.ref_set_time_step(dt)
        R.ref_calc_neighbor_list(cut)
        R.ref_reset_last_positions()
        R.ref_calc_force_energy()
        return R, cut

    xi = np.concatenate([philox_noise(seed, 2 * s, npart).reshape(-1) for s in range(nsteps)])
    common = dict(potential=0, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt, nsteps=nsteps,
                  T=T, gamma=gamma, seed=seed)

    R, cut = fresh()
    gf = np.exp(-gamma * dt)
    amp = np.sqrt(1 - np.exp(-2 * gamma * dt)) * np.sqrt(T)
    R.ref_baoab_loop(nsteps, gf, amp, xi.ctypes.data)
    d = inputs(pk, cut_distance=cut, **common)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    np.savez_compressed(os.path.join(OUT, "traj_baoab_harmonic_vv.npz"), **d)

    R, cut = fresh()
    amp = np.sqrt(2.0 * T * gamma / dt)
    R.ref_brownian_loop(nsteps, gamma, amp, xi.ctypes.data, 0.0, None)
    d = inputs(pk, cut_distance=cut, **common)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    np.savez_compressed(os.path.join(OUT, "traj_brownian_harmonic_vv.npz"), **d)

    R, cut = fresh()
    R.ref_brownian_loop(nsteps, gamma, amp, None, 0.0, None)
    d = inputs(pk, cut_distance=cut, **common)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    np.savez_compressed(os.path.join(OUT, "traj_drivenbrownian_harmonic_vv.npz"), **d)

    # active rings under Langevin: f0 = 0.05, taup = 10
    driving, taup = 0.05, 10.0
    R, cut = fresh()
    R.ref_set_types(0, 0, 0, 1)
    sp_amp = np.sqrt(2.0 * dt / taup)
    dpsi = np.concatenate([sp_amp * philox_noise(seed, 2 * s + 1, npart)[:, 0] for s in range(nsteps)])
    R.ref_langevin_loop(nsteps, gamma, amp, xi.ctypes.data, driving, dpsi.ctypes.data)
    d = inputs(pk, cut_distance=cut, driving=driving, taup=taup, **common)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    ang = np.zeros(npart)
    R.ref_get(14, ang)
    d["out_p_angle"] = ang
    np.savez_compressed(os.path.join(OUT, "traj_active_langevin_harmonic_vv.npz"), **d)
    print("stochastic cases: done")


def rigid_cases():
    # Rigid bumpy ellipses, WCA vertex-vertex: an NVE run from a non-overlapping
    # placement, then the force/torque sums at its final (colliding) state.
    pk = synth.make_ellipse_packing(64, 24, (1.2, 2.0), 0.25, seed=20261203 + 300)
    rng = np.random.default_rng(11)
    pvel = rng.normal(0.0, 0.3, 2 * pk.num_particles)
    pang = rng.normal(0.0, 0.5, pk.num_particles)
    dt, nsteps = 0.002, 400
    R, cut = setup_ref(pk, "wca", "vertexVertex")
    R.ref_set_time_step(dt)
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_rigid_force_energy()
    R.ref_set_particle_state(None, pvel.ctypes.data, None, pang.ctypes.data)
    R.ref_rigid_nve_loop(nsteps)
    d = inputs(pk, potential=3, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt,
               nsteps=nsteps, cut_distance=cut)
    d["p_vel"] = pvel
    d["p_angvel"] = pang
    d.update(grab(R, pk, ["pos", "ppos", "force"]))
    for name, fid, n in (("p_vel", 16, 2 * pk.num_particles), ("p_angvel", 17, pk.num_particles),
                         ("p_angle", 14, pk.num_particles), ("p_force", 12, 2 * pk.num_particles)):
        a = np.zeros(n)
        R.ref_get(fid, a)
        d["out_" + name] = a
    d["out_update_count"] = np.asarray(R.ref_update_count())
    np.savez_compressed(os.path.join(OUT, "traj_rigid_nve_wca.npz"), **d)
    print(f"traj_rigid_nve_wca: updates={int(d['out_update_count'])} maxF={np.abs(d['out_force']).max():.3e}")

    pk.pos = d["out_pos"].copy()
    R, cut = setup_ref(pk, "wca", "vertexVertex")
    R.ref_calc_neighbor_list(cut)
    R.ref_calc_rigid_force_energy()
    d = inputs(pk, potential=3, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, cut_distance=cut)
    d.update(grab(R, pk, ["force", "energy", "p_energy", "ppos"]))
    for name, fid in (("torque", 11), ("p_force", 12), ("p_torque", 13), ("moi", 15)):
        n = pk.num_vertices if name == "torque" else (2 if name == "p_force" else 1) * pk.num_particles
        a = np.zeros(n)
        R.ref_get(fid, a)
        d["out_" + name] = a
    np.savez_compressed(os.path.join(OUT, "rigid_force_wca.npz"), **d)
    print(f"rigid_force_wca: nv={pk.num_vertices} maxF={np.abs(d['out_force']).max():.3e}")


def rescale_cases():
    # NVE with velocity rescaling to Tinject before every step (NVERescale).
    pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 205)
    rng = np.random.default_rng(9)
    pk.vel = np.repeat(rng.normal(0.0, 0.1, size=(pk.num_particles, 2)), pk.nv_list, axis=0).reshape(-1)
    dt, nsteps, Tinject = 0.005, 120, 0.02
    R, cut = setup_ref(pk, "harmonic", "vertexVertex")
    R.ref_set_time_step(dt)
    R.ref_calc_neighbor_list(cut)
    R.ref_reset_last_positions()
    R.ref_calc_force_energy()
    R.ref_nve_rescale_loop(nsteps, Tinject)
    d = inputs(pk, potential=0, interaction=0, ea=1.0, el=1.0, eb=0.01, ec=1.0, lj_cutoff=2.5, dt=dt,
               nsteps=nsteps, T=Tinject, cut_distance=cut)
    d.update(grab(R, pk, ["pos", "vel", "force"]))
    d["out_update_count"] = np.asarray(R.ref_update_count())
    np.savez_compressed(os.path.join(OUT, "traj_nverescale_harmonic_vv.npz"), **d)
    print(f"traj_nverescale_harmonic_vv: updates={int(d['out_update_count'])}")


def soft_cases():
    # Soft-disk pre-packing (compressFIRE.cpp:53-90) from a unit box, as the
    # reference driver starts: setRandomParticles, the particle list, forces,
    # 10 FIRE iterations, the full FIRE minimisation and initVerticesOnParticles.
    cases = [("harmonic", 0, 1.0, 0.8, dict(), True), ("wca", 3, 1.0, 0.35, dict(), False),
             ("lj", 1, 3.0, 0.35, dict(lj=2.5), False)]
    for name, pot, cut, phi0, extra, full in cases:
        pk = packing_for(dict(workload="bidisperse_harmonic"), 0.70, "uniform", seed=20261203 + 301)
        extra_rad, seed = 1.1, 4242
        R = oracle.ref()
        R.ref_create(pk.num_particles, pk.nv_list)
        R.ref_set_box(1.0, 1.0)
        R.ref_set_types(pot, 0, 0, 0)
        R.ref_set_energy_costs(1.0, 1.0, 0.01, 1.0)
        R.ref_set_lj_cutoff(extra.get("lj", 2.5))
        R.ref_set_state(pk.pos.ctypes.data, pk.vel.ctypes.data, pk.rad.ctypes.data, pk.l0.ctypes.data,
                        pk.theta0.ctypes.data, pk.a0.ctypes.data)
        R.ref_set_random_particles(phi0, extra_rad, seed)
        n_p, n_v = pk.num_particles, pk.num_vertices
        geo = np.zeros(n_p + 2 * n_v + 2)
        R.ref_get_geometry(geo)
        d = dict(in_nv_list=np.asarray(pk.nv_list), in_a0=pk.a0, in_l0=pk.l0, in_rad=pk.rad, in_theta0=pk.theta0,
                 in_pos=pk.pos, param_potential=np.asarray(pot), param_lj_cutoff=np.asarray(extra.get("lj", 2.5)),
                 param_phi0=np.asarray(phi0), param_extra_rad=np.asarray(extra_rad), param_seed=np.asarray(seed),
                 param_cut=np.asarray(cut))
        d["out_a0"], d["out_l0"], d["out_rad"] = geo[:n_p], geo[n_p:n_p + n_v], geo[n_p + n_v:n_p + 2 * n_v]
        d["out_box"] = geo[-2:]
        d["out_ppos"] = np.zeros(2 * n_p)
        R.ref_get(9, d["out_ppos"])
        d["out_prad"] = np.zeros(n_p)
        R.ref_get_particle_radii(d["out_prad"])
        R.ref_calc_particle_neighbor_list(cut)
        ls = R.ref_particle_neighbor_list_size()
        d["out_plist_size"] = np.asarray(ls)
        d["out_pneighbors"] = np.zeros(n_p * ls, dtype=np.int64)
        R.ref_get_particle_neighbors(d["out_pneighbors"])
        d["out_pmax"] = np.zeros(n_p, dtype=np.int64)
        R.ref_get_particle_max_neighbor_list(d["out_pmax"])
        R.ref_calc_particle_force_energy()
        d["out_pforce"], d["out_penergy"] = np.zeros(2 * n_p), np.zeros(n_p)
        R.ref_get(12, d["out_pforce"])
        R.ref_get(4, d["out_penergy"])
        # FIRE as compressFIRE.cpp:58-65 sets it up: dt = 10 * 1e-2 * mean particle size
        sigma = 2 * np.sqrt(d["out_a0"].sum() / (np.pi * n_p))
        step = 10 * 1e-2 * sigma
        p7 = np.array([0.2, 0.5, 1.1, 0.99, step, 10 * step, 0.2])
        d["param_fire"] = p7
        d["param_min_step"] = np.asarray(20)
        R.ref_particle_fire_init(p7, 20, 0)
        R.ref_particle_fire_loop(10)
        d["out_fire10_ppos"], d["out_fire10_pvel"] = np.zeros(2 * n_p), np.zeros(2 * n_p)
        R.ref_get(9, d["out_fire10_ppos"])
        R.ref_get(16, d["out_fire10_pvel"])
        d["out_fire10_state"] = np.zeros(3)
        R.ref_fire_state(d["out_fire10_state"])
        if full:
            # restart from the random state for the driver loop
            R.ref_set_soft_particles(d["out_ppos"].ctypes.data, d["out_prad"].ctypes.data)
            R.ref_set_particle_state(None, np.zeros(2 * n_p).ctypes.data, None, None)
            R.ref_calc_particle_neighbor_list(cut)
            R.ref_calc_particle_force_energy()
            R.ref_particle_fire_init(p7, 20, 0)
            tol = 1e-10 / d["out_prad"].mean()
            d["param_tol"] = np.asarray(tol)
            d["out_min_iters"] = np.asarray(R.ref_particle_fire_minimize(cut, tol, 1000000))
            d["out_min_ppos"] = np.zeros(2 * n_p)
            R.ref_get(9, d["out_min_ppos"])
            d["out_min_maxf"] = np.asarray(R.ref_particle_max_unbalanced_force())
            d["out_min_pe"] = np.asarray(R.ref_particle_potential_energy())
            draws = np.zeros(2 * n_v)
            R.ref_drand48_stream(7, 0, 2 * n_v, draws)
            d["in_draws"] = draws
            R.ref_init_vertices_on_particles(draws)
            d["out_vpos"] = np.zeros(2 * n_v)
            R.ref_get(0, d["out_vpos"])
        np.savez_compressed(os.path.join(OUT, f"soft_{name}.npz"), **d)
        print(f"soft_{name}: np={n_p} list={ls} maxF={np.abs(d['out_pforce']).max():.3e}"
              + (f" iters={int(d['out_min_iters'])}" if full else ""))


def phi_cases():
    """DPM2D::getPhi (src/DPM2D.cu:1202-1220, current ring areas plus the vertex
    caps) and getPreferredPhi (:1222-1238, rest areas) on packings of three
    workloads, the first two deformed away from their rest shapes."""
    specs = [("smooth_lj", dict(workload="smooth_lj", n=64), "rsa", 0.40, 1.00),
             ("bidisperse", dict(workload="bidisperse_harmonic"), "uniform", 0.70, 0.97),
             ("monodisperse", dict(nv=24, n=64), "uniform", 0.55, 1.00)]
    d = {}
    for idx, (name, spec, placement, phi, squeeze) in enumerate(specs):
        pk = packing_for(spec, phi, placement, seed=20261203 + 500 + idx)
        if squeeze != 1.0:
            # ring areas away from a0: squeeze every ring along x about its centroid
            pos = pk.pos.reshape(-1, 2).copy()
            first = np.concatenate([[0], np.cumsum(pk.nv_list)[:-1]])
            for f, n in zip(first, pk.nv_list):
                c = pos[f:f + n].mean(axis=0)
                pos[f:f + n, 0] = c[0] + squeeze * (pos[f:f + n, 0] - c[0])
            pk.pos = pos.reshape(-1)
        R, _ = setup_ref(pk, "harmonic", "vertexVertex")
        R.ref_calc_force_energy()
        for k, v in inputs(pk).items():
            d[f"{name}_{k}"] = v
        d[f"{name}_out_phi"] = np.asarray(R.ref_phi())
        d[f"{name}_out_preferred_phi"] = np.asarray(R.ref_preferred_phi())
        print(f"phi_{name}: phi={float(d[name + '_out_phi']):.15f} preferred={float(d[name + '_out_preferred_phi']):.15f}")
    d["names"] = np.array([s[0] for s in specs])
    np.savez_compressed(os.path.join(OUT, "phi_cases.npz"), **d)


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build()
    which = sys.argv[1:] or ["force", "traj", "stochastic", "rigid", "rescale", "soft", "phi"]
    if "force" in which:
        force_cases()
    if "traj" in which:
        traj_cases()
    if "stochastic" in which:
        stochastic_cases()
    if "rigid" in which:
        rigid_cases()
    if "rescale" in which:
        rescale_cases()
    if "soft" in which:
        soft_cases()
    if "phi" in which:
        phi_cases()
