"""Oracle integrators: numpy restatements of the reference's step functions.

TEST INFRASTRUCTURE ONLY.  Forces come from the C restatement (oracle.c);
the updates restate:

* ``NVE::integrate`` (src/Simulator.cu:206-212),
* ``NVERescale::integrate`` (src/Simulator.cu:215-238),
* ``Langevin::integrate`` / ``updateThermalVel`` (src/Simulator.cu:23-30, 54-77),
* ``BAOAB::integrate`` (src/Simulator.cu:112-144),
* ``Brownian::integrate`` / ``DrivenBrownian`` (src/Simulator.cu:147-203),
* ``FIRE::minimizerVertexLoop`` (src/FIRE.cu:302-411),
* ``DPM2D::checkDisplacement`` with ``shift == false`` (src/DPM2D.cu:1390-1406).

Noise is injected by a callable ``noise(step) -> (Np, 2)`` array so that the
same draws can be fed to the reference kernels (oracle/_ref) and to this
restatement; ``philox_noise`` reproduces the library's counter-based stream.
"""
from __future__ import annotations

import math

import numpy as np

from . import System, normal2


class OracleState:
    def __init__(self, sys_: System, pk, cutoff_: float = 0.5, size_: float | None = None):
        self.s = sys_
        self.pos = pk.pos.copy()
        self.vel = pk.vel.copy()
        self.rad = pk.rad.copy()
        self.a0 = pk.a0.copy()
        self.l0 = pk.l0.copy()
        self.theta0 = pk.theta0.copy()
        size = 2 * self.rad.mean() if size_ is None else size_
        self.cut_distance = sys_.cut_distance(cutoff_)
        self.cutoff = cutoff_ * size
        self.update_count = 0
        self.rebuild()
        self.out = None
        self.forces()

    def rebuild(self):
        self.s.neighbor_list(self.pos, self.rad, self.cut_distance)
        self.last_pos = self.pos.copy()

    def check(self):
        d = (self.pos - self.last_pos).reshape(-1, 2)
        box = np.array([self.s.s.lx, self.s.s.ly])
        d -= box * np.round(d / box)
        if np.any(3 * np.sqrt((d * d).sum(1)) > self.cutoff):
            self.rebuild()
            self.update_count += 1

    def forces(self):
        self.out = self.s.force_energy(self.pos, self.rad, self.a0, self.l0, self.theta0)
        self.force = self.out["force"]
        return self.out

    def ring_of(self):
        return self.s.pid

    # ---------------------------------------------------------------- steps
    def nve_step(self, dt):
        self.vel += 0.5 * dt * self.force
        self.pos += dt * self.vel
        self.check()
        self.forces()
        self.vel += 0.5 * dt * self.force

    def self_propulsion(self, driving, dpsi):
        """DPM2D::addSelfPropulsion (src/DPM2D.cu:1995-2035) with given increments."""
        if not hasattr(self, "pangle"):
            self.pangle = np.zeros(self.s.np)
        a = self.pangle + dpsi + math.pi
        a = a - 2.0 * math.pi * np.floor(a / (2.0 * math.pi))
        self.pangle = a - math.pi
        p = self.pangle[self.s.pid]
        self.force = self.force + driving * np.stack([np.cos(p), np.sin(p)], axis=1).reshape(-1)

    def nve_rescale_step(self, dt, T_inject):
        """NVERescale::integrate / injectKineticEnergy (src/Simulator.cu:215-238)."""
        T = float(np.dot(self.vel, self.vel)) / len(self.vel)
        self.vel *= math.sqrt(T_inject / T)
        self.nve_step(dt)

    def langevin_step(self, dt, gamma, noise_amp, xi, driving=0.0, dpsi=None):
        self.vel += 0.5 * dt * self.force
        self.pos += dt * self.vel
        self.check()
        self.forces()
        if dpsi is not None:
            self.self_propulsion(driving, dpsi)
        r = xi[self.s.pid].reshape(-1)
        self.force = self.force + noise_amp * r - gamma * self.vel
        self.vel += 0.5 * dt * self.force

    def baoab_step(self, dt, gamma_factor, noise_amp, xi):
        self.vel += 0.5 * dt * self.force
        self.pos += 0.5 * dt * self.vel
        self.vel = gamma_factor * self.vel + noise_amp * xi[self.s.pid].reshape(-1)
        self.pos += 0.5 * dt * self.vel
        self.check()
        self.forces()
        self.vel += 0.5 * dt * self.force

    def brownian_step(self, dt, gamma, noise_amp, xi=None):
        self.check()
        self.forces()
        if xi is None:
            self.vel = self.force / gamma
        else:
            self.vel = (self.force + noise_amp * xi[self.s.pid].reshape(-1)) / gamma
        self.pos += dt * self.vel


class OracleFIRE:
    """FIRE scalars + iteration (src/FIRE.cu:29-41, 338-411)."""

    def __init__(self, params, min_step, num_step):
        self.a_start, self.f_dec, self.f_inc, self.f_a, self.dt, self.dt_max, self.a = params
        self.min_step = min_step
        self.num_step = num_step

    def iterate(self, st: OracleState):
        p = float(np.dot(st.vel, st.force))
        if p > 0:
            self.num_step += 1
            if self.num_step > self.min_step:
                self.dt = min(self.dt * self.f_inc, self.dt_max)
                self.a *= self.f_a
        else:
            self.num_step = 0
            self.dt = max(self.dt * self.f_dec, self.dt_max / 10)
            self.a = self.a_start
            st.pos -= 0.5 * self.dt * st.vel
            st.vel[:] = 0.0
        st.vel += 0.5 * self.dt * st.force
        vv = float(np.dot(st.vel, st.vel))
        ff = float(np.dot(st.force, st.force))
        if ff > 0:
            st.vel = (1 - self.a) * st.vel + self.a * st.force * math.sqrt(vv / ff)
        st.pos += self.dt * st.vel
        st.check()
        st.forces()
        st.vel += 0.5 * self.dt * st.force


class OracleRigid:
    """Rigid rings: RigidNVE::integrate (src/Simulator.cu:316-371) with forces
    from oc_rigid_force_energy and vertex moves from oc_translate_rotate."""

    def __init__(self, sys_: System, pk, cutoff_: float = 0.5):
        import ctypes as C

        from . import lib

        self.C, self.L = C, lib()
        self.s = sys_
        self.pos = pk.pos.copy()
        self.rad = pk.rad.copy()
        size = 2 * self.rad.mean()
        self.cut_distance = sys_.cut_distance(cutoff_)
        self.cutoff = cutoff_ * size
        self.update_count = 0
        self.s.neighbor_list(self.pos, self.rad, self.cut_distance)
        self.last_pos = self.pos.copy()
        self.forces()
        self.pvel = np.zeros(2 * sys_.np)
        self.pangvel = np.zeros(sys_.np)
        self.pangle = np.zeros(sys_.np)

    def forces(self):
        self.out = self.s.rigid_force_energy(self.pos, self.rad)
        self.ppos = self.out["ppos"]

    def check(self):
        d = (self.pos - self.last_pos).reshape(-1, 2)
        box = np.array([self.s.s.lx, self.s.s.ly])
        d -= box * np.round(d / box)
        if np.any(3 * np.sqrt((d * d).sum(1)) > self.cutoff):
            self.s.neighbor_list(self.pos, self.rad, self.cut_distance)
            self.last_pos = self.pos.copy()
            self.update_count += 1

    def nve_step(self, dt):
        plast, alast = self.ppos.copy(), self.pangle.copy()
        self.pvel += 0.5 * dt * self.out["p_force"]
        self.pangvel += 0.5 * dt * self.out["p_torque"]
        pnew = self.ppos + dt * self.pvel
        self.pangle = self.pangle + dt * self.pangvel
        self.L.oc_translate_rotate(self.C.byref(self.s.s), pnew, plast, self.pangle, alast, self.pos)
        self.check()
        self.forces()
        self.pvel += 0.5 * dt * self.out["p_force"]
        self.pangvel += 0.5 * dt * self.out["p_torque"]


def philox_noise(seed: int, stream: int, num_rings: int) -> np.ndarray:
    """(Np, 2) standard normals of one Philox stream, one pair per ring."""
    return np.stack([normal2(seed, stream, q) for q in range(num_rings)])


def nve_adjoint_reference(sys_: System, pk, nsteps: int, dt: float, eps: float = 1e-6):
    """dJ/dx0 of J = U + K after ``nsteps`` velocity-Verlet steps, by the
    adjoint of the Verlet map with Hessian-vector products taken as central
    differences of the oracle's forces: an FP64 reference gradient that uses
    no derivative code.  Returns (J, dJ/dx0, dJ/dv0)."""
    st = OracleState(sys_, pk)
    xs = [st.pos.copy()]
    for _ in range(nsteps):
        st.nve_step(dt)
        xs.append(st.pos.copy())
    J = float(st.out["potential_energy"]) + 0.5 * float(np.dot(st.vel, st.vel))

    def force(x):
        sys_.neighbor_list(x, pk.rad, st.cut_distance)
        return sys_.force_energy(x, pk.rad, pk.a0, pk.l0, pk.theta0)["force"]

    def hvp(x, v):
        return -(force(x + eps * v) - force(x - eps * v)) / (2 * eps)

    xb = -force(xs[-1])
    vb = st.vel.copy()
    for n in reversed(range(nsteps)):
        xb = xb - 0.5 * dt * hvp(xs[n + 1], vb)
        vb = vb + dt * xb
        xb = xb - 0.5 * dt * hvp(xs[n], vb)
    return J, xb, vb


def compress_search_step(R, sigma: float, phi: float, prev_phi: float, dphi: float, current: tuple, saved: tuple,
                         fire_dt: float = 1e-2, tol0: float = 1e-10, max_iter: int = 100000,
                         min_dphi: float = 0.0, cut_distance: float | None = None) -> dict:
    """One search step of the quasi-static compression of compressFIRE.cpp:101-205
    on the reference's own kernels (oracle/_ref ``R`` holding the system), without
    the driver's file output and its Langevin thermalisation:

    * FIRE (vertexFIREparams {0.2, 0.5, 1.1, 0.99, dt, 10 dt, 0.2}, minStep 20,
      dt = fire_dt * sigma, :102-106) from a fresh list and fresh forces
      (:107-109), iterated while max |F| > tol0 / sigma (:115-125);
    * jammed: tol < F < 2 tol (:138) -> state 1;
    * under-jammed: F < tol -> this state becomes the saved one and phi grows
      by dphi, scale sqrt((phi + dphi) / phi) (:152-160);
    * over-jammed: F > 2 tol -> dphi halves, the saved state comes back and
      its phi grows by the halved step (:161-171);
    * scaleVertices about the ring centroids of the last force evaluation,
      then getPhi (:196-197).
    ``current`` = (rad, l0, a0) of the system as it is (the reference library
    does not return them), ``saved`` = (pos, rad, l0, a0) of the last
    under-jammed state.  A halved step below ``min_dphi`` ends the search
    (state 3).  Returns the new state, phi, saved phi, dphi, current and saved
    arrays, the FIRE iterations and the final max |F|."""
    dt = fire_dt * sigma
    R.ref_fire_init(np.array([0.2, 0.5, 1.1, 0.99, dt, 10 * dt, 0.2]), 20, 0)
    if cut_distance is None:
        cut_distance = R.ref_set_displacement_cutoff(0.5, 2 * float(np.mean(current[0])))
    R.ref_calc_neighbor_list(cut_distance)
    R.ref_calc_force_energy()
    R.ref_reset_last_positions()
    tol = tol0 / sigma
    it, fmax = 0, R.ref_max_unbalanced_force()
    while fmax > tol and it != max_iter:
        R.ref_fire_loop(1)
        fmax = R.ref_max_unbalanced_force()
        it += 1
    state, scale = 0, 1.0
    if tol < fmax < 2 * tol:
        state = 1
    elif fmax < tol:
        scale = math.sqrt((phi + dphi) / phi)
        prev_phi = phi
        pos = np.zeros(2 * len(current[0]))
        R.ref_get(0, pos)
        saved = (pos, *current)
    elif fmax > 2 * tol:
        dphi *= 0.5
        scale = math.sqrt((prev_phi + dphi) / prev_phi)
        spos, srad, sl0, sa0 = (np.ascontiguousarray(a, dtype=np.float64) for a in saved)
        R.ref_set_state(spos.ctypes.data, None, srad.ctypes.data, sl0.ctypes.data, None, sa0.ctypes.data)
        R.ref_calc_force_energy()  # ring centroids of the restored state
        current = saved[1:]
    if state == 0 and dphi < min_dphi:
        state = 3
    if state == 0:
        R.ref_scale_vertices(scale)
        phi = R.ref_phi()
        current = (current[0] * scale, current[1] * scale, current[2] * scale * scale)
    return {"state": state, "phi": phi, "prev_phi": prev_phi, "dphi": dphi, "current": current, "saved": saved,
            "iterations": it, "fmax": fmax, "scale": scale}
