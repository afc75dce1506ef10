"""The adjoint of the velocity-Verlet map (oracle.integrators.nve_adjoint_reference,
the recursion that cudaring_b200.diff.nve_gradient runs on the GPU) against
central differences of the oracle's own trajectories, on the CPU."""
import numpy as np
import pytest

import oracle
from cudaring_b200 import synth
from oracle.integrators import OracleState, nve_adjoint_reference


def test_verlet_adjoint_matches_trajectory_differences():
    c = synth.workload_config("bidisperse_harmonic", 4)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.6, seed=3, placement="uniform")
    pk.rad = pk.rad * 1.2
    pk.vel = np.repeat(np.random.default_rng(1).normal(0, 0.05, size=(4, 2)), pk.nv_list, axis=0).reshape(-1)
    S = oracle.System(pk.nv_list, pk.box, "harmonic", "vertexVertex", 1.0, 1.0, 0.01, 1.0)
    nsteps, dt = 40, 0.005
    J, g, _ = nve_adjoint_reference(S, pk, nsteps, dt)

    def run(x0):
        q = synth.Packing(nv_list=pk.nv_list, pos=x0, vel=pk.vel.copy(), rad=pk.rad, l0=pk.l0, theta0=pk.theta0,
                          a0=pk.a0, box=pk.box, centres=pk.centres)
        st = OracleState(S, q)
        for _ in range(nsteps):
            st.nve_step(dt)
        return float(st.out["potential_energy"]) + 0.5 * float(np.dot(st.vel, st.vel))

    h = 1e-6
    for i in np.random.default_rng(2).choice(len(pk.pos), 5, replace=False):
        e = np.zeros_like(pk.pos)
        e[i] = h
        fd = (run(pk.pos + e) - run(pk.pos - e)) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-5, abs=1e-7 * np.abs(g).max())
