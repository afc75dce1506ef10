"""The CPU oracle (oracle/oracle.c + oracle/integrators.py) against the golden
fixtures produced by the reference's own kernels (tests/golden/make_golden.py).

These tests pin the oracle: once it agrees with the reference here, the GPU
tests may use it as the checker on inputs that have no golden file.
"""
import numpy as np
import pytest

import oracle
from oracle.integrators import OracleFIRE, OracleState, philox_noise
from cudaring_b200.synth import Packing

from conftest import golden_files, load_golden, rel_inf

TOL = 1e-12  # relative to the largest force component


def packing_of(g):
    return Packing(nv_list=g["nv_list"], pos=g["pos"].copy(), vel=g["vel"].copy(), rad=g["rad"], l0=g["l0"],
                   theta0=g["theta0"], a0=g["a0"], box=g["box"], centres=np.zeros((len(g["nv_list"]), 2)))


def system_of(g):
    pot = {0: "harmonic", 1: "lennardJones", 2: "adhesive", 3: "wca"}[int(g["param_potential"])]
    inter = {0: "vertexVertex", 1: "vertexSmooth"}[int(g["param_interaction"])]
    return oracle.System(g["nv_list"], g["box"], pot, inter, float(g["param_ea"]), float(g["param_el"]),
                         float(g["param_eb"]), float(g["param_ec"]), l1=float(g.get("param_l1", 0.0)),
                         l2=float(g.get("param_l2", 0.0)), lj_cutoff=float(g["param_lj_cutoff"]),
                         monomer=int(g.get("param_monomer", 0)), stiff=float(g.get("param_stiff", 0.0)),
                         ext=float(g.get("param_ext", 0.0)))


@pytest.mark.parametrize("path", golden_files("force_"), ids=lambda p: p.split("/")[-1][:-4])
def test_force_energy_matches_reference(path):
    g = load_golden(path)
    S = system_of(g)
    nbr, cnt, ls = S.neighbor_list(g["pos"], g["rad"], float(g["param_cut_distance"]))
    assert ls == int(g["out_list_size"])
    assert np.array_equal(cnt, g["out_max_neighbor_list"])
    assert np.array_equal(nbr[: len(g["out_neighbors"])], g["out_neighbors"])
    out = S.force_energy(g["pos"], g["rad"], g["a0"], g["l0"], g["theta0"])
    assert rel_inf(out["force"], g["out_force"]) < TOL
    assert rel_inf(out["energy"], g["out_energy"]) < TOL
    assert rel_inf(out["p_energy"], g["out_p_energy"]) < TOL
    assert np.allclose(out["area"], g["out_area"], rtol=1e-13, atol=0)
    assert np.allclose(out["perimeter"], g["out_perimeter"], rtol=1e-13, atol=0)
    assert np.allclose(out["theta"], g["out_theta"], rtol=1e-12, atol=1e-14)
    assert np.allclose(out["length"], g["out_length"], rtol=1e-13, atol=0)
    assert np.allclose(out["ppos"], g["out_ppos"], rtol=1e-13, atol=1e-13)
    assert out["potential_energy"] == pytest.approx(float(g["out_potential_energy"]), rel=1e-12)


def _state(g):
    pk = packing_of(g)
    st = OracleState(system_of(g), pk)
    assert st.cut_distance == pytest.approx(float(g["param_cut_distance"]), rel=0, abs=0)
    return st


def test_nve_trajectory_harmonic():
    g = load_golden(golden_files("traj_nve_harmonic_vv")[0])
    st = _state(g)
    for _ in range(int(g["param_nsteps"])):
        st.nve_step(float(g["param_dt"]))
    assert st.update_count == int(g["out_update_count"])
    assert rel_inf(st.pos, g["out_pos"]) < 1e-12
    assert rel_inf(st.vel, g["out_vel"]) < 1e-10
    assert rel_inf(st.force, g["out_force"]) < 1e-10


def test_nve_trajectory_lj_smooth():
    g = load_golden(golden_files("traj_nve_lj_smooth")[0])
    st = _state(g)
    for _ in range(int(g["param_nsteps"])):
        st.nve_step(float(g["param_dt"]))
    assert st.update_count == int(g["out_update_count"])
    assert rel_inf(st.pos, g["out_pos"]) < 1e-12
    assert rel_inf(st.vel, g["out_vel"]) < 1e-9
    assert rel_inf(st.force, g["out_force"]) < 1e-9


def test_nve_rescale_trajectory():
    g = load_golden(golden_files("traj_nverescale_harmonic_vv")[0])
    st = _state(g)
    for _ in range(int(g["param_nsteps"])):
        st.nve_rescale_step(float(g["param_dt"]), float(g["param_T"]))
    assert st.update_count == int(g["out_update_count"])
    assert rel_inf(st.pos, g["out_pos"]) < 1e-12
    assert rel_inf(st.vel, g["out_vel"]) < 1e-10


def test_fire_trajectory():
    g = load_golden(golden_files("traj_fire_harmonic_vv")[0])
    st = _state(g)
    fire = OracleFIRE(list(g["param_fire"]), 20, 0)
    for _ in range(int(g["param_nsteps"])):
        fire.iterate(st)
    assert fire.dt == pytest.approx(g["out_fire_state"][0], rel=1e-12)
    assert fire.a == pytest.approx(g["out_fire_state"][1], rel=1e-9)
    assert fire.num_step == int(g["out_fire_state"][2])
    assert rel_inf(st.pos, g["out_pos"]) < 1e-10
    assert rel_inf(st.force, g["out_force"]) < 1e-7


def test_langevin_trajectory_with_philox_noise():
    g = load_golden(golden_files("traj_langevin_harmonic_vv")[0])
    st = _state(g)
    dt, T, gamma, seed = (float(g["param_dt"]), float(g["param_T"]), float(g["param_gamma"]), int(g["param_seed"]))
    amp = np.sqrt(2.0 * T * gamma / dt)
    for s in range(int(g["param_nsteps"])):
        st.langevin_step(dt, gamma, amp, philox_noise(seed, 2 * s, len(g["nv_list"])))
    assert rel_inf(st.pos, g["out_pos"]) < 1e-12
    assert rel_inf(st.vel, g["out_vel"]) < 1e-10


def test_rigid_force_matches_reference():
    g = load_golden(golden_files("rigid_force_wca")[0])
    S = system_of(g)
    S.neighbor_list(g["pos"], g["rad"], float(g["param_cut_distance"]))
    out = S.rigid_force_energy(g["pos"], g["rad"])
    assert rel_inf(out["force"], g["out_force"]) < TOL
    assert rel_inf(out["p_force"], g["out_p_force"]) < TOL
    assert rel_inf(out["torque"], g["out_torque"]) < TOL
    assert rel_inf(out["p_torque"], g["out_p_torque"]) < 1e-11
    assert np.allclose(out["moi"], g["out_moi"], rtol=1e-12, atol=0)
    assert np.allclose(out["ppos"], g["out_ppos"], rtol=1e-13, atol=1e-13)
    assert rel_inf(out["p_energy"], g["out_p_energy"]) < TOL


def test_rigid_nve_trajectory():
    from oracle.integrators import OracleRigid

    g = load_golden(golden_files("traj_rigid_nve_wca")[0])
    rig = OracleRigid(system_of(g), packing_of(g))
    rig.pvel = g["p_vel"].copy()
    rig.pangvel = g["p_angvel"].copy()
    for _ in range(int(g["param_nsteps"])):
        rig.nve_step(float(g["param_dt"]))
    assert rig.update_count == int(g["out_update_count"])
    assert rel_inf(rig.pos, g["out_pos"]) < 1e-11
    assert rel_inf(rig.pvel, g["out_p_vel"]) < 1e-8
    assert rel_inf(rig.pangvel, g["out_p_angvel"]) < 1e-8
    assert rel_inf(rig.pangle, g["out_p_angle"]) < 1e-9


@pytest.mark.parametrize("kind", ["baoab", "brownian", "drivenbrownian", "active_langevin"])
def test_stochastic_integrators_with_philox_noise(kind):
    g = load_golden(golden_files(f"traj_{kind}_harmonic_vv")[0])
    st = _state(g)
    dt, T, gamma, seed = (float(g["param_dt"]), float(g["param_T"]), float(g["param_gamma"]), int(g["param_seed"]))
    npart = len(g["nv_list"])
    for s in range(int(g["param_nsteps"])):
        xi = philox_noise(seed, 2 * s, npart)
        if kind == "baoab":
            st.baoab_step(dt, np.exp(-gamma * dt), np.sqrt(1 - np.exp(-2 * gamma * dt)) * np.sqrt(T), xi)
        elif kind == "brownian":
            st.brownian_step(dt, gamma, np.sqrt(2 * T * gamma / dt), xi)
        elif kind == "drivenbrownian":
            st.brownian_step(dt, gamma, 0.0, None)
        else:
            sp = np.sqrt(2 * dt / float(g["param_taup"]))
            st.langevin_step(dt, gamma, np.sqrt(2 * T * gamma / dt), xi, float(g["param_driving"]),
                             sp * philox_noise(seed, 2 * s + 1, npart)[:, 0])
    assert rel_inf(st.pos, g["out_pos"]) < 1e-12
    assert rel_inf(st.vel, g["out_vel"]) < 1e-9
    if kind == "active_langevin":
        assert np.allclose(st.pangle, g["out_p_angle"], rtol=0, atol=1e-12)


def test_philox_known_answer():
    # Known-answer vectors of Philox4x32-10 published with Random123 (kat_vectors):
    # counter 0, key 0 and counter/key of all ones.
    import ctypes as C
    L = oracle.lib()
    L.oc_philox4x32.argtypes = [C.POINTER(C.c_uint32 * 4), C.POINTER(C.c_uint32 * 2), C.POINTER(C.c_uint32 * 4)]
    out = (C.c_uint32 * 4)()
    L.oc_philox4x32(C.byref((C.c_uint32 * 4)(0, 0, 0, 0)), C.byref((C.c_uint32 * 2)(0, 0)), C.byref(out))
    assert list(out) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    ff = 0xFFFFFFFF
    L.oc_philox4x32(C.byref((C.c_uint32 * 4)(ff, ff, ff, ff)), C.byref((C.c_uint32 * 2)(ff, ff)), C.byref(out))
    assert list(out) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def test_philox_normals_are_standard():
    z = np.stack([oracle.normal2(99, 3, i) for i in range(4000)]).reshape(-1)
    assert abs(z.mean()) < 0.05
    assert abs(z.std() - 1.0) < 0.05


def _phi_case(g, name):
    return {k[len(name) + 1:]: v for k, v in g.items() if k.startswith(name + "_")}


@pytest.mark.parametrize("name", ["smooth_lj", "bidisperse", "monodisperse"])
def test_packing_fraction_matches_reference(name):
    c = _phi_case(load_golden(golden_files("phi_cases")[0]), name)
    S = oracle.System(c["nv_list"], c["box"], "harmonic", "vertexVertex", 1.0, 1.0, 0.01, 1.0)
    area = S.force_energy(c["pos"], c["rad"], c["a0"], c["l0"], c["theta0"])["area"]
    assert oracle.packing_fraction(c["nv_list"], c["rad"], area, c["box"]) == pytest.approx(float(c["out_phi"]),
                                                                                           rel=1e-14)
    assert oracle.packing_fraction(c["nv_list"], c["rad"], c["a0"], c["box"]) == pytest.approx(
        float(c["out_preferred_phi"]), rel=1e-14)
