"""GPU parity: the CUDA path, called through the C ABI, against the golden
fixtures of the reference kernels and against the pinned CPU oracle.

Bar: forces and energies within 1e-12 of the largest force component (FP64
reordering only), neighbour lists equal as index sets, trajectories within
the bounds stated per test (FP64 rounding amplified by the dynamics).
"""
import numpy as np
import pytest

import oracle
from cudaring_b200 import DPM2D, simControl, synth
from oracle.integrators import OracleState

from conftest import golden_files, load_golden, rel_inf
from test_oracle_golden import packing_of, system_of

pytestmark = pytest.mark.gpu
TOL = 1e-12
POT = {0: "harmonic", 1: "lennardJones", 2: "adhesive", 3: "wca"}
INTER = {0: "vertexVertex", 1: "vertexSmooth"}


def dpm_of(g):
    pk = packing_of(g)
    d = DPM2D.from_packing(pk, potential=POT[int(g["param_potential"])],
                           interaction=INTER[int(g["param_interaction"])], ea=float(g["param_ea"]),
                           el=float(g["param_el"]), eb=float(g["param_eb"]), ec=float(g["param_ec"]),
                           LJcutoff=float(g["param_lj_cutoff"]), l1=float(g.get("param_l1", 0.0)),
                           l2=float(g.get("param_l2", 0.0)))
    if int(g.get("param_monomer", 0)) == 1:
        d.setMonomerType(simControl.monomerEnum.FENE)
        d.setFENEconstants(float(g["param_stiff"]), float(g["param_ext"]))
    if "param_dt" in g:
        d.setTimeStep(float(g["param_dt"]))
    cut = d.setDisplacementCutoff(0.5, 2 * g["rad"].mean())
    assert cut == float(g["param_cut_distance"])
    return d, cut


@pytest.mark.parametrize("path", golden_files("force_"), ids=lambda p: p.split("/")[-1][:-4])
def test_force_energy_and_neighbors_match_reference(cuda_device, path):
    g = load_golden(path)
    d, cut = dpm_of(g)
    d.calcNeighborList(cut)
    assert d.getNeighborListSize() == int(g["out_list_size"])
    assert np.array_equal(d.getMaxNeighborList(), g["out_max_neighbor_list"])
    assert np.array_equal(d.getNeighbors(), g["out_neighbors"])
    d.calcForceEnergy()
    assert rel_inf(d.getVertexForces(), g["out_force"]) < TOL
    assert rel_inf(d.getVertexEnergies(), g["out_energy"]) < TOL
    assert rel_inf(d.getParticleEnergies(), g["out_p_energy"]) < TOL
    assert np.allclose(d.getAreas(), g["out_area"], rtol=1e-12, atol=0)
    assert np.allclose(d.getPerimeters(), g["out_perimeter"], rtol=1e-13, atol=0)
    assert np.allclose(d.getSegmentAngles(), g["out_theta"], rtol=1e-12, atol=1e-13)
    assert np.allclose(d.getSegmentLengths(), g["out_length"], rtol=1e-13, atol=0)
    assert np.allclose(d.getParticlePositions(), g["out_ppos"], rtol=1e-12, atol=1e-12)
    assert d.getPotentialEnergy() == pytest.approx(float(g["out_potential_energy"]), rel=1e-12)
    d.close()


@pytest.mark.parametrize("name", ["smooth_lj", "bidisperse", "monodisperse"])
def test_packing_fraction_matches_reference(cuda_device, name):
    """cr_get_phi / cr_get_preferred_phi against DPM2D::getPhi / getPreferredPhi
    (src/DPM2D.cu:1202-1238) on rings deformed away from their rest areas."""
    g = load_golden(golden_files("phi_cases")[0])
    c = {k[len(name) + 1:]: v for k, v in g.items() if k.startswith(name + "_")}
    d = DPM2D.from_packing(packing_of(c), potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01,
                           ec=1.0)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * c["rad"].mean()))
    d.calcForceEnergy()
    assert d.getPhi() == pytest.approx(float(c["out_phi"]), rel=1e-14)
    assert d.getPreferredPhi() == pytest.approx(float(c["out_preferred_phi"]), rel=1e-14)
    d.close()


def _prepared(g):
    d, cut = dpm_of(g)
    d.calcNeighborList(cut)
    d.resetLastPositions()
    d.calcForceEnergy()
    return d


def test_nve_trajectory_harmonic(cuda_device):
    g = load_golden(golden_files("traj_nve_harmonic_vv")[0])
    d = _prepared(g)
    d.initNVE(0.0, readState=True)
    d.NVELoop(int(g["param_nsteps"]))
    assert d.getUpdateCount() == int(g["out_update_count"])
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-12
    assert rel_inf(d.getVertexVelocities(), g["out_vel"]) < 1e-10
    assert rel_inf(d.getVertexForces(), g["out_force"]) < 1e-10
    assert d.getPotentialEnergy() == pytest.approx(float(g["out_potential_energy"]), rel=1e-9)
    assert d.getKineticEnergy() == pytest.approx(float(g["out_kinetic_energy"]), rel=1e-9)


def test_nve_trajectory_lj_smooth(cuda_device):
    g = load_golden(golden_files("traj_nve_lj_smooth")[0])
    d = _prepared(g)
    d.initNVE(0.0, readState=True)
    d.NVELoop(int(g["param_nsteps"]))
    assert d.getUpdateCount() == int(g["out_update_count"])
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-12
    assert rel_inf(d.getVertexVelocities(), g["out_vel"]) < 1e-9
    assert rel_inf(d.getVertexForces(), g["out_force"]) < 1e-9


def test_nve_one_call_equals_many_calls(cuda_device):
    g = load_golden(golden_files("traj_nve_lj_smooth")[0])
    a = _prepared(g)
    a.initNVE(0.0, readState=True)
    a.NVELoop(150)
    b = _prepared(g)
    b.initNVE(0.0, readState=True)
    for _ in range(10):
        b.NVELoop(15)
    assert np.array_equal(a.getVertexPositions(), b.getVertexPositions())
    assert np.array_equal(a.getVertexVelocities(), b.getVertexVelocities())


def test_fire_trajectory(cuda_device):
    g = load_golden(golden_files("traj_fire_harmonic_vv")[0])
    d = _prepared(g)
    d.initFIRE(g["param_fire"], 20, 0, len(g["rad"]))
    d.vertexFIRELoop(int(g["param_nsteps"]))
    st = d.getFIREState()
    assert st[0] == pytest.approx(g["out_fire_state"][0], rel=1e-12)
    assert st[2] == g["out_fire_state"][2]
    assert st[1] == pytest.approx(g["out_fire_state"][1], rel=1e-9)
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-10
    assert rel_inf(d.getVertexForces(), g["out_force"]) < 1e-7


def test_langevin_trajectory_philox(cuda_device):
    g = load_golden(golden_files("traj_langevin_harmonic_vv")[0])
    d = _prepared(g)
    d.setSeed(int(g["param_seed"]))
    d.initLangevin(float(g["param_T"]), float(g["param_gamma"]), readState=True)
    d.langevinLoop(int(g["param_nsteps"]))
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-12
    assert rel_inf(d.getVertexVelocities(), g["out_vel"]) < 1e-9


def test_nve_rescale_trajectory(cuda_device):
    g = load_golden(golden_files("traj_nverescale_harmonic_vv")[0])
    d = _prepared(g)
    T = float(g["param_T"])
    d.initNVERescale(T)
    assert d.getTemperature() == pytest.approx(T, rel=1e-12)
    d.setVertexVelocities(g["vel"])
    d.NVERescaleLoop(int(g["param_nsteps"]))
    assert d.getUpdateCount() == int(g["out_update_count"])
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-12
    assert rel_inf(d.getVertexVelocities(), g["out_vel"]) < 1e-9


def test_conserve_momentum(cuda_device):
    g = load_golden(golden_files("traj_nve_harmonic_vv")[0])
    d = _prepared(g)
    d.setVertexVelocities(g["vel"] + 0.25)
    d.conserveMomentum()
    v = d.getVertexVelocities().reshape(-1, 2)
    assert np.abs(v.mean(axis=0)).max() < 1e-14
    assert np.allclose(v, (g["vel"] + 0.25).reshape(-1, 2) - (g["vel"] + 0.25).reshape(-1, 2).mean(axis=0),
                       rtol=0, atol=1e-14)


@pytest.mark.parametrize("kind", ["baoab", "brownian", "drivenbrownian", "active_langevin"])
def test_stochastic_integrators_match_reference(cuda_device, kind):
    g = load_golden(golden_files(f"traj_{kind}_harmonic_vv")[0])
    d = _prepared(g)
    d.setSeed(int(g["param_seed"]))
    noise = {"baoab": simControl.noiseEnum.baoab, "brownian": simControl.noiseEnum.brownian,
             "drivenbrownian": simControl.noiseEnum.drivenBrownian,
             "active_langevin": simControl.noiseEnum.langevin}[kind]
    d.setNoiseType(noise)
    if kind == "active_langevin":
        d.setParticleType(simControl.particleEnum.active)
        d.setSelfPropulsionParams(float(g["param_driving"]), float(g["param_taup"]))
    d.initLangevin(float(g["param_T"]), float(g["param_gamma"]), readState=True)
    d.langevinLoop(int(g["param_nsteps"]))
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-12
    assert rel_inf(d.getVertexVelocities(), g["out_vel"]) < 1e-9
    if kind == "active_langevin":
        assert np.allclose(d.getParticleAngles(), g["out_p_angle"], rtol=0, atol=1e-12)


def _lj_smooth_packing(n, phi=0.40, seed=5, placement="rsa"):
    c = synth.workload_config("smooth_lj", n)
    return c, synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=seed, placement=placement)


@pytest.mark.parametrize("lanes", [1, 2, 4])
def test_smooth_lj_256_rings_vs_oracle(cuda_device, lanes):
    c, pk = _lj_smooth_packing(256)
    c = dict(c, ea=1.0, el=1.0, eb=0.01)
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    d.setLanes(lanes)
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    d.calcForceEnergy()
    S = oracle.System(pk.nv_list, pk.box, c["potential"], c["interaction"], c["ea"], c["el"], c["eb"], c["ec"],
                      lj_cutoff=c["LJcutoff"])
    S.neighbor_list(pk.pos, pk.rad, S.cut_distance(0.5))
    out = S.force_energy(pk.pos, pk.rad, pk.a0, pk.l0, pk.theta0)
    assert rel_inf(d.getVertexForces(), out["force"]) < TOL
    assert d.getPotentialEnergy() == pytest.approx(out["potential_energy"], rel=1e-12)


def test_stiff_area_constant_within_reference_conditioning(cuda_device):
    # With the reference driver's ea = 1e5 the reference's shoelace area, summed
    # on absolute box coordinates, carries a rounding error of order
    # nv * eps * L^2; its area force error is ea * dA / a0^2 * |x_next - x_prev| / 2.
    # This build sums ring-relative offsets (smaller error), so the two may
    # differ by the reference's own bound, which this test allows.
    c, pk = _lj_smooth_packing(256)
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    d.calcForceEnergy()
    S = oracle.System(pk.nv_list, pk.box, c["potential"], c["interaction"], c["ea"], c["el"], c["eb"], c["ec"],
                      lj_cutoff=c["LJcutoff"])
    S.neighbor_list(pk.pos, pk.rad, S.cut_distance(0.5))
    out = S.force_energy(pk.pos, pk.rad, pk.a0, pk.l0, pk.theta0)
    eps = np.finfo(float).eps
    dA = 4 * pk.nv_list.max() * eps * float(pk.box.max()) ** 2
    bound = c["ea"] * dA / pk.a0.min() ** 2 * 2 * pk.l0.max()
    err = np.abs(d.getVertexForces() - out["force"]).max()
    assert err < max(bound, TOL * np.abs(out["force"]).max())


def test_full_size_config_neighbor_sets_and_forces(cuda_device):
    # 1024 rings, nv 32/45 (39,424 vertices), smooth LJ rc 2.5, phi 0.85
    c = synth.workload_config("smooth_lj")
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], c["phi"], seed=20261204)
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    S = oracle.System(pk.nv_list, pk.box, c["potential"], c["interaction"], c["ea"], c["el"], c["eb"], c["ec"],
                      lj_cutoff=c["LJcutoff"])
    nbr, cnt, ls = S.neighbor_list(pk.pos, pk.rad, S.cut_distance(0.5))
    assert d.getNeighborListSize() == ls
    assert np.array_equal(d.getMaxNeighborList(), cnt)
    assert np.array_equal(d.getNeighbors(), nbr)
    d.calcForceEnergy()
    out = S.force_energy(pk.pos, pk.rad, pk.a0, pk.l0, pk.theta0)
    assert rel_inf(d.getVertexForces(), out["force"]) < TOL


def test_nve_energy_error_is_second_order(cuda_device):
    # velocity Verlet: the energy error over a fixed time scales as dt^2
    g = load_golden(golden_files("traj_nve_harmonic_vv")[0])
    errs = []
    for dt, n in ((0.004, 250), (0.002, 500)):
        d = _prepared(g)
        d.setTimeStep(dt)
        d.initNVE(0.0, readState=True)
        e0 = d.getEnergy()
        es = []
        for _ in range(10):
            d.NVELoop(n // 10)
            es.append(d.getEnergy())
        errs.append(max(abs(e - e0) for e in es) / abs(e0))
    assert errs[0] < 5e-3
    assert 2.5 < errs[0] / errs[1] < 6.0


def test_force_is_minus_gradient(cuda_device):
    # central differences of the total energy on a small smooth-LJ system
    c, pk = _lj_smooth_packing(8, phi=0.3, seed=11)
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    d.calcForceEnergy()
    f = d.getVertexForces()
    rng = np.random.default_rng(0)
    h = 1e-6
    for idx in rng.choice(len(f), 12, replace=False):
        e = []
        for s in (+1, -1):
            x = pk.pos.copy()
            x[idx] += s * h
            d.setVertexPositions(x)
            d.calcForceEnergy()
            e.append(d.getPotentialEnergy())
        fd = -(e[0] - e[1]) / (2 * h)
        assert fd == pytest.approx(f[idx], rel=1e-5, abs=1e-6 * max(1.0, np.abs(f).max()))


def test_getters_write_into_given_arrays(cuda_device):
    # out= downloads into the caller's array (a pinned buffer needs no staging)
    c = synth.workload_config("smooth_lj", 8)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=5, placement="rsa")
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "LJcutoff")})
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    for get in (d.getVertexPositions, d.getVertexVelocities, d.getVertexForces):
        ref = get()
        buf = np.full_like(ref, np.nan)
        assert get(out=buf) is buf and np.array_equal(buf, ref)
        with pytest.raises(ValueError):
            get(out=np.empty(ref.size - 1))
    d.close()
