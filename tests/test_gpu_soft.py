"""Soft-disk pre-packing on the GPU against the reference's fixtures
(tests/golden/soft_*.npz) and the pinned restatement (oracle/particles.py):
setRandomParticles, the particle list (brute-force and cell-list builds),
particle forces, particle FIRE, the driver's minimisation loop and
initVerticesOnParticles."""
import numpy as np
import pytest

from oracle import particles as P
from cudaring_b200 import DPM2D, synth
from cudaring_b200.synth import Packing

from conftest import golden_files, load_golden, rel_inf

pytestmark = pytest.mark.gpu

POTS = {0: "harmonic", 1: "lennardJones", 2: "adhesive", 3: "wca"}


def _dpm(g):
    n = len(g["in_nv_list"])
    pk = Packing(nv_list=g["in_nv_list"], pos=g["in_pos"], vel=np.zeros_like(g["in_pos"]), rad=g["in_rad"],
                 l0=g["in_l0"], theta0=g["in_theta0"], a0=g["in_a0"], box=np.array([1.0, 1.0]),
                 centres=np.zeros((n, 2)))
    return DPM2D.from_packing(pk, potential=POTS[int(g["param_potential"])], LJcutoff=float(g["param_lj_cutoff"]))


def _random(d, g):
    d.setRandomParticles(float(g["param_phi0"]), float(g["param_extra_rad"]), int(g["param_seed"]))


@pytest.mark.parametrize("path", golden_files("soft_"), ids=lambda p: p.split("/")[-1][:-4])
def test_random_particles_list_and_forces_match_reference(cuda_device, path):
    g = load_golden(path)
    with _dpm(g) as d:
        _random(d, g)
        assert np.array_equal(d.getBoxSize(), g["out_box"])
        assert np.array_equal(d.getRestAreas(), g["out_a0"])
        assert np.array_equal(d.getRestLengths(), g["out_l0"])
        assert np.array_equal(d.getVertexRadii(), g["out_rad"])
        assert np.array_equal(d.getParticlePositions(), g["out_ppos"])
        assert np.array_equal(d.getParticleRadii(), g["out_prad"])
        d.calcParticleNeighborList(float(g["param_cut"]))
        assert d.getParticleNeighborListSize() == int(g["out_plist_size"])
        assert np.array_equal(d.getParticleMaxNeighborList(), g["out_pmax"])
        assert np.array_equal(d.getParticleNeighbors(), g["out_pneighbors"])
        d.calcParticleForceEnergy()
        assert rel_inf(d.getParticleForces(), g["out_pforce"]) < 1e-12
        assert rel_inf(d.getParticleEnergies(), g["out_penergy"]) < 1e-12
        assert d.getParticlePotentialEnergy() == pytest.approx(float(g["out_penergy"].sum()), rel=1e-12)
        assert d.getParticleMaxUnbalancedForce() == pytest.approx(float(np.abs(g["out_pforce"]).max()), rel=1e-12)


def test_particle_fire_loop_matches_reference(cuda_device):
    g = load_golden(golden_files("soft_harmonic")[0])
    with _dpm(g) as d:
        _random(d, g)
        d.calcParticleNeighborList(float(g["param_cut"]))
        d.calcParticleForceEnergy()
        d.initParticleFIRE(g["param_fire"], int(g["param_min_step"]), 0)
        d.particleFIRELoop(4)
        d.particleFIRELoop(6)  # two calls: the bend pending between calls is applied once
        assert rel_inf(d.getParticlePositions(), g["out_fire10_ppos"]) < 1e-12
        assert rel_inf(d.getParticleVelocities(), g["out_fire10_pvel"]) < 1e-9
        dt, a, num_step = d.getParticleFIREState()
        assert dt == pytest.approx(float(g["out_fire10_state"][0]), rel=1e-15)
        assert a == pytest.approx(float(g["out_fire10_state"][1]), rel=1e-15)
        assert num_step == int(g["out_fire10_state"][2])


def test_particle_fire_minimization_matches_reference(cuda_device):
    g = load_golden(golden_files("soft_harmonic")[0])
    cut, tol = float(g["param_cut"]), float(g["param_tol"])
    with _dpm(g) as d:
        _random(d, g)
        d.calcParticleNeighborList(cut)
        d.calcParticleForceEnergy()
        d.resetParticleLastPositions()
        d.initParticleFIRE(g["param_fire"], int(g["param_min_step"]), 0)
        it = d.particleFIREMinimize(cut, tol, 1000000)
        assert d.getParticleMaxUnbalancedForce() <= tol
        ref_it = int(g["out_min_iters"])
        assert abs(it - ref_it) <= max(5, int(0.05 * ref_it))
        # the same minimum: FIRE sums run in another order than the
        # reference's, so the paths agree to rounding, amplified over the run
        assert np.abs(d.getParticlePositions() - g["out_min_ppos"]).max() < 1e-6
        assert d.getParticlePotentialEnergy() == pytest.approx(float(g["out_min_pe"]), rel=1e-6, abs=1e-15)


def test_vertices_on_particles_match_reference(cuda_device):
    g = load_golden(golden_files("soft_harmonic")[0])
    with _dpm(g) as d:
        _random(d, g)
        d.setParticlePositions(g["out_min_ppos"])
        d.initVerticesOnParticles(g["in_draws"])
        assert np.abs(d.getVertexPositions() - g["out_vpos"]).max() < 1e-13
        assert not np.any(d.getVertexVelocities())
        d2 = d  # the vertex model runs from the placed vertices
        cut = d2.setDisplacementCutoff(0.5, 2 * d2.getMeanVertexRadius())
        d2.calcNeighborList(cut)
        d2.calcForceEnergy()
        assert np.all(np.isfinite(d2.getVertexForces()))


@pytest.mark.parametrize("phi0", [0.5, 0.85])
def test_cell_list_build_and_forces_match_oracle(cuda_device, phi0):
    # 1024 rings: the particle cells are many per side, so the cell-list path
    # (not the brute-force one of the 32-ring fixtures) builds the list
    c = synth.workload_config("smooth_lj")
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.85, seed=11, placement="uniform")
    pk.box = np.array([1.0, 1.0])
    with DPM2D.from_packing(pk) as d:
        d.setRandomParticles(phi0, 1.1, 99)
        ppos, prad = d.getParticlePositions(), d.getParticleRadii()
        d.calcParticleNeighborList(1.0)
        rows, cnt, ls = P.particle_neighbor_list(ppos, prad, [1.0, 1.0], 1.0)
        assert d.getParticleNeighborListSize() == ls
        assert np.array_equal(d.getParticleMaxNeighborList(), cnt)
        assert np.array_equal(d.getParticleNeighbors(), rows)
        d.calcParticleForceEnergy()
        f, e = P.particle_force_energy(ppos, prad, [1.0, 1.0], rows, cnt, ls)
        assert rel_inf(d.getParticleForces(), f) < 1e-12
        assert rel_inf(d.getParticleEnergies(), e) < 1e-12


def test_soft_prepack_driver_end_to_end(cuda_device):
    # compressFIRE.cpp:53-86 in one call on 1024 rings, then the vertex model
    c = synth.workload_config("smooth_lj")
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.85, seed=12, placement="uniform")
    pk.box = np.array([1.0, 1.0])
    with DPM2D.from_packing(pk) as d:
        it = d.softPrepack(0.6, extraRad=1.1, seed=5)
        assert it > 0
        tol = 1e-10 / d.getMeanParticleSigma()
        assert d.getParticleMaxUnbalancedForce() <= tol
        # every ring sits on its disk: centroid within the jitter of the centre
        d.calcParticlePositions()
        cen = d.getParticlePositions()
        assert np.all(np.isfinite(cen))
        cut = d.setDisplacementCutoff(0.5, 2 * d.getMeanVertexRadius())
        d.calcNeighborList(cut)
        d.calcForceEnergy()
        assert np.all(np.isfinite(d.getVertexForces()))
