"""GPU parity of the rigid-ring path against the reference kernels' golden
fixtures, plus a check of the (corrected) rigid Langevin thermostat."""
import numpy as np
import pytest

from cudaring_b200 import DPM2D, simControl, synth

from conftest import golden_files, load_golden, rel_inf
from test_gpu_parity import dpm_of

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_rigid_force_torque_match_reference(cuda_device):
    g = load_golden(golden_files("rigid_force_wca")[0])
    d, cut = dpm_of(g)
    d.setShapeType(simControl.shapeEnum.rigid)
    d.calcNeighborList(cut)
    d.calcRigidForceEnergy()
    assert rel_inf(d.getVertexForces(), g["out_force"]) < TOL
    assert rel_inf(d.getVertexTorques(), g["out_torque"]) < TOL
    assert rel_inf(d.getParticleForces(), g["out_p_force"]) < TOL
    assert rel_inf(d.getParticleTorques(), g["out_p_torque"]) < 1e-11
    assert rel_inf(d.getParticleEnergies(), g["out_p_energy"]) < TOL
    assert np.allclose(d.getParticlePositions(), g["out_ppos"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("chunks", [1, 8])
def test_rigid_nve_trajectory(cuda_device, chunks):
    g = load_golden(golden_files("traj_rigid_nve_wca")[0])
    d, cut = dpm_of(g)
    d.setShapeType(simControl.shapeEnum.rigid)
    d.calcNeighborList(cut)
    d.resetLastPositions()
    d.initRigidNVE(0.0, readState=True)
    d.setParticleVelocities(g["p_vel"])
    d.setParticleAngularVelocities(g["p_angvel"])
    n = int(g["param_nsteps"])
    for _ in range(chunks):
        d.rigidNVELoop(n // chunks)
    assert d.getUpdateCount() == int(g["out_update_count"])
    assert rel_inf(d.getVertexPositions(), g["out_pos"]) < 1e-11
    assert rel_inf(d.getParticleVelocities(), g["out_p_vel"]) < 1e-8
    assert rel_inf(d.getParticleAngularVelocities(), g["out_p_angvel"]) < 1e-8
    assert rel_inf(d.getParticleAngles(), g["out_p_angle"]) < 1e-9
    assert np.allclose(d.getParticlePositions(), g["out_ppos"], rtol=1e-10, atol=1e-10)


def test_rigid_langevin_temperature(cuda_device):
    # corrected thermostat: ring kinetic energy per translational degree of freedom -> T/2
    c = synth.workload_config("rigid_ellipses", 256)
    pk = synth.make_ellipse_packing(c["n"], c["nv"], c["ratio_range"], 0.2, seed=5)
    d = DPM2D.from_packing(pk, potential="wca", interaction="vertexVertex", ec=1.0, dt=0.002)
    d.setShapeType(simControl.shapeEnum.rigid)
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    d.setSeed(77)
    T = 0.1
    d.initRigidLangevin(T, 1.0, readState=False)
    d.rigidLangevinLoop(3000)
    ke = []
    for _ in range(40):
        d.rigidLangevinLoop(100)
        ke.append(d.getParticleKineticEnergy())
    t_meas = 2.0 * np.mean(ke) / (2 * pk.num_particles)
    assert t_meas == pytest.approx(T, rel=0.08)


def test_rigid_mixed_precision_forces_and_langevin(cuda_device):
    # FP32 vertex pair terms on FP64 offsets: forces and torques within FP32
    # rounding of the FP64 path; a Langevin run stays finite and at temperature
    c = synth.workload_config("rigid_ellipses", 256)
    pk = synth.make_ellipse_packing(c["n"], c["nv"], c["ratio_range"], 0.25, seed=6)
    d = DPM2D.from_packing(pk, potential="wca", interaction="vertexVertex", ec=1.0, dt=0.001)
    d.setShapeType(simControl.shapeEnum.rigid)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * pk.rad.mean()))
    d.setSeed(4)
    d.initRigidLangevin(0.1, 1.0, readState=False)
    d.rigidLangevinLoop(500)  # thermal contacts
    out = {}
    for prec in ("fp64", "mixed"):
        d.setPrecision(prec)
        d.calcRigidForceEnergy()
        out[prec] = (d.getParticleForces(), d.getParticleTorques(), d.getPotentialEnergy())
    assert rel_inf(out["mixed"][0], out["fp64"][0]) < 1e-5
    assert rel_inf(out["mixed"][1], out["fp64"][1]) < 1e-5
    assert out["fp64"][2] > 0.0
    assert out["mixed"][2] == pytest.approx(out["fp64"][2], rel=1e-5)
    d.setSeed(5)
    d.initRigidLangevin(0.1, 1.0, readState=False)
    d.rigidLangevinLoop(2000)
    assert np.all(np.isfinite(d.getVertexPositions()))
    ke = d.getParticleKineticEnergy()
    assert 0.02 < 2.0 * ke / (2 * pk.num_particles) < 0.5
