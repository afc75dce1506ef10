"""Mixed precision against the FP64 path of the same library.

The FP64 path is pinned to the reference (test_gpu_parity.py); the mixed
path (FP32 pair terms on FP64-formed minimum-image offsets, near-contact
smooth units in FP64, FP64 shape terms / integration / compensated
reductions) is checked against it on the same state.  Bars (norm-wise force
error ||F_mixed - F_fp64||_2 / ||F_fp64||_2):

* vertex-vertex LJ on a thermal state of the smooth-LJ workload: <= 2e-6
  (measured 8e-7 at 39,424 vertices);
* smooth vertex-segment LJ on the same state: <= 1e-6.  FP32 unit
  arithmetic alone gives ~7e-6 here: around the LJ minimum one rounding of
  the distance or of r^6 moves a unit force by ~1e-6 of the net force, so
  slots with a unit closer than 1.2 radSum run in FP64;
* pair-only forces (shape constants zero, no FP64 shape force diluting the
  pair error) within 2e-6 for every potential and both interaction kinds on
  a dilute overlapping packing;
* the forces are a function of the positions alone (the order in which
  slots are visited, set by the last evaluation, changes only FP64 rounding);
* the NVE energy error of a mixed run within 2x of the FP64 run from the
  same state (plus a floor of 1e-9 relative for runs where both are at
  rounding level).
"""
import numpy as np
import pytest

from cudaring_b200 import DPM2D, simControl, synth, workloads

pytestmark = pytest.mark.gpu


def l2_rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _forces(d, precision):
    d.setPrecision(precision)
    d.calcForceEnergy()
    return d.getVertexForces(), d.getPotentialEnergy()


@pytest.fixture(scope="module")
def thermal_state(cuda_device):
    # 256 rings of the smooth-LJ deformable workload, relaxed by FIRE at
    # phi 0.85 and thermalised by 300 NVE steps at T = 0.01
    d, info = workloads.prepared_deformable("smooth_lj", 256, seed=77)
    d.initNVE(0.01)
    d.NVELoop(300)
    z = dict(nv_list=d.numVertexInParticleList, pos=d.getVertexPositions(), vel=d.getVertexVelocities(),
             rad=d.getVertexRadii(), l0=d.getRestLengths(), a0=d.getRestAreas(), box=d.getBoxSize(),
             theta0=np.repeat(2 * np.pi / d.numVertexInParticleList, d.numVertexInParticleList).astype(float),
             config=info["config"])
    d.close()
    return z


def _dpm_from(z):
    c = z["config"]
    pk = synth.Packing(nv_list=z["nv_list"], pos=z["pos"], vel=z["vel"], rad=z["rad"], l0=z["l0"],
                       theta0=z["theta0"], a0=z["a0"], box=z["box"], centres=np.zeros((len(z["nv_list"]), 2)))
    d = DPM2D.from_packing(pk, **{k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec",
                                                     "LJcutoff", "dt")})
    cut = d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius())
    d.calcNeighborList(cut)
    d.resetLastPositions()
    return d


@pytest.mark.parametrize("lanes", [1, 2, 4])
@pytest.mark.parametrize("interaction,bar", [("vertexVertex", 2e-6), ("vertexSmooth", 1e-6)])
def test_thermal_state_force_error(thermal_state, lanes, interaction, bar):
    d = _dpm_from(thermal_state)
    d.setInteractionType(getattr(simControl.interactionEnum, interaction))
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.setLanes(lanes)
    f64, e64 = _forces(d, "fp64")
    fmx, emx = _forces(d, "mixed")
    assert d.getPrecision() == "mixed"
    assert l2_rel(fmx, f64) <= bar
    assert emx == pytest.approx(e64, rel=1e-6)


@pytest.mark.parametrize("potential,interaction", [
    ("harmonic", "vertexVertex"), ("harmonic", "vertexSmooth"), ("lennardJones", "vertexVertex"),
    ("lennardJones", "vertexSmooth"), ("wca", "vertexVertex"), ("wca", "vertexSmooth"),
    ("adhesive", "vertexVertex"), ("adhesive", "vertexSmooth")])
def test_pair_only_force_error(cuda_device, potential, interaction):
    c = synth.workload_config("smooth_lj", 64)
    pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], 0.40, seed=3, placement="rsa")
    # radii enlarged so that rings of every potential overlap their neighbours
    pk.rad = pk.rad * 1.8
    d = DPM2D.from_packing(pk, potential=potential, interaction=interaction, ea=0.0, el=0.0, eb=0.0, ec=1.0,
                           LJcutoff=2.5, l1=0.1, l2=0.2)
    cut = d.setDisplacementCutoff(0.5, 2 * pk.rad.mean())
    d.calcNeighborList(cut)
    f64, e64 = _forces(d, "fp64")
    assert np.linalg.norm(f64) > 0.0
    fmx, emx = _forces(d, "mixed")
    assert l2_rel(fmx, f64) <= 2e-6
    assert emx == pytest.approx(e64, rel=2e-6, abs=1e-9 * abs(e64))


def _energy_error(z, precision, steps, chunk):
    d = _dpm_from(z)
    d.setPrecision(precision)
    d.initNVE(0.0, readState=True)
    e0 = d.getEnergy()
    worst = 0.0
    for _ in range(steps // chunk):
        d.NVELoop(chunk)
        worst = max(worst, abs(d.getEnergy() - e0) / abs(e0))
    d.close()
    return worst


def test_nve_energy_error_within_twice_fp64(thermal_state):
    e64 = _energy_error(thermal_state, "fp64", 4000, 500)
    emx = _energy_error(thermal_state, "mixed", 4000, 500)
    assert emx <= 2.0 * e64 + 1e-9


def test_mixed_step_kernel_matches_force_kernel(thermal_state):
    # the fused step kernel stores the forces of the positions it moved to;
    # the force-only kernel re-evaluated there gives the same mixed forces
    d = _dpm_from(thermal_state)
    d.setPrecision("mixed")
    d.calcForceEnergy()
    d.initNVE(0.0, readState=True)
    d.NVELoop(3)
    f_step = d.getVertexForces()
    d.calcForceEnergy()
    assert l2_rel(f_step, d.getVertexForces()) < 1e-12


@pytest.mark.parametrize("lanes", [1, 2])
def test_mixed_forces_do_not_depend_on_visit_order(thermal_state, lanes):
    # first evaluation after a rebuild: the near-slot record is stale; the
    # second one visits the near slots first.  Same positions, same forces.
    d = _dpm_from(thermal_state)
    d.setLanes(lanes)
    d.setPrecision("mixed")
    d.initNVE(0.0, readState=True)
    d.NVELoop(40)
    x = d.getVertexPositions()
    d.calcForceEnergy()
    f_hist = d.getVertexForces()
    d.setVertexPositions(x)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.calcForceEnergy()
    f_fresh = d.getVertexForces()
    d.calcForceEnergy()
    f_again = d.getVertexForces()
    assert l2_rel(f_fresh, f_hist) < 1e-13
    assert l2_rel(f_again, f_fresh) < 1e-13
    d.close()
