"""The multi-step kernel (the middle steps of NVE, Langevin and BAOAB runs in
launches of up to 64 steps with grid barriers between steps) against one
launch per step: positions, velocities, the rebuild count and the energies
must be identical, with rebuilds inside the run, for the integrators and
both lane counts it serves (FP64: identical; mixed precision: to rounding)."""
import numpy as np
import pytest

from cudaring_b200 import DPM2D, simControl, synth

pytestmark = pytest.mark.gpu


def _packing(n=64, phi=0.80, seed=23):
    c = synth.workload_config("smooth_lj", n)
    return c, synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=seed, placement="uniform")


def _run(pk, c, multistep, kind, precision, lanes, nsteps, T):
    kw = dict(potential="harmonic", interaction="vertexSmooth", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    d = DPM2D.from_packing(pk, **kw, dt=0.005)
    d.setPrecision(precision)
    d.setLanes(lanes)
    d.setMultistep(multistep)
    d.setSeed(11)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2 * pk.rad.mean()))
    if kind == "nve":
        d.initNVE(T, readState=False)
        d.NVELoop(nsteps)
    elif kind == "langevin":
        d.initLangevin(T, 1.0, readState=False)
        d.langevinLoop(nsteps)
    else:
        d.setNoiseType(simControl.noiseEnum.baoab)
        d.initLangevin(T, 1.0, readState=False)
        d.langevinLoop(nsteps)
    out = (d.getVertexPositions(), d.getVertexVelocities(), d.getUpdateCount(), d.getPotentialEnergy())
    d.close()
    return out


@pytest.mark.parametrize("kind", ["nve", "langevin", "baoab"])
@pytest.mark.parametrize("lanes", [2, 1])
def test_multistep_matches_one_launch_per_step(cuda_device, kind, lanes):
    c, pk = _packing()
    a = _run(pk, c, True, kind, "fp64", lanes, 400, 0.05)
    b = _run(pk, c, False, kind, "fp64", lanes, 400, 0.05)
    assert a[2] == b[2] and a[2] >= 3  # rebuilds happened inside the run
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert a[3] == b[3]


@pytest.mark.parametrize("kind", ["nve", "langevin"])
def test_multistep_mixed_agrees_to_rounding(cuda_device, kind):
    # the two kernels are separate compilations of the same FP32 unit code,
    # whose products may be fused differently: over a few steps the states
    # agree to FP32 rounding of the pair terms
    c, pk = _packing()
    a = _run(pk, c, True, kind, "mixed", 2, 10, 0.05)
    b = _run(pk, c, False, kind, "mixed", 2, 10, 0.05)
    assert a[2] == b[2]
    assert np.max(np.abs(a[0] - b[0])) < 1e-9
    assert np.max(np.abs(a[1] - b[1])) < 1e-7
    assert a[3] == pytest.approx(b[3], rel=1e-9)


@pytest.mark.parametrize("nsteps", [2, 3, 64, 65, 130])
def test_multistep_step_counts(cuda_device, nsteps):
    # sequences whose middle part ends inside, at and past a launch's budget
    c, pk = _packing(n=32, seed=5)
    a = _run(pk, c, True, "nve", "fp64", 2, nsteps, 1e-3)
    b = _run(pk, c, False, "nve", "fp64", 2, nsteps, 1e-3)
    assert a[2] == b[2]
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
