"""Batches of independent systems (cr_batch_*) against the single-system
path of the same library, system by system.

Forces: every system of a batch evaluates the same tiles with the same
arithmetic as its own context, so forces and energies agree to FP64 rounding
(1e-12 of the largest component).  FIRE: the per-system iteration matches
the single-system one; the runs start from sums reduced in a different
order, so trajectories agree to the minimiser's tolerance.  Compression:
the batched protocol reaches the same packing fractions as the per-system
loop (cudaring_b200.compress.compress_system).  Directly against the CPU
checkers: every system's forces against the oracle, and one compression
search step of every system against the same step of compressFIRE.cpp run on
the reference's own kernels (oracle/_ref).
"""
import math

import numpy as np
import pytest

import oracle
from cudaring_b200 import DPM2D, synth
from cudaring_b200.batch import Batch
from cudaring_b200.compress import batch_packings, compress_system
from oracle.integrators import compress_search_step

from conftest import rel_inf

pytestmark = pytest.mark.gpu


def _systems(workload, sizes, phi, seed, placement="rsa", rad_scale=1.0):
    out = []
    for k, n in enumerate(sizes):
        c = synth.workload_config(workload, n)
        pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], phi, seed=seed + k, placement=placement)
        pk.rad = pk.rad * rad_scale
        out.append(pk)
    return out


def _single(pk, **kw):
    d = DPM2D.from_packing(pk, **kw)
    d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
    d.resetLastPositions()
    d.calcForceEnergy()
    return d


@pytest.mark.parametrize("potential,interaction,workload,rad_scale", [
    ("harmonic", "vertexVertex", "bidisperse_harmonic", 1.5), ("lennardJones", "vertexSmooth", "smooth_lj", 1.0),
    ("wca", "vertexSmooth", "smooth_lj", 1.3)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_forces_match_single(cuda_device, potential, interaction, workload, rad_scale, precision):
    pks = _systems(workload, [8, 24, 40, 16, 64], 0.40, seed=101, rad_scale=rad_scale)
    kw = dict(potential=potential, interaction=interaction, ea=1.0, el=1.0, eb=0.01, ec=1.0, LJcutoff=2.5)
    b = Batch.from_packings(pks, **kw)
    b.setPrecision(precision)
    b.setLanes(2)  # the single-system default here; FP32 sums follow the lane split
    b.setDisplacementCutoff(0.5)
    b.calcNeighborLists()
    b.calcForceEnergy()
    f = b.getVertexForces()
    u = b.getPotentialEnergies()
    assert np.all(np.isfinite(f))
    for s, pk in enumerate(pks):
        d = _single(pk, **kw)
        d.setLanes(2)
        d.setPrecision(precision)
        d.calcForceEnergy()
        fs = d.getVertexForces()
        assert np.abs(fs).max() > 0
        assert rel_inf(f[b.system_slice(s)], fs) < 1e-12
        if precision == "fp64":
            assert u[s] == pytest.approx(d.getPotentialEnergy(), rel=1e-12)
        else:
            # FP32 unit energies: the batch kernel is compiled separately and
            # may contract products into FMAs differently, so the two agree
            # to FP32 rounding of the energy magnitude
            scale = np.abs(d.getParticleEnergies()).sum() + np.abs(d.getVertexEnergies()).sum()
            assert abs(u[s] - d.getPotentialEnergy()) <= 1e-7 * scale
        d.close()
    phi = b.getPhis()
    for s, pk in enumerate(pks):
        d = _single(pk, **kw)
        assert phi[s] == pytest.approx(d.getPhi(), rel=1e-13)
        d.close()


def test_batch_fire_matches_single(cuda_device):
    pks = _systems("bidisperse_harmonic", [16, 32, 20], 0.70, seed=7, placement="uniform")
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    sig = b.getMeanParticleSizes()
    dt = 1e-2 * sig
    b.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-2, 1e-1, 0.2], 20, dt=dt)
    tol = 1e-10 / sig
    its, fmax = b.fireMinimize(tol, 20000)
    pos = b.getVertexPositions()
    for s, pk in enumerate(pks):
        assert fmax[s] <= tol[s]
        d = _single(pk, **kw)
        d.initFIRE([0.2, 0.5, 1.1, 0.99, dt[s], 10 * dt[s], 0.2], 20, 0, d.numVertices)
        it1, f1 = d.minimizeFIRE(tol[s], 20000)
        assert f1 <= tol[s]
        assert abs(its[s] - it1) <= max(20, 0.05 * it1)
        assert rel_inf(pos[b.system_slice(s)], d.getVertexPositions()) < 1e-6
        d.close()


@pytest.mark.parametrize("workload,potential,interaction,lanes", [
    ("bidisperse_harmonic", "harmonic", "vertexVertex", 1), ("smooth_lj", "lennardJones", "vertexSmooth", 2)])
def test_batch_fire_persistent_matches_one_launch_per_op(cuda_device, workload, potential, interaction, lanes):
    # the persistent kernel (up to 64 iterations per launch, grid barriers,
    # rebuilds between launches) against one launch per op: the same ops in
    # the same order, so the same iterates bit for bit
    pks = _systems(workload, [16, 32, 20], 0.40 if workload == "smooth_lj" else 0.70, seed=7,
                   placement="rsa" if workload == "smooth_lj" else "uniform")
    kw = dict(potential=potential, interaction=interaction, ea=1.0, el=1.0, eb=0.01, ec=1.0, LJcutoff=2.5)
    out = []
    for persistent in (False, True):
        b = Batch.from_packings(pks, **kw)
        b.setLanes(lanes)
        b.setPersistent(persistent)
        b.setDisplacementCutoff(0.5)
        sig = b.getMeanParticleSizes()
        b.initFIRE([0.2, 0.5, 1.1, 0.99, 1e-3, 1e-2, 0.2], 20, dt=1e-3 * sig)
        n0 = b.getLaunchCount()
        its, fmax = b.fireMinimize(1e-10 / sig, 3000)
        out.append((its, fmax, b.getVertexPositions(), b.getVertexVelocities(), b.getLaunchCount() - n0))
    (i2, f2, x2, v2, l2), (i1, f1, x1, v1, l1) = out
    assert np.array_equal(i1, i2) and np.array_equal(f1, f2)
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert i1.max() > 200
    assert l1 * 10 < l2  # the persistent kernel ran (a few launches per 64 iterations)


def test_batch_compress_persistent_matches_one_launch_per_op(cuda_device):
    pks = batch_packings(4, seed=11, rings=(16, 40))
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    prm = dict(dphi=2e-2, min_dphi=2e-3, fire_dt=1e-2, tol0=1e-6, max_fire_iters=400, max_steps=6)
    out = []
    for persistent in (True, False):
        b = Batch.from_packings(pks, **kw)
        b.setPersistent(persistent)
        b.setDisplacementCutoff(0.5)
        res = b.compress(**prm)
        out.append((res, b.getVertexPositions()))
    (r1, x1), (r2, x2) = out
    for k in ("phi", "steps", "state", "fire_iterations"):
        assert np.array_equal(r1[k], r2[k]), k
    assert np.array_equal(x1, x2)


def test_batch_scale_matches_single(cuda_device):
    pks = _systems("bidisperse_harmonic", [16, 24], 0.40, seed=3)
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    b.calcNeighborLists()
    b.scaleVertices(np.array([1.01, 0.99]))
    b.calcForceEnergy()
    pos, phi = b.getVertexPositions(), b.getPhis()
    for s, (pk, f) in enumerate(zip(pks, (1.01, 0.99))):
        d = _single(pk, **kw)
        d.scaleVertices(f)
        d.calcForceEnergy()
        assert rel_inf(pos[b.system_slice(s)], d.getVertexPositions()) < 1e-14
        assert phi[s] == pytest.approx(d.getPhi(), rel=1e-13)
        d.close()


def test_batch_compress_matches_per_system_loop(cuda_device):
    pks = batch_packings(3, seed=5, rings=(16, 40))
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    prm = dict(dphi=2e-2, min_dphi=1e-3, fire_dt=1e-2, tol0=1e-6, max_fire_iters=50000, max_steps=5)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    res = b.compress(**prm)
    assert np.all(res["steps"] >= 1)
    for s, pk in enumerate(pks):
        d = DPM2D.from_packing(pk, **kw)
        d.calcNeighborList(d.setDisplacementCutoff(0.5, 2.0 * d.getMeanVertexRadius()))
        one = compress_system(d, **prm)
        assert one["steps"] == res["steps"][s]
        assert one["state"] == res["state"][s]
        # FIRE stops at max |F| <= tol0 / sigma: the two runs' end points (and
        # so the areas behind phi) agree to the residual force, not to rounding
        assert one["phi"] == pytest.approx(res["phi"][s], rel=1e-6)
        d.close()


@pytest.mark.parametrize("criterion,max_fire_iters,energy_tol", [("force", 50000, 0.0), ("force", 150, 0.0),
                                                                 ("energy", 50000, 1e-9)])
def test_batch_compress_device_loop_matches_stepwise(cuda_device, criterion, max_fire_iters, energy_tol):
    # the whole protocol as one graph launch against the host-driven loop on
    # the same systems: the same kernels in the same order, so the same
    # states bit for bit (150 iterations: the FIRE limit binds every step)
    pks = batch_packings(4, seed=11, rings=(16, 40))
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    prm = dict(dphi=2e-2, min_dphi=2e-3, fire_dt=1e-2, tol0=1e-6, max_fire_iters=max_fire_iters, max_steps=8,
               criterion=criterion, energy_tol=energy_tol)
    out = []
    for stepwise in (False, True):
        b = Batch.from_packings(pks, **kw)
        b.setDisplacementCutoff(0.5)
        res = b.compress(stepwise=stepwise, **prm)
        out.append((res, b.getVertexPositions(), b.getVertexRadii()))
    (dev, xd, rd), (host, xh, rh) = out
    assert np.all(dev["steps"] >= 1)
    for k in ("steps", "state", "fire_iterations"):
        assert np.array_equal(dev[k], host[k]), k
    assert np.array_equal(dev["phi"], host["phi"])
    assert np.array_equal(xd, xh) and np.array_equal(rd, rh)
    if max_fire_iters == 150:
        assert np.all(dev["fire_iterations"] <= 150 * dev["steps"])


def test_batch_autotune_and_lanes(cuda_device):
    pks = _systems("smooth_lj", [16, 32], 0.40, seed=9)
    kw = dict(potential="lennardJones", interaction="vertexSmooth", ea=1.0, el=1.0, eb=0.01, ec=1.0, LJcutoff=2.5)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    b.calcNeighborLists()
    b.calcForceEnergy()
    f1 = b.getVertexForces()
    lanes = b.autotune(5)
    assert lanes in (1, 2, 4)
    assert b.getTileShape() in [(1, 128), (1, 192), (2, 128), (2, 192), (4, 256)]
    assert b.getTileShape()[0] == lanes
    for shape in [(1, 128), (1, 192), (2, 128), (2, 192), (4, 256)]:
        b.setTileShape(*shape)
        assert b.getTileShape() == shape
        b.calcForceEnergy()
        assert rel_inf(b.getVertexForces(), f1) < 1e-12
    for L in (1, 2, 4):
        b.setLanes(L)
        b.calcForceEnergy()
        assert rel_inf(b.getVertexForces(), f1) < 1e-12


def _reference_system(pk, potential_id, interaction_id, ea, el, eb, ec, lj=2.5):
    """oracle/_ref (the reference's kernels as host code) holding one packing."""
    R = oracle.ref()
    R.ref_create(pk.num_particles, np.ascontiguousarray(pk.nv_list, dtype=np.int64))
    R.ref_set_box(float(pk.box[0]), float(pk.box[1]))
    R.ref_set_types(potential_id, interaction_id, 0, 0)
    R.ref_set_energy_costs(ea, el, eb, ec)
    R.ref_set_lj_cutoff(lj)
    arrs = [np.ascontiguousarray(a, dtype=np.float64)
            for a in (pk.pos, np.zeros_like(pk.pos), pk.rad, pk.l0, pk.theta0, pk.a0)]
    R.ref_set_state(*[a.ctypes.data for a in arrs])
    _reference_system.keep = arrs
    return R


def test_batch_forces_match_oracle(cuda_device):
    # every system of a batch against the CPU oracle directly (not only the
    # single-system path): smooth LJ, systems of 8 to 40 rings
    pks = _systems("smooth_lj", [8, 24, 40], 0.40, seed=103)
    kw = dict(potential="lennardJones", interaction="vertexSmooth", ea=1.0, el=1.0, eb=0.01, ec=1.0, LJcutoff=2.5)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    b.calcNeighborLists()
    b.calcForceEnergy()
    f, u = b.getVertexForces(), b.getPotentialEnergies()
    for s, pk in enumerate(pks):
        S = oracle.System(pk.nv_list, pk.box, "lennardJones", "vertexSmooth", 1.0, 1.0, 0.01, 1.0, lj_cutoff=2.5)
        S.neighbor_list(pk.pos, pk.rad, S.cut_distance(0.5))
        out = S.force_energy(pk.pos, pk.rad, pk.a0, pk.l0, pk.theta0)
        assert rel_inf(f[b.system_slice(s)], out["force"]) < 1e-12
        assert u[s] == pytest.approx(out["potential_energy"], rel=1e-12)


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_batch_compress_step_matches_reference(cuda_device):
    # one search step of every system (FIRE to tol0 / sigma, then the
    # jammed / under / over decision and the scale) against the same step of
    # compressFIRE.cpp run on the reference's own kernels
    pks = batch_packings(3, seed=5, rings=(16, 40))
    kw = dict(potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0)
    prm = dict(dphi=2e-2, min_dphi=1e-3, fire_dt=1e-2, tol0=1e-6, max_fire_iters=50000, max_steps=1)
    b = Batch.from_packings(pks, **kw)
    b.setDisplacementCutoff(0.5)
    res = b.compress(**prm)
    pos = b.getVertexPositions()
    for s, pk in enumerate(pks):
        R = _reference_system(pk, 0, 0, 1.0, 1.0, 0.01, 1.0)
        R.ref_calc_force_energy()
        phi0 = R.ref_phi()
        sigma = 2 * math.sqrt(pk.a0.sum() / (math.pi * pk.num_particles))  # getMeanParticleSize
        out = compress_search_step(R, sigma, phi0, phi0, prm["dphi"], (pk.rad, pk.l0, pk.a0),
                                   (pk.pos, pk.rad, pk.l0, pk.a0), fire_dt=prm["fire_dt"], tol0=prm["tol0"],
                                   max_iter=prm["max_fire_iters"], min_dphi=prm["min_dphi"])
        # a search still running after its one allowed step reads state 2 in the batch
        assert res["state"][s] == (2 if out["state"] == 0 else out["state"])
        assert res["steps"][s] == 1
        # FIRE paths agree to rounding, so iteration counts and the relaxed
        # state agree to the residual force, not bit for bit
        assert abs(int(res["fire_iterations"][s]) - out["iterations"]) <= max(20, 0.05 * out["iterations"])
        assert res["phi"][s] == pytest.approx(out["phi"], rel=1e-6)
        ref_pos = np.zeros(2 * pk.num_vertices)
        R.ref_get(0, ref_pos)
        assert rel_inf(pos[b.system_slice(s)], ref_pos) < 1e-5
