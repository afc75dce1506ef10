"""Quasi-static compression to jamming, one system at a time.

The protocol of the reference's compressFIRE driver (compressFIRE.cpp:101-205,
without its file output and the optional Langevin thermalisation): at each
compression step, FIRE with dt = fire_dt * sigma and force tolerance
tol0 / sigma (sigma the mean particle size, DPM2D::getMeanParticleSize),
then

* jammed:       tol < F < 2 tol   -> stop,
* under-jammed: F <= tol          -> keep this state, grow phi by dphi,
* over-jammed:  F >= 2 tol        -> halve dphi, go back to the last
  under-jammed state and grow its phi by the halved step,

with F the largest force component (criterion "energy" reads the potential
energy per ring against energy_tol instead, the form the reference keeps
commented out beside it).  A system also stops once its halved step falls
below ``min_dphi``.

``compress_system`` runs it on one :class:`DPM2D` context through the
single-system API; the batched ``Batch.compress`` runs the same protocol on
every system of a batch at once (cr_batch_compress).
"""
from __future__ import annotations

import math

import numpy as np

from .dpm2d import DPM2D
from .synth import Packing


def compress_system(d: DPM2D, dphi=1e-3, min_dphi=1e-6, fire_dt=1e-2, tol0=1e-10, energy_tol=1e-20,
                    max_fire_iters=100000, max_steps=1000, criterion="force", cutoff=0.5) -> dict:
    d.calcForceEnergy()
    phi = d.getPhi()
    prev = phi
    state, steps, fire_total = 0, 0, 0
    # the starting configuration is the first "last under-jammed" state
    saved = (d.getVertexPositions(), d.getVertexRadii(), d.getRestLengths(), d.getRestAreas())
    while steps < max_steps and state == 0:
        sigma = d.getMeanParticleSize()
        dt = fire_dt * sigma
        tol = tol0 / sigma
        d.initFIRE([0.2, 0.5, 1.1, 0.99, dt, 10 * dt, 0.2], 20, 0, d.numVertices)
        cut = d.setDisplacementCutoff(cutoff, 2.0 * d.getMeanVertexRadius())
        d.calcNeighborList(cut)
        d.resetLastPositions()
        d.calcForceEnergy()
        its, fmax = d.minimizeFIRE(tol, max_fire_iters)
        fire_total += its
        steps += 1
        if criterion == "energy":
            u = d.getPotentialEnergy() / d.numParticles
            jam, over, under = energy_tol < u < 2 * energy_tol, u >= 2 * energy_tol, u <= energy_tol
        else:
            jam, over, under = tol < fmax < 2 * tol, fmax >= 2 * tol, fmax <= tol
        if jam:
            state = 1
            break
        if under:
            scale = math.sqrt((phi + dphi) / phi)
            prev = phi
            saved = (d.getVertexPositions(), d.getVertexRadii(), d.getRestLengths(), d.getRestAreas())
        else:
            dphi *= 0.5
            scale = math.sqrt((prev + dphi) / prev)
            d.setVertexPositions(saved[0])
            d.setVertexRadii(saved[1])
            d.setRestLengths(saved[2])
            d.setRestAreas(saved[3])
        if dphi < min_dphi:
            state = 3
            scale = 1.0
        if scale != 1.0:
            d.calcNeighborList(d.setDisplacementCutoff(cutoff, 2.0 * d.getMeanVertexRadius()))
            d.calcForceEnergy()  # ring centroids of the current positions
            d.scaleVertices(scale)
        d.calcNeighborList(d.setDisplacementCutoff(cutoff, 2.0 * d.getMeanVertexRadius()))
        d.calcForceEnergy()
        phi = d.getPhi()
    if state == 0:
        state = 2
    return {"phi": phi, "steps": steps, "state": state, "fire_iterations": fire_total}


def batch_packings(num_systems: int, seed: int, rings=(16, 512), calA0_range=(1.0, 1.2)) -> list[Packing]:
    """Systems of the batched compression workload: ring counts uniform in
    ``rings`` (even), bidisperse 1:1.4 with nv 16/22, calA0 uniform in
    ``calA0_range``, rings on a triangular lattice without overlap (packing
    fraction about 0.5-0.57; ``prepare_batch`` brings them to the start)."""
    from .workloads import lattice_packing

    rng = np.random.default_rng(seed)
    out = []
    for s in range(num_systems):
        n = int(rng.integers(rings[0], rings[1] + 1))
        n += n % 2
        nv = [16] * (n // 2) + [22] * (n // 2)
        a0 = [1.0] * (n // 2) + [1.4 ** 2] * (n // 2)
        calA0 = float(rng.uniform(*calA0_range))
        out.append(lattice_packing(nv, a0, calA0, seed=seed * 1000 + s))
    return out


def prepare_batch(b, phi0: float = 0.60, step: float = 0.02, tol0: float = 1e-6, fire_dt: float = 1e-2,
                  max_fire_iters: int = 20000) -> np.ndarray:
    """Compress every system of a batch to packing fraction ``phi0`` in
    steps of at most ``step``, relaxing with FIRE to tol0 / sigma after each."""
    b.setDisplacementCutoff(0.5)
    b.calcNeighborLists()
    b.calcForceEnergy()
    phi = b.getPhis()
    for _ in range(1000):
        if np.all(phi >= phi0 * (1 - 1e-12)):
            break
        target = np.minimum(phi + step, phi0)
        b.scaleVertices(np.sqrt(target / phi))
        sigma = b.getMeanParticleSizes()
        b.initFIRE([0.2, 0.5, 1.1, 0.99, fire_dt, 10 * fire_dt, 0.2], 20, dt=fire_dt * sigma)
        b.fireMinimize(tol0 / sigma, max_fire_iters)
        b.calcForceEnergy()
        phi = b.getPhis()
    return phi
