"""Prepared benchmark states built with the library itself.

A dense packing cannot be placed directly: rings are first placed without
overlap at low packing fraction, then compressed the way the reference's
compressFIRE driver does it (compressFIRE.cpp:101-205): scale the rings about
their centroids with ``scaleVertices(sqrt(phi_new / phi))`` (src/DPM2D.cu:1802-1811)
and relax with FIRE after every step.  At the end the whole system (box,
positions, radii, rest lengths, rest areas) is rescaled uniformly so the ring
sizes are the nominal ones again; a uniform rescaling leaves the packing
fraction unchanged.
"""
from __future__ import annotations

import math

import numpy as np

from . import synth
from .dpm2d import DPM2D, simControl


def lattice_packing(nv_list, a0_list, calA0, seed: int, spacing_scale: float = 1.02) -> synth.Packing:
    """Rings on a triangular lattice of discs (no overlap), random site order."""
    nv_list = np.asarray(nv_list, dtype=np.int64)
    a0 = np.asarray(a0_list, dtype=np.float64)
    n = len(nv_list)
    ring_r = np.sqrt(2.0 * a0 / (nv_list * np.sin(2.0 * np.pi / nv_list)))
    rads = np.array([synth.ring_rest_shape(int(k), float(a), calA0)[2] for k, a in zip(nv_list, a0)])
    a = 2.0 * float((ring_r + rads).max()) * spacing_scale
    nx = int(math.ceil(math.sqrt(n * 2.0 / math.sqrt(3.0))))
    ny = int(math.ceil(n / nx))
    ny += ny % 2
    rng = np.random.Generator(np.random.MT19937(seed))
    sites = rng.permutation(nx * ny)[:n]
    ix, iy = sites % nx, sites // nx
    centres = np.stack([(ix + 0.5 * (iy % 2)) * a, iy * a * math.sqrt(3.0) / 2.0], axis=1)
    box = np.array([nx * a, ny * a * math.sqrt(3.0) / 2.0])
    pk = synth.make_packing(nv_list, a0, calA0, 0.5, seed=seed, placement="uniform")
    # re-place vertices around the lattice centres (make_packing's uniform centres are discarded)
    pid = np.repeat(np.arange(n), nv_list)
    offs = pk.pos.reshape(-1, 2) - pk.centres[pid]
    pos = offs + centres[pid]
    pk.pos = pos.reshape(-1).copy()
    pk.centres = centres
    pk.box = box
    pk.meta["placement"] = "lattice"
    return pk


def compress(d: DPM2D, phi0: float, phi1: float, dphi: float = 0.05, fire_dt: float = 2e-3,
             tol_mid: float = 1e-2, tol_end: float = 1e-4, max_iter: int = 20000) -> dict:
    """Grow rings from preferred packing fraction phi0 to phi1 with FIRE relaxation.

    Uses the potential currently set on ``d``; large steps need a bounded
    (harmonic) repulsion, as Lennard-Jones overlaps of a few percent of a ring
    radius give forces that no FIRE step survives.
    """
    phi = phi0
    iters = 0
    cutoff_ = 0.5
    fmax = float("nan")
    while True:
        size = 2.0 * d.getMeanVertexRadius()
        cut = d.setDisplacementCutoff(cutoff_, size)
        d.calcNeighborList(cut)
        d.resetLastPositions()
        d.calcForceEnergy()
        d.initFIRE([0.2, 0.5, 1.1, 0.99, fire_dt, 10 * fire_dt, 0.2], 20, 0, d.numVertices)
        it, fmax = d.minimizeFIRE(tol_end if phi >= phi1 else tol_mid, max_iter)
        iters += it
        if phi >= phi1:
            break
        new = min(phi1, phi + dphi)
        d.calcParticlePositions()
        d.scaleVertices(math.sqrt(new / phi))
        phi = new
    return {"fire_iterations": iters, "max_force": fmax}


def rescale_lengths(d: DPM2D, f: float) -> None:
    """Multiply every length of the system by f (areas by f^2)."""
    d.setBoxSize(d.getBoxSize() * f)
    d.setVertexPositions(d.getVertexPositions() * f)
    d.setVertexRadii(d.getVertexRadii() * f)
    d.setRestLengths(d.getRestLengths() * f)
    d.setRestAreas(d.getRestAreas() * f * f)


def prepared_deformable(workload: str = "smooth_lj", rings: int | None = None, seed: int = 20261203,
                        phi_start: float = 0.40,
                        placement: str | None = None) -> tuple[DPM2D, dict]:
    """A relaxed packing of a deformable-ring workload at its target phi.

    "smooth_lj": 1024 rings nv 32/45, smooth vertex-segment LJ (rc 2.5),
    calA0 1.05, phi 0.85.  ``rings`` scales the ring count (even small/large
    split).
    """
    c = synth.workload_config(workload, rings)
    n = len(c["nv"])
    if placement is None:
        placement = "rsa" if n <= 4096 else "lattice"
    if placement == "lattice":
        pk = lattice_packing(c["nv"], c["a0"], c["calA0"], seed)
        phi_start = synth.preferred_phi(pk.nv_list, pk.a0, pk.rad, pk.box)
    else:
        pk = synth.make_packing(c["nv"], c["a0"], c["calA0"], phi_start, seed=seed, placement="rsa")
    kw = {k: c[k] for k in ("potential", "interaction", "ea", "el", "eb", "ec", "dt") if k in c}
    if "LJcutoff" in c:
        kw["LJcutoff"] = c["LJcutoff"]
    d = DPM2D.from_packing(pk, **kw)
    # Compress with soft shape constants and harmonic repulsion (bounded
    # forces, large stable FIRE steps), rescale to the nominal ring size, then
    # switch to the configuration's potential and shape constants and relax
    # with a FIRE step small enough for its stiffest mode.
    d.setPotentialType(simControl.potentialEnum.harmonic)
    d.setEnergyCosts(1.0, 1.0, 0.01, c["ec"])
    info = compress(d, phi_start, c["phi"])
    rescale_lengths(d, math.sqrt(phi_start / c["phi"]))
    d.setPotentialType(getattr(simControl.potentialEnum, c["potential"]))
    d.setEnergyCosts(c["ea"], c["el"], c["eb"], c["ec"])
    if "LJcutoff" in c:
        d.setLJcutoff(c["LJcutoff"])
    final = compress(d, c["phi"], c["phi"], fire_dt=1e-4, tol_end=1e-4, max_iter=30000)
    info["fire_iterations"] += final["fire_iterations"]
    info["max_force"] = final["max_force"]
    size = 2.0 * d.getMeanVertexRadius()
    cut = d.setDisplacementCutoff(0.5, size)
    d.calcNeighborList(cut)
    d.resetLastPositions()
    d.calcForceEnergy()
    info.update(config=c, placement=placement, phi=d.getPreferredPhi(), cut_distance=cut, seed=seed)
    return d, info


def prepared_ellipses(n: int | None = None, seed: int = 20261205, phi_start: float = 0.2, dphi: float = 0.01,
                      relax_steps: int = 200, ec_compress: float = 100.0, wca_steps: int = 3000) -> tuple[DPM2D, dict]:
    """Rigid bumpy ellipses (4096 rings of 24 vertices, aspect
    ratio U[1.2, 2.0], WCA) at their target rigid packing fraction.

    Rings are placed without overlap at ``phi_start`` and compressed affinely
    (ring centres and box scaled by sqrt(phi / phi_new), shapes unchanged) in
    steps of ``dphi`` under a stiff harmonic repulsion (bounded forces), each
    step followed by ``relax_steps`` steps of rigid Langevin dynamics at the
    configuration's temperature; then the WCA potential is switched on and the
    packing relaxed with ``wca_steps`` steps at a tenth of the time step.
    """
    import time

    c = synth.workload_config("rigid_ellipses", n)
    t0 = time.perf_counter()
    pk = synth.make_ellipse_packing(c["n"], c["nv"], c["ratio_range"], phi_start, seed=seed)
    d = DPM2D.from_packing(pk, potential="harmonic", interaction=c["interaction"], ec=ec_compress, dt=c["dt"])
    d.setShapeType(simControl.shapeEnum.rigid)
    cut = d.setDisplacementCutoff(0.5, 2.0 * float(pk.rad.mean()))
    ring_of = np.repeat(np.arange(pk.num_particles), pk.nv_list)
    d.setSeed(seed)
    phi, steps = phi_start, 0
    while phi < c["phi"] - 1e-12:
        nxt = min(c["phi"], phi + dphi)
        s = math.sqrt(phi / nxt)
        d.calcParticlePositions()
        cen = d.getParticlePositions().reshape(-1, 2)[ring_of]
        x = d.getVertexPositions().reshape(-1, 2)
        box = d.getBoxSize()
        rel = x - cen
        rel -= box * np.round(rel / box)
        d.setBoxSize(box * s)
        d.setVertexPositions((cen * s + rel).reshape(-1))
        d.calcNeighborList(cut)
        d.initRigidLangevin(c["T"], c["gamma"], readState=False)
        d.rigidLangevinLoop(relax_steps)
        phi, steps = nxt, steps + 1
    d.setPotentialType(getattr(simControl.potentialEnum, c["potential"]))
    d.setEnergyCosts(0.0, 0.0, 0.0, c["ec"])
    cut = d.setDisplacementCutoff(0.5, 2.0 * float(pk.rad.mean()))
    d.calcNeighborList(cut)
    d.setTimeStep(0.1 * c["dt"])
    d.initRigidLangevin(c["T"], c["gamma"], readState=False)
    d.rigidLangevinLoop(wca_steps)
    d.setTimeStep(c["dt"])
    box = d.getBoxSize()
    info = dict(config=c, phi=float(np.sum(pk.a0) / (box[0] * box[1])), compression_steps=steps,
                prep_seconds=time.perf_counter() - t0, cut_distance=cut)
    return d, info


def tile_system(d: DPM2D, k: int, config: dict) -> DPM2D:
    """A k x k periodic tiling of the system held by ``d`` (positions,
    velocities, radii, rest lengths / areas / angles, box) as a new context
    with the workload ``config``'s potential and constants; lists built and
    forces evaluated.  A tiling of a periodic packing is itself a packing at
    the same packing fraction."""
    nvl = d.numVertexInParticleList
    box = d.getBoxSize()
    pos = d.getVertexPositions().reshape(-1, 2)
    copies = [(pos + np.array([ix * box[0], iy * box[1]])).reshape(-1) for iy in range(k) for ix in range(k)]
    n = k * k
    pk = synth.Packing(nv_list=np.tile(nvl, n), pos=np.concatenate(copies), vel=np.tile(d.getVertexVelocities(), n),
                       rad=np.tile(d.getVertexRadii(), n), l0=np.tile(d.getRestLengths(), n),
                       theta0=np.tile(d.getRestAngles(), n), a0=np.tile(d.getRestAreas(), n), box=box * k,
                       centres=np.zeros((n * d.numParticles, 2)))
    kw = {key: config[key] for key in ("potential", "interaction", "ea", "el", "eb", "ec", "dt") if key in config}
    if "LJcutoff" in config:
        kw["LJcutoff"] = config["LJcutoff"]
    t = DPM2D.from_packing(pk, **kw)
    cut = t.setDisplacementCutoff(0.5, 2.0 * t.getMeanVertexRadius())
    t.calcNeighborList(cut)
    t.resetLastPositions()
    t.calcForceEnergy()
    return t
