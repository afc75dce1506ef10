"""Packings in the reference's on-disk directory format.

The reference's ``ioDPMFile`` (include/FileIO.h) stores a deformable packing
as one text file per array in a directory:

=============================  =============================  ==============
file                           content                        rows
=============================  =============================  ==============
``numVertexInParticleList.dat`` vertices per ring (integer)    N_p
``positions.dat``              x <TAB> y <TAB>                N_v
``velocities.dat``             vx <TAB> vy <TAB>              N_v
``radii.dat``                  vertex radius                  N_v
``restAreas.dat``              a0 per ring                    N_p
``restLengths.dat``            l0 per vertex                  N_v
``restAngles.dat``             theta0 per vertex              N_v
``boxSize.dat``                Lx, Ly (one per line)          2
``shapes.dat``                 area, perimeter, p^2/(4 pi a)  N_p
``params.dat``                 ``name <TAB> value`` lines
=============================  =============================  ==============

Writers follow ``saveDeformablePacking`` (FileIO.h:403-435) and the
``save1DFile`` / ``save2DFile`` / ``save1DIndexFile`` helpers (:153-245):
``setprecision(14)`` (defs.h:16) decimal text, 2-D rows tab-separated with a
trailing tab.  ``digits`` raises the precision (17 round-trips FP64 exactly).
Readers follow ``readDeformablePackingFromDirectory`` (:278-326) and
``readDeformableState`` (:468-474): the first token(s) of each line.
"""
from __future__ import annotations

import math
import os

import numpy as np

from .synth import Packing

PRECISION = 14  # defs.h:16


def _fmt(x: float, digits: int) -> str:
    # std::ostream << setprecision(p) << double: the %g form with p significant digits
    return f"{x:.{digits}g}"


def _save_1d(path: str, data, digits: int) -> None:
    with open(path, "w") as f:
        for x in np.asarray(data, dtype=float).reshape(-1):
            f.write(_fmt(float(x), digits) + "\n")


def _save_1d_index(path: str, data) -> None:
    with open(path, "w") as f:
        for x in np.asarray(data).reshape(-1):
            f.write(f"{int(x)}\n")


def _save_2d(path: str, data, cols: int, digits: int) -> None:
    a = np.asarray(data, dtype=float).reshape(-1, cols)
    with open(path, "w") as f:
        for row in a:
            f.write("".join(_fmt(float(x), digits) + "\t" for x in row) + "\n")


def _read_1d(path: str, rows: int) -> np.ndarray:
    with open(path) as f:
        vals = [float(line.split()[0]) for _, line in zip(range(rows), f)]
    if len(vals) != rows:
        raise ValueError(f"{path}: expected {rows} rows, found {len(vals)}")
    return np.asarray(vals, dtype=np.float64)


def _read_2d(path: str, rows: int) -> np.ndarray:
    out = np.empty((rows, 2), dtype=np.float64)
    n = 0
    with open(path) as f:
        for line in f:
            if n == rows:
                break
            t = line.split()
            out[n, 0], out[n, 1] = float(t[0]), float(t[1])
            n += 1
    if n != rows:
        raise ValueError(f"{path}: expected {rows} rows, found {n}")
    return out.reshape(-1)


def save_packing(dirname: str, d, digits: int = PRECISION, params: dict | None = None) -> None:
    """``ioDPMFile::savePacking`` for a deformable :class:`DPM2D` context."""
    os.makedirs(dirname, exist_ok=True)
    j = lambda name: os.path.join(dirname, name)  # noqa: E731
    nvl = d.numVertexInParticleList
    d.calcParticleShape()
    area, perim = d.getAreas(), d.getPerimeters()
    lines = [("numParticles", d.numParticles)]
    for k, v in (params or {}).items():
        lines.append((k, v))
    with open(j("params.dat"), "w") as f:
        for k, v in lines:
            f.write(f"{k}\t{v}\n")
    _save_1d_index(j("numVertexInParticleList.dat"), nvl)
    _save_1d(j("radii.dat"), d.getVertexRadii(), digits)
    _save_2d(j("positions.dat"), d.getVertexPositions(), 2, digits)
    _save_1d(j("restAreas.dat"), d.getRestAreas(), digits)
    _save_1d(j("restLengths.dat"), d.getRestLengths(), digits)
    _save_1d(j("restAngles.dat"), d.getRestAngles(), digits)
    _save_2d(j("velocities.dat"), d.getVertexVelocities(), 2, digits)
    _save_2d(j("shapes.dat"), np.stack([area, perim, perim * perim / (4 * math.pi * area)], axis=1), 3, digits)
    _save_1d(j("boxSize.dat"), d.getBoxSize(), digits)


def save_packing_arrays(dirname: str, pk: Packing, digits: int = PRECISION) -> None:
    """The same files from a :class:`Packing` (no context needed)."""
    os.makedirs(dirname, exist_ok=True)
    j = lambda name: os.path.join(dirname, name)  # noqa: E731
    with open(j("params.dat"), "w") as f:
        f.write(f"numParticles\t{pk.num_particles}\n")
    _save_1d_index(j("numVertexInParticleList.dat"), pk.nv_list)
    _save_1d(j("radii.dat"), pk.rad, digits)
    _save_2d(j("positions.dat"), pk.pos, 2, digits)
    _save_1d(j("restAreas.dat"), pk.a0, digits)
    _save_1d(j("restLengths.dat"), pk.l0, digits)
    _save_1d(j("restAngles.dat"), pk.theta0, digits)
    _save_2d(j("velocities.dat"), pk.vel, 2, digits)
    _save_1d(j("boxSize.dat"), pk.box, digits)


def load_packing(dirname: str, num_particles: int | None = None, read_state: bool = True) -> Packing:
    """``readDeformablePackingFromDirectory`` (+ ``readDeformableState``)."""
    j = lambda name: os.path.join(dirname, name)  # noqa: E731
    if num_particles is None:
        with open(j("numVertexInParticleList.dat")) as f:
            num_particles = sum(1 for line in f if line.strip())
    nvl = _read_1d(j("numVertexInParticleList.dat"), num_particles).astype(np.int64)
    nv = int(nvl.sum())
    pos = _read_2d(j("positions.dat"), nv)
    vel = _read_2d(j("velocities.dat"), nv) if read_state and os.path.exists(j("velocities.dat")) \
        else np.zeros(2 * nv)
    return Packing(nv_list=nvl, pos=pos, vel=vel, rad=_read_1d(j("radii.dat"), nv),
                   l0=_read_1d(j("restLengths.dat"), nv), theta0=_read_1d(j("restAngles.dat"), nv),
                   a0=_read_1d(j("restAreas.dat"), num_particles), box=_read_1d(j("boxSize.dat"), 2),
                   centres=np.zeros((num_particles, 2)))
