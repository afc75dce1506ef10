"""Seeded synthetic ring-polymer packings that follow cudaRing's conventions.

The reference builds its inputs in ``DPM2D::setPolySizeDistribution``
(src/DPM2D.cu:1545-1588), ``DPM2D::setRandomParticles`` (src/DPM2D.cu:1601-1629)
and ``DPM2D::initVerticesOnParticles`` (src/DPM2D.cu:1678-1691):

* rest length ``l0 = 2 sqrt(pi * calA0 * (nv tan(pi/nv)/pi) * a0) / nv``,
  rest angle ``theta0 = 2 pi / nv``, vertex radius ``rad = l0 / 2``
  (src/DPM2D.cu:1577-1581);
* vertices on a circle of radius ``R = sqrt(2 a0 / (nv sin(2 pi / nv)))``
  around the ring centre, counter-clockwise, at angle ``2 pi v / nv`` where
  ``v`` is the global vertex index (src/DPM2D.cu:1685-1687);
* the packing fraction is ``(sum_p A_p + pi sum_p r_first(p)^2 (nv_p/2 - 1)) / (Lx Ly)``
  (src/DPM2D.cu:1202-1220, with ``kernelCalcVertexArea`` at
  include/cudaKernel.cuh:1636-1642); the box is sized with the rest areas ``a0``
  (``getPreferredPhi``).

Everything here is plain numpy: it builds host arrays that are then handed to
the library through its C ABI.  Vertex positions get a per-coordinate uniform
jitter in ``[-jitter, jitter] * l0`` (the reference uses ``1e-3 * l0 * U[0,1)``;
the workloads of this project use +-0.05 l0).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

__all__ = ["Packing", "ring_rest_shape", "make_packing", "preferred_phi", "rsa_centres",
           "workload_config"]


@dataclass
class Packing:
    """Host arrays for one 2-D periodic system, in the reference's layout."""

    nv_list: np.ndarray          # int64 [Np] vertices per ring
    pos: np.ndarray              # float64 [2 Nv] AoS x0,y0,x1,y1,...
    vel: np.ndarray              # float64 [2 Nv]
    rad: np.ndarray              # float64 [Nv]
    l0: np.ndarray               # float64 [Nv]
    theta0: np.ndarray           # float64 [Nv]
    a0: np.ndarray               # float64 [Np]
    box: np.ndarray              # float64 [2]
    centres: np.ndarray          # float64 [Np, 2] ring centres used for placement
    meta: dict = field(default_factory=dict)

    @property
    def num_particles(self) -> int:
        return int(self.nv_list.shape[0])

    @property
    def num_vertices(self) -> int:
        return int(self.nv_list.sum())

    def first_vertex(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.nv_list)[:-1]]).astype(np.int64)

    def particle_id(self) -> np.ndarray:
        return np.repeat(np.arange(self.num_particles, dtype=np.int64), self.nv_list)


def ring_rest_shape(nv: int, a0: float, calA0: float) -> tuple[float, float, float]:
    """(l0, theta0, rad) for one ring (src/DPM2D.cu:1577-1581)."""
    calA0_ring = calA0 * nv * math.tan(math.pi / nv) / math.pi
    l0 = 2.0 * math.sqrt(math.pi * calA0_ring * a0) / nv
    return l0, 2.0 * math.pi / nv, 0.5 * l0


def preferred_phi(nv_list: np.ndarray, a0: np.ndarray, rad: np.ndarray, box: np.ndarray) -> float:
    """``DPM2D::getPreferredPhi`` (src/DPM2D.cu:1222-1240)."""
    first = np.concatenate([[0], np.cumsum(nv_list)[:-1]])
    vertex_area = rad[first] ** 2 * (0.5 * nv_list - 1)
    return float((a0.sum() + math.pi * vertex_area.sum()) / (box[0] * box[1]))


def rsa_centres(radii: np.ndarray, box: float, rng: np.random.Generator,
                max_tries: int = 2000) -> np.ndarray:
    """Random sequential addition of non-overlapping discs in a periodic box.

    Large discs are placed first.  Used to build overlap-free starting
    configurations; raises if a disc cannot be placed.
    """
    n = radii.shape[0]
    order = np.argsort(-radii, kind="stable")
    rmax = float(radii.max())
    ncell = max(1, int(box // (2 * rmax)))
    csize = box / ncell
    cells: dict[tuple[int, int], list[int]] = {}
    centres = np.zeros((n, 2))
    for idx in order:
        r = radii[idx]
        for _ in range(max_tries):
            c = rng.uniform(0.0, box, size=2)
            cx, cy = int(c[0] // csize) % ncell, int(c[1] // csize) % ncell
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for j in cells.get(((cx + dx) % ncell, (cy + dy) % ncell), ()):
                        d = c - centres[j]
                        d -= box * np.round(d / box)
                        if d @ d < (r + radii[j]) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                centres[idx] = c
                cells.setdefault((cx, cy), []).append(idx)
                break
        else:
            raise RuntimeError("rsa_centres: could not place disc; lower the density")
    return centres


def make_packing(nv_list, a0_list, calA0, phi: float, seed: int, jitter: float = 0.05,
                 placement: str = "uniform", disc_scale: float = 1.0) -> Packing:
    """Build a seeded packing.

    ``calA0`` may be a scalar or one value per ring.  ``placement`` is
    ``"uniform"`` (ring centres uniform in the box, the benchmark workloads'
    convention; rings may overlap) or ``"rsa"`` (non-overlapping discs of radius
    ``disc_scale * (R + rad)``).
    """
    nv_list = np.asarray(nv_list, dtype=np.int64)
    a0 = np.asarray(a0_list, dtype=np.float64)
    np_ = nv_list.shape[0]
    calA0 = np.broadcast_to(np.asarray(calA0, dtype=np.float64), (np_,))
    rng = np.random.Generator(np.random.MT19937(seed))
    nv_tot = int(nv_list.sum())
    l0 = np.empty(nv_tot)
    theta0 = np.empty(nv_tot)
    rad = np.empty(nv_tot)
    first = np.concatenate([[0], np.cumsum(nv_list)[:-1]]).astype(np.int64)
    ring_r = np.empty(np_)
    for p in range(np_):
        nv = int(nv_list[p])
        l, t, r = ring_rest_shape(nv, float(a0[p]), float(calA0[p]))
        l0[first[p]:first[p] + nv] = l
        theta0[first[p]:first[p] + nv] = t
        rad[first[p]:first[p] + nv] = r
        ring_r[p] = math.sqrt(2.0 * a0[p] / (nv * math.sin(2.0 * math.pi / nv)))
    vertex_area = rad[first] ** 2 * (0.5 * nv_list - 1)
    L = math.sqrt((a0.sum() + math.pi * vertex_area.sum()) / phi)
    box = np.array([L, L])
    if placement == "uniform":
        centres = rng.uniform(0.0, L, size=(np_, 2))
    elif placement == "rsa":
        centres = rsa_centres(disc_scale * (ring_r + rad[first]), L, rng)
    else:
        raise ValueError(placement)
    pos = np.empty((nv_tot, 2))
    vid = np.arange(nv_tot)
    pid = np.repeat(np.arange(np_), nv_list)
    ang = 2.0 * math.pi * vid / nv_list[pid]
    pos[:, 0] = ring_r[pid] * np.cos(ang) + centres[pid, 0]
    pos[:, 1] = ring_r[pid] * np.sin(ang) + centres[pid, 1]
    pos += jitter * l0[:, None] * rng.uniform(-1.0, 1.0, size=(nv_tot, 2))
    return Packing(nv_list=nv_list, pos=pos.reshape(-1).copy(), vel=np.zeros(2 * nv_tot), rad=rad,
                   l0=l0, theta0=theta0, a0=a0.copy(), box=box, centres=centres,
                   meta={"seed": seed, "phi": phi, "jitter": jitter, "placement": placement})


def ellipse_vertices(nv: int, a: float, b: float, orientation: float) -> np.ndarray:
    """nv points at equal arc length on the ellipse x=a cos t, y=b sin t,
    counter-clockwise, rotated by ``orientation`` (BumpyEllipse::initEllipse,
    src/BumpyEllipse.cu:39-75, places vertices at equal arc length too; here
    the arc length is integrated numerically on a fine grid)."""
    t = np.linspace(0.0, 2.0 * np.pi, 20001)
    ds = np.hypot(a * np.sin(t), b * np.cos(t))
    s = np.concatenate([[0.0], np.cumsum(0.5 * (ds[1:] + ds[:-1]) * np.diff(t))])
    targets = np.arange(nv) * s[-1] / nv
    tk = np.interp(targets, s, t)
    x, y = a * np.cos(tk), b * np.sin(tk)
    c, sn = np.cos(orientation), np.sin(orientation)
    return np.stack([c * x - sn * y, sn * x + c * y], axis=1)


def make_ellipse_packing(n: int, nv: int, ratio_range: tuple[float, float], phi: float, seed: int,
                         a0: float = 1.0, placement: str = "rsa") -> Packing:
    """Rigid "bumpy ellipse" rings: aspect ratio a/b uniform in ratio_range,
    area a0 (a = sqrt(ratio a0 / pi), b = a / ratio), nv vertices at equal arc
    length, vertex radius half the arc spacing, random orientation.  The box
    is sized with the rigid packing fraction sum(a0) / L^2 (DPM2D::getRigidPhi,
    src/DPM2D.cu:1242-1252); ``placement`` "rsa" places circumscribing discs
    without overlap, "uniform" anywhere."""
    rng = np.random.Generator(np.random.MT19937(seed))
    ratios = rng.uniform(ratio_range[0], ratio_range[1], n)
    orient = rng.uniform(0.0, 2.0 * np.pi, n)
    L = math.sqrt(n * a0 / phi)
    pts, rads, l0s, th0s, rcirc = [], [], [], [], []
    for q in range(n):
        a = math.sqrt(ratios[q] * a0 / math.pi)
        b = a / ratios[q]
        v = ellipse_vertices(nv, a, b, orient[q])
        seg = np.roll(v, -1, axis=0) - v
        lens = np.hypot(seg[:, 0], seg[:, 1])
        r = 0.5 * lens.mean()
        pts.append(v)
        rads.append(np.full(nv, r))
        l0s.append(lens)
        th0s.append(np.full(nv, 2.0 * np.pi / nv))
        rcirc.append(a + r)
    rcirc = np.array(rcirc)
    if placement == "rsa":
        centres = rsa_centres(rcirc, L, rng)
    else:
        centres = rng.uniform(0.0, L, size=(n, 2))
    pos = np.concatenate([p + c for p, c in zip(pts, centres)]).reshape(-1)
    nv_list = np.full(n, nv, dtype=np.int64)
    return Packing(nv_list=nv_list, pos=pos, vel=np.zeros_like(pos), rad=np.concatenate(rads),
                   l0=np.concatenate(l0s), theta0=np.concatenate(th0s), a0=np.full(n, a0), box=np.array([L, L]),
                   centres=centres, meta={"seed": seed, "phi": phi, "ratios": ratios, "placement": placement})


def workload_config(name: str, scale_rings: int | None = None) -> dict:
    """Ring counts and parameters of the benchmark workloads, by name.

    "bidisperse_harmonic": 32 rings, nv 16/22 bidisperse 1:1.4, harmonic,
        calA0 1.0, phi 0.70.
    "smooth_lj": 1024 rings, nv 32/45 (1:1.4), smooth LJ rc 2.5, calA0 1.05,
        phi 0.85; the shape constants are those of the reference's NVE driver
        (ea 1e5, el 20, eb 10; runNVE.cpp:39), stiff enough that the LJ well
        (epsilon 1) does not crumple the rings.
    "rigid_ellipses": 4096 rigid ellipses, 24 vertices, WCA, phi 0.65.
    "dense_harmonic": 256 rings, nv 32, harmonic, phi 0.88 (derivatives).
    The batched FIRE compression workload lives in the batch module.
    ``scale_rings`` overrides the ring count (even split small/large).
    """
    if name == "bidisperse_harmonic":
        n = scale_rings or 32
        nv = [16] * (n // 2) + [22] * (n - n // 2)
        a0 = [1.0] * (n // 2) + [1.4 ** 2] * (n - n // 2)
        return dict(nv=nv, a0=a0, calA0=1.0, phi=0.70, potential="harmonic", interaction="vertexVertex",
                    ea=1.0, el=1.0, eb=0.01, ec=1.0, dt=0.005, T=1e-3)
    if name == "smooth_lj":
        n = scale_rings or 1024
        nv = [32] * (n // 2) + [45] * (n - n // 2)
        a0 = [1.0] * (n // 2) + [1.4 ** 2] * (n - n // 2)
        return dict(nv=nv, a0=a0, calA0=1.05, phi=0.85, potential="lennardJones", interaction="vertexSmooth",
                    LJcutoff=2.5, ea=1e5, el=20.0, eb=10.0, ec=1.0, dt=0.002, T=0.01)
    if name == "rigid_ellipses":
        n = scale_rings or 4096
        return dict(rigid=True, n=n, nv=24, ratio_range=(1.2, 2.0), phi=0.65, potential="wca",
                    interaction="vertexVertex", ea=0.0, el=0.0, eb=0.0, ec=1.0, dt=0.001, T=0.1, gamma=1.0,
                    driving=0.1, taup=100.0)
    if name == "dense_harmonic":
        n = scale_rings or 256
        return dict(nv=[32] * n, a0=[1.0] * n, calA0=1.0, phi=0.88, potential="harmonic",
                    interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01, ec=1.0, dt=0.002, T=0.0)
    raise ValueError(f"unknown workload {name!r}")
