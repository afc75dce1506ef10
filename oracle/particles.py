"""CPU restatement of the soft-disk pre-packing stage (test infrastructure only).

Only tests/ and the golden-fixture script use this module, as the checker.  It
restates, in plain Python over numpy arrays, the particle-level steps that
compressFIRE.cpp:53-90 runs before vertex FIRE:

* ``Drand48``: the POSIX drand48 generator (48-bit LCG, a = 0x5DEECE66D,
  c = 0xB, srand48(s) sets the state to (s << 16) | 0x330E), the source of
  every random number of DPM2D::setRandomParticles and initVerticesOnParticles;
* ``set_random_particles``: DPM2D::setRandomParticles (src/DPM2D.cu:1601-1629);
* ``particle_neighbor_list``: kernelCalcParticleNeighborList
  (include/cudaKernel.cuh:1765-1789) with DPM2D::calcParticleNeighborList's
  size rule (src/DPM2D.cu:3521-3545); extractOtherParticle returns the
  listing particle's own radius (include/cudaKernel.cuh:289-296), so the
  test sums it twice;
* ``particle_force_energy``: kernelCalcParticleInteraction
  (include/cudaKernel.cuh:1185-1219) with the pair terms of
  calcContactInteraction / calcLJInteraction / calcAdhesiveInteraction /
  calcWCAInteraction (include/cudaKernel.cuh:531-668);
* ``ParticleFire``: FIRE::minimizerParticleLoop (src/FIRE.cu:45-171) with the
  masses of DPM2D::setParticleMassFIRE (src/DPM2D.cu:3676-3684), and the
  driver loop of compressFIRE.cpp:66-78;
* ``vertices_on_particles``: DPM2D::initVerticesOnParticles
  (src/DPM2D.cu:1678-1691).

Pinned against the reference's own kernels compiled as host code
(oracle/_ref, entry points ref_*particle* of oracle/ref_shim/ref_driver.cpp)
through the fixtures tests/golden/soft_*.npz.
"""
from __future__ import annotations

import math

import numpy as np

PI = 3.141592653589793238462643383279502884197  # include/defs.h:14
WCA_CUT = 1.122462048  # include/defs.h:17
POT = {"harmonic": 0, "lennardJones": 1, "adhesive": 2, "wca": 3}


class Drand48:
    """drand48() after srand48(seed)."""

    A, C, M = 0x5DEECE66D, 0xB, 1 << 48

    def __init__(self, seed: int):
        self.x = ((seed & 0xFFFFFFFF) << 16) | 0x330E

    def __call__(self) -> float:
        self.x = (self.A * self.x + self.C) % self.M
        return self.x / float(self.M)

    def take(self, n: int) -> np.ndarray:
        return np.array([self() for _ in range(n)])


def preferred_phi(nv_list, a0, rad, box) -> float:
    """DPM2D::getPreferredPhi (src/DPM2D.cu:1222-1238), kernelCalcVertexArea (:1636-1642)."""
    first = np.concatenate([[0], np.cumsum(nv_list)[:-1]]).astype(int)
    phi = 0.0
    for a in a0:  # sequential, as the reduction runs
        phi += float(a)
    va = 0.0
    for q, n in enumerate(nv_list):
        r = rad[first[q]]
        va += r * r * (0.5 * n - 1)
    phi += PI * va
    return phi / (box[0] * box[1])


def set_random_particles(nv_list, a0, l0, rad, box, phi0, extra_rad, seed):
    """Returns (a0, l0, rad, box, particle_pos, particle_rad) after the call."""
    scale = math.sqrt(preferred_phi(nv_list, a0, rad, box) / phi0)
    box = np.array([1.0, 1.0])
    a0 = np.array(a0, dtype=float)
    ppos = np.zeros(2 * len(nv_list))
    prad = np.zeros(len(nv_list))
    rnd = Drand48(seed)
    for q, n in enumerate(nv_list):
        a0[q] /= scale * scale
        for dim in range(2):
            ppos[2 * q + dim] = box[dim] * rnd()
        prad[q] = extra_rad * math.sqrt((2.0 * a0[q]) / (n * math.sin(2.0 * PI / n)))
    return a0, np.asarray(l0) / scale, np.asarray(rad) / scale, box, ppos, prad


def _pbc(d, L):
    return d - L * np.round(d / L)


def particle_neighbor_list(ppos, prad, box, cut_distance, list_size=0):
    """(rows [np][size] ascending, -1 padded; counts; size)."""
    n = len(prad)
    x = ppos.reshape(n, 2)
    rows = []
    for i in range(n):
        d = np.hypot(_pbc(x[i, 0] - x[:, 0], box[0]), _pbc(x[i, 1] - x[:, 1], box[1]))
        ok = -(1.0 - d / (prad[i] + prad[i])) < cut_distance
        ok[i] = False
        rows.append(np.nonzero(ok)[0])
    cnt = np.array([len(r) for r in rows], dtype=np.int64)
    mx = int(cnt.max()) if n else 0
    if mx > list_size:
        list_size = int(2 ** math.ceil(math.log2(mx)))
    out = np.full((n, list_size), -1, dtype=np.int64)
    for i, r in enumerate(rows):
        out[i, : len(r)] = r
    return out.reshape(-1), cnt, list_size


def _pair(pot, d, rsum, ec, lj_cutoff=2.5, l1=0.0, l2=0.0):
    """(gradMultiple, half-pair energy) of the reference pair functions, or None."""
    if pot == 0:
        ov = 1 - d / rsum
        if ov > 0:
            return ec * ov / rsum, (0.5 * ec * ov * ov) * 0.5
        return None
    if pot == 1:
        if d <= lj_cutoff * rsum:
            r6 = 1 / lj_cutoff ** 6
            ecut = 4 * ec * (r6 * r6 - r6)
            fshift = 24 * ec * (2 * r6 - 1) * r6 / lj_cutoff
            ratio = rsum / d
            a6 = ratio ** 6
            a12 = a6 * a6
            gm = 24 * ec * (2 * a12 - a6) / d - fshift / rsum
            return gm, 0.5 * (4 * ec * (a12 - a6) - ecut - abs(fshift / rsum) * (d - lj_cutoff * rsum))
        return None
    if pot == 2:
        if d < (1 + l2) * rsum:
            ov = 1 - d / rsum
            if d < (1 + l1) * rsum:
                return ec * ov / rsum, 0.5 * ec * (ov * ov - l1 * l2) * 0.5
            k = ec * l1 / (l2 - l1)
            return -k * (ov + l2) / rsum, -(0.5 * k * (ov + l2) ** 2) * 0.5
        return None
    if d <= WCA_CUT * rsum:
        ratio = rsum / d
        a6 = ratio ** 6
        a12 = a6 * a6
        return 24 * ec * (2 * a12 - a6) / d, 0.5 * ec * (4 * (a12 - a6) + 1)
    return None


def particle_force_energy(ppos, prad, box, rows, cnt, list_size, potential="harmonic", ec=1.0, **kw):
    """(force [2 np], energy [np]) over the list."""
    pot = POT[potential] if isinstance(potential, str) else int(potential)
    n = len(prad)
    x = ppos.reshape(n, 2)
    f = np.zeros((n, 2))
    e = np.zeros(n)
    for i in range(n):
        for k in range(cnt[i]):
            j = int(rows[i * list_size + k])
            dl = np.array([_pbc(x[i, 0] - x[j, 0], box[0]), _pbc(x[i, 1] - x[j, 1], box[1])])
            d = math.sqrt(dl[0] * dl[0] + dl[1] * dl[1])
            r = _pair(pot, d, prad[i] + prad[j], ec, **kw)
            if r is not None:
                f[i] += r[0] * dl / d
                e[i] += r[1]
    return f.reshape(-1), e


class ParticleFire:
    """The particle FIRE minimiser and its driver loop."""

    def __init__(self, ppos, prad, box, params, min_step=20, num_step=0, potential="harmonic", ec=1.0, **kw):
        self.x = np.array(ppos, dtype=float)
        self.r = np.asarray(prad, dtype=float)
        self.box = np.asarray(box, dtype=float)
        self.v = np.zeros_like(self.x)
        self.a_start, self.f_dec, self.f_inc, self.f_a, self.dt, self.dt_max, self.a = [float(p) for p in params]
        self.min_step, self.num_step = int(min_step), int(num_step)
        self.mass = np.repeat(PI / (self.r * self.r), 2)
        self.pot, self.ec, self.kw = potential, ec, kw
        self.last = self.x.copy()
        self.rows = self.cnt = None
        self.size = 0

    def build(self, cut):
        self.rows, self.cnt, self.size = particle_neighbor_list(self.x, self.r, self.box, cut, self.size)
        self.last = self.x.copy()

    def forces(self):
        self.f, self.e = particle_force_energy(self.x, self.r, self.box, self.rows, self.cnt, self.size,
                                               self.pot, self.ec, **self.kw)

    def loop(self, nsteps=1):
        n = len(self.r)
        for _ in range(nsteps):
            for q in range(n):
                total = 0.0
                for dim in range(2):
                    i = 2 * q + dim
                    self.v[i] += 0.5 * self.dt * self.f[i] / self.mass[i]
                    self.x[i] += self.dt * self.v[i]
                    total += self.f[i]
                if total == 0:
                    self.v[2 * q: 2 * q + 2] = 0
            self.forces()
            for q in range(n):
                total = 0.0
                for dim in range(2):
                    i = 2 * q + dim
                    self.v[i] += 0.5 * self.dt * self.f[i] / self.mass[i]
                    total += self.f[i]
                if total == 0:
                    self.v[2 * q: 2 * q + 2] = 0
            if float(np.dot(self.v, self.f)) < 0:
                self.v[:] = 0
                self.num_step = 0
                self.dt = max(self.dt * self.f_dec, self.dt_max / 10)
                self.a = self.a_start
            elif self.num_step > self.min_step:
                self.dt = min(self.dt * self.f_inc, self.dt_max)
                self.a *= self.f_a
            vv = float(np.dot(self.v, self.v))
            ff = float(np.dot(self.f, self.f))
            if ff == 0:
                self.v[:] = 0
            else:
                self.v = (1 - self.a) * self.v + self.a * self.f * math.sqrt(vv / ff)
            self.num_step += 1

    def max_force(self):
        return math.sqrt(float(np.max(self.f * self.f)))

    def max_displacement(self):
        n = len(self.r)
        d = (self.x - self.last).reshape(n, 2)
        return float(np.max(np.hypot(_pbc(d[:, 0], self.box[0]), _pbc(d[:, 1], self.box[1]))))

    def minimize(self, cut, tol, max_iterations):
        """compressFIRE.cpp:66-78; returns the iterations."""
        cutoff = (1 + cut) * min(1.0, float(self.r.min()))
        it = 0
        while self.max_force() > tol and it != max_iterations:
            self.loop(1)
            if 3 * self.max_displacement() > cutoff:
                self.build(cut)
            it += 1
        return it


def vertices_on_particles(nv_list, a0, l0, ppos, draws):
    """Vertex positions [2 nv] from the particle positions and 2 nv uniforms."""
    out = np.zeros(2 * int(np.sum(nv_list)))
    v = 0
    for q, n in enumerate(nv_list):
        rad = math.sqrt((2.0 * a0[q]) / (n * math.sin(2.0 * PI / n)))
        for _ in range(n):
            ang = (2.0 * PI * v) / n
            out[2 * v] = rad * math.cos(ang) + ppos[2 * q] + 1e-03 * l0[v] * draws[2 * v]
            out[2 * v + 1] = rad * math.sin(ang) + ppos[2 * q + 1] + 1e-03 * l0[v] * draws[2 * v + 1]
            v += 1
    return out
