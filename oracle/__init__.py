"""Python bindings for the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this package, and only as the checker.  Two native libraries back it:

* ``oracle/liboracle.so`` -- the plain-C restatement of the reference
  algorithm (``oracle/oracle.c``), built by ``make -C oracle``;
* ``oracle/_ref/libcrref.so`` -- the reference's own kernels compiled as host
  code (``oracle/build_ref.sh``), present when the reference checkout was
  available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

POTENTIALS = {"harmonic": 0, "lennardJones": 1, "adhesive": 2, "wca": 3}
INTERACTIONS = {"vertexVertex": 0, "vertexSmooth": 1, "cellSmooth": 2, "all": 3}
WCA_CUT = 1.122462048  # include/defs.h:17


class OcSys(C.Structure):
    _fields_ = [("np", C.c_long), ("nv", C.c_long),
                ("nv_list", C.c_void_p), ("first", C.c_void_p), ("pid", C.c_void_p),
                ("lx", C.c_double), ("ly", C.c_double),
                ("ea", C.c_double), ("el", C.c_double), ("eb", C.c_double), ("ec", C.c_double),
                ("l1", C.c_double), ("l2", C.c_double),
                ("lj_cutoff", C.c_double), ("lj_ecut", C.c_double), ("lj_fshift", C.c_double),
                ("stiff", C.c_double), ("ext_sq", C.c_double),
                ("potential", C.c_int), ("interaction", C.c_int), ("monomer", C.c_int)]


def reference_dir() -> str:
    """The reference checkout: $CUDARING_REFERENCE, else /root/reference."""
    return os.environ.get("CUDARING_REFERENCE", "/root/reference")


def build(quiet: bool = True) -> None:
    """Build liboracle.so (and _ref when the reference checkout exists)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, stdout=out)
    ref_src = reference_dir()
    if os.path.isdir(ref_src):
        subprocess.run([os.path.join(HERE, "build_ref.sh"), ref_src], check=True, stdout=out)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        sysp = C.POINTER(OcSys)
        L.oc_particle_shape.argtypes = [sysp, _dp, _dp, _dp, _dp, _dp]
        L.oc_particle_positions.argtypes = [sysp, _dp, _dp]
        L.oc_shape_force_energy.argtypes = [sysp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.oc_vertex_interaction.argtypes = [sysp, _dp, _dp, _lp, _lp, C.c_long, _dp, _dp]
        L.oc_smooth_interaction.argtypes = [sysp, _dp, _dp, _lp, _lp, C.c_long, _dp, _dp]
        L.oc_all_to_all_interaction.argtypes = [sysp, _dp, _dp, _dp, _dp]
        L.oc_neighbor_list.argtypes = [sysp, _dp, _dp, C.c_double, C.c_long, _lp, _lp]
        L.oc_neighbor_list.restype = C.c_long
        L.oc_check_displacement.argtypes = [sysp, _dp, _dp, C.c_double]
        L.oc_check_displacement.restype = C.c_int
        L.oc_calc_force_energy.argtypes = [sysp, _dp, _dp, _dp, _dp, _dp, _lp, _lp, C.c_long,
                                           _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.oc_rigid_force_energy.argtypes = [sysp, _dp, _dp, _lp, _lp, C.c_long, _dp, _dp, _dp, _dp,
                                            _dp, _dp, _dp, _dp]
        L.oc_translate_rotate.argtypes = [sysp, _dp, _dp, _dp, _dp, _dp]
        L.oc_normal2.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _dp]
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libcrref.so"))


def ref():
    """The reference kernels compiled as host code (raises if not built)."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libcrref.so")
        if not os.path.exists(path):
            raise FileNotFoundError("oracle/_ref/libcrref.so not built (needs the reference checkout)")
        R = C.CDLL(path)
        R.ref_create.argtypes = [C.c_long, _lp]
        R.ref_num_vertices.restype = C.c_long
        R.ref_set_box.argtypes = [C.c_double, C.c_double]
        R.ref_set_types.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
        R.ref_set_energy_costs.argtypes = [C.c_double] * 4
        R.ref_set_lj_cutoff.argtypes = [C.c_double]
        R.ref_get_lj_constants.argtypes = [_dp]
        R.ref_set_attraction.argtypes = [C.c_double, C.c_double]
        R.ref_set_fene.argtypes = [C.c_double, C.c_double]
        R.ref_set_time_step.argtypes = [C.c_double]
        R.ref_set_state.argtypes = [C.c_void_p] * 6
        R.ref_set_displacement_cutoff.argtypes = [C.c_double, C.c_double]
        R.ref_set_displacement_cutoff.restype = C.c_double
        R.ref_calc_neighbor_list.argtypes = [C.c_double]
        R.ref_update_count.restype = C.c_long
        R.ref_neighbor_list_size.restype = C.c_long
        R.ref_get_neighbors.argtypes = [_lp]
        R.ref_get_max_neighbor_list.argtypes = [_lp]
        R.ref_get.argtypes = [C.c_int, _dp]
        R.ref_set_particle_state.argtypes = [C.c_void_p] * 4
        for fn in ("ref_potential_energy", "ref_kinetic_energy", "ref_max_unbalanced_force",
                   "ref_total_force_magnitude", "ref_phi", "ref_preferred_phi"):
            getattr(R, fn).restype = C.c_double
        R.ref_nve_loop.argtypes = [C.c_long]
        R.ref_nve_rescale_loop.argtypes = [C.c_long, C.c_double]
        R.ref_langevin_loop.argtypes = [C.c_long, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_void_p]
        R.ref_brownian_loop.argtypes = [C.c_long, C.c_double, C.c_double, C.c_void_p, C.c_double, C.c_void_p]
        R.ref_baoab_loop.argtypes = [C.c_long, C.c_double, C.c_double, C.c_void_p]
        R.ref_fire_init.argtypes = [_dp, C.c_long, C.c_long]
        R.ref_fire_state.argtypes = [_dp]
        R.ref_fire_loop.argtypes = [C.c_long]
        R.ref_scale_vertices.argtypes = [C.c_double]
        R.ref_rigid_nve_loop.argtypes = [C.c_long]
        # soft-disk pre-packing
        R.ref_set_soft_particles.argtypes = [C.c_void_p, C.c_void_p]
        R.ref_get_particle_radii.argtypes = [_dp]
        R.ref_get_geometry.argtypes = [_dp]
        R.ref_calc_particle_neighbor_list.argtypes = [C.c_double]
        R.ref_particle_neighbor_list_size.restype = C.c_long
        R.ref_get_particle_neighbors.argtypes = [_lp]
        R.ref_get_particle_max_neighbor_list.argtypes = [_lp]
        for fn in ("ref_particle_max_unbalanced_force", "ref_particle_potential_energy",
                   "ref_particle_max_displacement"):
            getattr(R, fn).restype = C.c_double
        R.ref_particle_fire_init.argtypes = [_dp, C.c_long, C.c_long]
        R.ref_particle_fire_loop.argtypes = [C.c_long]
        R.ref_particle_fire_minimize.argtypes = [C.c_double, C.c_double, C.c_long]
        R.ref_particle_fire_minimize.restype = C.c_long
        R.ref_init_vertices_on_particles.argtypes = [_dp]
        R.ref_set_random_particles.argtypes = [C.c_double, C.c_double, C.c_long]
        R.ref_drand48_stream.argtypes = [C.c_long, C.c_long, C.c_long, _dp]
        _REF = R
    return _REF


def _ptr(a):
    return None if a is None else a.ctypes.data


def lj_constants(lj_cutoff: float, ec: float) -> tuple[float, float]:
    """LJecut and LJfshift as DPM2D::setLJcutoff computes them (src/DPM2D.cu:1923-1932)."""
    ratio6 = 1.0 / lj_cutoff ** 6
    return 4 * ec * (ratio6 * ratio6 - ratio6), 24 * ec * (2 * ratio6 - 1) * ratio6 / lj_cutoff


class System:
    """Host-array model driven by the C restatement (oracle.c)."""

    def __init__(self, nv_list, box, potential="harmonic", interaction="vertexVertex",
                 ea=1.0, el=1.0, eb=0.01, ec=1.0, l1=0.0, l2=0.0, lj_cutoff=2.5, monomer=0,
                 stiff=0.0, ext=0.0):
        self.nv_list = np.ascontiguousarray(nv_list, dtype=np.int64)
        self.np = int(self.nv_list.shape[0])
        self.nv = int(self.nv_list.sum())
        self.first = np.concatenate([[0], np.cumsum(self.nv_list)[:-1]]).astype(np.int64)
        self.pid = np.repeat(np.arange(self.np, dtype=np.int64), self.nv_list)
        ecut, fshift = lj_constants(lj_cutoff, ec)
        self.s = OcSys(self.np, self.nv, self.nv_list.ctypes.data, self.first.ctypes.data,
                       self.pid.ctypes.data, float(box[0]), float(box[1]), ea, el, eb, ec, l1, l2,
                       lj_cutoff, ecut, fshift, stiff, ext * ext, POTENTIALS[potential],
                       INTERACTIONS[interaction], monomer)
        self.list_size = 0
        self.nbr = np.full(self.nv, -1, dtype=np.int64)
        self.cnt = np.zeros(self.nv, dtype=np.int64)

    def cut_distance(self, cutoff_: float) -> float:
        """DPM2D::setDisplacementCutoff's cutDistance (src/DPM2D.cu:1300-1316)."""
        pot = self.s.potential
        base = {0: 1.0, 1: self.s.lj_cutoff, 3: WCA_CUT, 2: 1.0 + self.s.l2}[pot]
        return base + cutoff_

    def neighbor_list(self, pos, rad, cut_distance):
        """DPM2D::calcNeighborList (src/DPM2D.cu:3479-3507)."""
        L = lib()
        self.cnt[:] = 0
        self.nbr[:] = -1
        mx = L.oc_neighbor_list(C.byref(self.s), pos, rad, cut_distance, self.list_size, self.nbr, self.cnt)
        if mx > self.list_size:
            self.list_size = int(2 ** np.ceil(np.log2(mx)))
            self.nbr = np.full(self.nv * self.list_size, -1, dtype=np.int64)
            L.oc_neighbor_list(C.byref(self.s), pos, rad, cut_distance, self.list_size, self.nbr, self.cnt)
        return self.nbr, self.cnt, self.list_size

    def force_energy(self, pos, rad, a0, l0, theta0):
        L = lib()
        out = dict(force=np.zeros(2 * self.nv), energy=np.zeros(self.nv), p_energy=np.zeros(self.np),
                   length=np.zeros(self.nv), theta=np.zeros(self.nv), area=np.zeros(self.np),
                   perimeter=np.zeros(self.np), ppos=np.zeros(2 * self.np))
        L.oc_calc_force_energy(C.byref(self.s), pos, rad, a0, l0, theta0, self.nbr, self.cnt,
                               self.list_size, out["force"], out["energy"], out["p_energy"],
                               out["length"], out["theta"], out["area"], out["perimeter"], out["ppos"])
        pe = out["energy"].sum()
        if self.s.interaction in (1, 2):
            pe += out["p_energy"].sum()
        out["potential_energy"] = pe
        return out

    def rigid_force_energy(self, pos, rad):
        L = lib()
        out = {k: np.zeros(n) for k, n in (("ppos", 2 * self.np), ("force", 2 * self.nv), ("torque", self.nv),
                                            ("energy", self.nv), ("moi", self.np), ("p_force", 2 * self.np),
                                            ("p_torque", self.np), ("p_energy", self.np))}
        L.oc_rigid_force_energy(C.byref(self.s), pos, rad, self.nbr, self.cnt, self.list_size, out["ppos"],
                                out["force"], out["torque"], out["energy"], out["moi"], out["p_force"],
                                out["p_torque"], out["p_energy"])
        return out


def packing_fraction(nv_list, rad, ring_area, box) -> float:
    """DPM2D::getPhi / getPreferredPhi for the periodic box (src/DPM2D.cu:1202-1238):
    ring areas (current or rest) plus pi * r_first^2 * (nv / 2 - 1) per ring
    (kernelCalcVertexArea, include/cudaKernel.cuh:1636-1642), over the box area.
    Ring terms are summed in ring order, as the reference's reduce does on the host."""
    nv_list = np.asarray(nv_list, dtype=np.int64)
    first = np.concatenate([[0], np.cumsum(nv_list)[:-1]])
    r = np.asarray(rad, dtype=np.float64)[first]
    s = 0.0
    for a in np.asarray(ring_area, dtype=np.float64):
        s += float(a)
    v = 0.0
    for rr, n in zip(r, nv_list):
        v += float(rr * rr * (0.5 * n - 1))
    return (s + np.pi * v) / (float(box[0]) * float(box[1]))


def normal2(seed: int, stream: int, index: int) -> np.ndarray:
    out = np.zeros(2)
    lib().oc_normal2(seed, stream, index, out)
    return out
