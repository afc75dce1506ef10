"""``Batch``: many independent deformable-ring systems advanced together.

Wraps the ``cr_batch_*`` entry points of include/cudaring.h.  A batch holds
S systems, each with its own periodic box, ring count and packing fraction;
arrays are the single-system layout concatenated over systems (system s's
rings and vertices follow system s-1's).  Every op is one launch over all
systems; each system has its own neighbour list, FIRE scalars and flags.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import CudaRingError, lib
from .dpm2d import simControl


class CompressParams(C.Structure):
    """``cr_compress_params`` (include/cudaring.h)."""

    _fields_ = [("dphi", C.c_double), ("min_dphi", C.c_double), ("fire_dt", C.c_double), ("tol0", C.c_double),
                ("energy_tol", C.c_double), ("max_fire_iters", C.c_long), ("max_steps", C.c_long),
                ("criterion", C.c_int)]


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Batch:
    def __init__(self, num_particles, nv_lists):
        """``num_particles[s]`` rings in system s; ``nv_lists[s]`` their vertex counts."""
        self._L = lib()
        self.num_particles = np.asarray(num_particles, dtype=np.int64)
        nvl = np.concatenate([np.asarray(x, dtype=np.int64) for x in nv_lists])
        assert len(nvl) == int(self.num_particles.sum())
        h = C.c_void_p()
        rc = self._L.cr_batch_create(len(self.num_particles), self.num_particles.ctypes.data, nvl.ctypes.data,
                                     C.byref(h))
        if rc != 0:
            raise CudaRingError("cr_batch_create", rc, "batch creation failed")
        self._h = h
        self.nv_list = nvl
        self.S = len(self.num_particles)
        self.np = int(nvl.size)
        self.nv = int(nvl.sum())
        self.num_vertices = np.array([int(np.sum(x)) for x in nv_lists], dtype=np.int64)
        self.vertex_offsets = np.concatenate([[0], np.cumsum(self.num_vertices)])
        self.ring_offsets = np.concatenate([[0], np.cumsum(self.num_particles)])

    # ------------------------------------------------------------ plumbing
    def _call(self, name, *args):
        rc = getattr(self._L, name)(self._h, *args)
        if rc != 0:
            msg = self._L.cr_batch_last_error(self._h)
            raise CudaRingError(name, rc, msg.decode() if msg else "")

    def _get(self, name, n, dtype=np.float64):
        out = np.empty(n, dtype=dtype)
        self._call(name, out.ctypes.data)
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._L.cr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------- parameters
    def setPotentialType(self, v): self._call("cr_batch_set_potential_type", int(v))
    def setInteractionType(self, v): self._call("cr_batch_set_interaction_type", int(v))
    def setEnergyCosts(self, ea, el, eb, ec): self._call("cr_batch_set_energy_costs", ea, el, eb, ec)
    def setLJcutoff(self, c): self._call("cr_batch_set_lj_cutoff", c)
    def setAttractionConstants(self, l1, l2): self._call("cr_batch_set_attraction_constants", l1, l2)

    def setPrecision(self, precision):
        self._call("cr_batch_set_precision", int({"fp64": 0, "mixed": 1}.get(precision, precision)))

    def setLanes(self, lanes): self._call("cr_batch_set_lanes", int(lanes))

    def getLanes(self):
        out = C.c_int()
        self._call("cr_batch_get_lanes", C.byref(out))
        return out.value

    def setTileShape(self, lanes, block):
        self._call("cr_batch_set_tile_shape", int(lanes), int(block))

    def getTileShape(self):
        lanes, block = C.c_int(), C.c_int()
        self._call("cr_batch_get_tile_shape", C.byref(lanes), C.byref(block))
        return lanes.value, block.value

    def autotune(self, reps=20):
        """Times the batched FIRE force kernel for every tile shape whose tile
        holds the longest ring and keeps the fastest; returns its lane count
        (getTileShape gives the shape)."""
        out = C.c_int()
        self._call("cr_batch_autotune", int(reps), C.byref(out))
        return out.value

    def profileFireTile(self, reps=20):
        out = C.c_double()
        self._call("cr_batch_profile_fire_tile", int(reps), C.byref(out))
        return out.value

    def setBoxSizes(self, boxes): self._call("cr_batch_set_box_sizes", _f64(boxes).ctypes.data)
    def getBoxSizes(self): return self._get("cr_batch_get_box_sizes", 2 * self.S).reshape(self.S, 2)

    # ---------------------------------------------------------------- state
    def setVertexPositions(self, a): self._call("cr_batch_set_vertex_positions", _f64(a).ctypes.data)
    def getVertexPositions(self): return self._get("cr_batch_get_vertex_positions", 2 * self.nv)
    def setVertexVelocities(self, a): self._call("cr_batch_set_vertex_velocities", _f64(a).ctypes.data)
    def getVertexVelocities(self): return self._get("cr_batch_get_vertex_velocities", 2 * self.nv)
    def getVertexForces(self): return self._get("cr_batch_get_vertex_forces", 2 * self.nv)
    def getVertexEnergies(self): return self._get("cr_batch_get_vertex_energies", self.nv)
    def setVertexRadii(self, a): self._call("cr_batch_set_vertex_radii", _f64(a).ctypes.data)
    def getVertexRadii(self): return self._get("cr_batch_get_vertex_radii", self.nv)
    def setRestAreas(self, a): self._call("cr_batch_set_rest_areas", _f64(a).ctypes.data)
    def getRestAreas(self): return self._get("cr_batch_get_rest_areas", self.np)
    def setRestLengths(self, a): self._call("cr_batch_set_rest_lengths", _f64(a).ctypes.data)
    def getRestLengths(self): return self._get("cr_batch_get_rest_lengths", self.nv)
    def setRestAngles(self, a): self._call("cr_batch_set_rest_angles", _f64(a).ctypes.data)

    def setActive(self, active):
        a = np.ascontiguousarray(active, dtype=np.int32)
        self._call("cr_batch_set_active", a.ctypes.data)

    # ------------------------------------------------------ forces and FIRE
    def setDisplacementCutoff(self, cutoff):
        out = C.c_double()
        self._call("cr_batch_set_displacement_cutoff", cutoff, C.byref(out))
        return out.value

    def calcNeighborLists(self): self._call("cr_batch_calc_neighbor_lists")
    def calcForceEnergy(self): self._call("cr_batch_calc_force_energy")
    def getPotentialEnergies(self): return self._get("cr_batch_get_potential_energies", self.S)
    def getMaxUnbalancedForces(self): return self._get("cr_batch_get_max_unbalanced_forces", self.S)
    def getPhis(self): return self._get("cr_batch_get_phis", self.S)
    def getPreferredPhis(self): return self._get("cr_batch_get_preferred_phis", self.S)
    def getMeanParticleSizes(self): return self._get("cr_batch_get_mean_particle_sizes", self.S)

    def initFIRE(self, params, minStep, dt=None):
        self._call("cr_batch_init_fire", _f64(params).ctypes.data, None if dt is None else _f64(dt).ctypes.data,
                   int(minStep))

    def fireMinimize(self, tol, maxIter):
        tol = _f64(np.broadcast_to(np.asarray(tol, dtype=float), (self.S,)))
        its = np.zeros(self.S, dtype=np.int64)
        fmax = np.zeros(self.S)
        self._call("cr_batch_fire_minimize", tol.ctypes.data, int(maxIter), its.ctypes.data, fmax.ctypes.data)
        return its, fmax

    def scaleVertices(self, scale):
        self._call("cr_batch_scale_vertices", _f64(np.broadcast_to(scale, (self.S,))).ctypes.data)

    def compress(self, dphi=1e-3, min_dphi=1e-6, fire_dt=1e-2, tol0=1e-10, energy_tol=1e-20, max_fire_iters=100000,
                 max_steps=1000, criterion="force", stepwise=False):
        """Quasi-static compression to jamming of every system: the whole
        protocol on the device as one graph launch (cr_batch_compress), or,
        with stepwise=True, driven from the host between steps and FIRE
        chunks (cr_batch_compress_stepwise); both give the same states."""
        prm = CompressParams(dphi, min_dphi, fire_dt, tol0, energy_tol, int(max_fire_iters), int(max_steps),
                             {"force": 0, "energy": 1}[criterion])
        phi = np.zeros(self.S)
        steps = np.zeros(self.S, dtype=np.int64)
        state = np.zeros(self.S, dtype=np.int32)
        iters = np.zeros(self.S, dtype=np.int64)
        fn = "cr_batch_compress_stepwise" if stepwise else "cr_batch_compress"
        self._call(fn, C.byref(prm), phi.ctypes.data, steps.ctypes.data, state.ctypes.data, iters.ctypes.data)
        return {"phi": phi, "steps": steps, "state": state, "fire_iterations": iters}

    def setPersistent(self, on):
        """Persistent FIRE kernel for batches that fit the GPU at once (default on)."""
        self._call("cr_batch_set_persistent", int(bool(on)))

    def getListCapacity(self):
        out = C.c_int()
        self._call("cr_batch_get_list_capacity", C.byref(out))
        return out.value

    def getLaunchCount(self):
        out = C.c_longlong()
        self._call("cr_batch_get_launch_count", C.byref(out))
        return out.value

    # ------------------------------------------------------------- helpers
    def system_slice(self, s, per="vertex", dim=2):
        off = self.vertex_offsets if per == "vertex" else self.ring_offsets
        return slice(dim * int(off[s]), dim * int(off[s + 1]))

    @classmethod
    def from_packings(cls, packings, potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01,
                      ec=1.0, LJcutoff=2.5, l1=0.0, l2=0.0):
        b = cls([p.num_particles for p in packings], [p.nv_list for p in packings])
        b.setPotentialType(getattr(simControl.potentialEnum, potential))
        b.setInteractionType(getattr(simControl.interactionEnum, interaction))
        b.setEnergyCosts(ea, el, eb, ec)
        b.setLJcutoff(LJcutoff)
        b.setAttractionConstants(l1, l2)
        b.setBoxSizes(np.concatenate([p.box for p in packings]))
        b.setVertexRadii(np.concatenate([p.rad for p in packings]))
        b.setRestAreas(np.concatenate([p.a0 for p in packings]))
        b.setRestLengths(np.concatenate([p.l0 for p in packings]))
        b.setRestAngles(np.concatenate([p.theta0 for p in packings]))
        b.setVertexPositions(np.concatenate([p.pos for p in packings]))
        b.setVertexVelocities(np.concatenate([p.vel for p in packings]))
        return b
