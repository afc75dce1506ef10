"""``DPM2D``: the reference's model API (include/DPM2D.h) over libcudaring.

Method names, argument meaning and units follow farceri/cudaRing's ``DPM2D``
class so code written against it reads the same; every call goes through the
C ABI in include/cudaring.h.  Host arrays are numpy float64 / int64 in the
reference's layout (AoS ``[x0, y0, x1, y1, ...]``).  Loop methods take an
optional step count (the reference advances one step per call).

Errors raise :class:`CudaRingError` with the library's status and message
(the reference prints and carries on; a drop-in that silently continues on a
bad size would hide the same bugs).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import CudaRingError, lib


class simControl:
    """simControlStruct enums (include/DPM2D.h:22-32)."""

    class potentialEnum:
        harmonic, lennardJones, adhesive, wca = 0, 1, 2, 3

    class interactionEnum:
        vertexVertex, vertexSmooth, cellSmooth, all = 0, 1, 2, 3

    class monomerEnum:
        harmonic, FENE = 0, 1

    class particleEnum:
        passive, active, activeShape = 0, 1, 2

    class noiseEnum:
        langevin, baoab, brownian, drivenBrownian = 0, 1, 2, 3

    class shapeEnum:
        deformable, rigid = 0, 1

    class geometryEnum:
        normal, fixedBox, fixedSides, roundBox = 0, 1, 2, 3


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class DPM2D:
    """One periodic 2-D system of ring polymers on the current CUDA device."""

    def __init__(self, numVertexInParticleList):
        self._L = lib()
        nvl = np.ascontiguousarray(numVertexInParticleList, dtype=np.int64)
        h = C.c_void_p()
        rc = self._L.cr_create(len(nvl), nvl.ctypes.data, C.byref(h))
        if rc != 0:
            raise CudaRingError("cr_create", rc, "context creation failed")
        self._h = h
        self.numVertexInParticleList = nvl
        self.numParticles = int(len(nvl))
        self.numVertices = int(nvl.sum())

    # ------------------------------------------------------------ plumbing
    def _call(self, name, *args):
        rc = getattr(self._L, name)(self._h, *args)
        if rc != 0:
            msg = self._L.cr_last_error(self._h)
            raise CudaRingError(name, rc, msg.decode() if msg else "")

    def _get(self, name, n, dtype=np.float64, out=None):
        """Download into a new array, or into `out` (n contiguous elements of
        dtype, e.g. a pinned buffer: the copy then needs no staging)."""
        if out is None:
            out = np.empty(n, dtype=dtype)
        elif out.dtype != dtype or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous {np.dtype(dtype).name} array of {n} elements")
        self._call(name, out.ctypes.data)
        return out

    def _scalar(self, name):
        out = C.c_double()
        self._call(name, C.byref(out))
        return out.value

    def close(self):
        if getattr(self, "_h", None):
            self._L.cr_destroy(self._h)
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

    # -------------------------------------------------------------- switches
    def setPotentialType(self, v): self._call("cr_set_potential_type", int(v))
    def setInteractionType(self, v): self._call("cr_set_interaction_type", int(v))
    def setMonomerType(self, v): self._call("cr_set_monomer_type", int(v))
    def setParticleType(self, v): self._call("cr_set_particle_type", int(v))
    def setNoiseType(self, v): self._call("cr_set_noise_type", int(v))
    def setShapeType(self, v): self._call("cr_set_shape_type", int(v))
    def setGeometryType(self, v): self._call("cr_set_geometry_type", int(v))

    # ------------------------------------------------------------ parameters
    def setBoxSize(self, box): self._call("cr_set_box_size", _f64(box).ctypes.data)
    def getBoxSize(self): return self._get("cr_get_box_size", 2)
    def setEnergyCosts(self, ea, el, eb, ec): self._call("cr_set_energy_costs", ea, el, eb, ec)
    def setLJcutoff(self, c): self._call("cr_set_lj_cutoff", c)
    def setAttractionConstants(self, l1, l2): self._call("cr_set_attraction_constants", l1, l2)
    def setFENEconstants(self, stiff, ext): self._call("cr_set_fene_constants", stiff, ext)

    def setTimeStep(self, dt):
        self._call("cr_set_time_step", dt)
        return dt

    def setSelfPropulsionParams(self, driving, taup): self._call("cr_set_self_propulsion_params", driving, taup)
    def setSeed(self, seed): self._call("cr_set_seed", C.c_ulonglong(seed))

    # ----------------------------------------------------------------- state
    def setVertexPositions(self, a): self._call("cr_set_vertex_positions", _f64(a).ctypes.data)
    def getVertexPositions(self, out=None): return self._get("cr_get_vertex_positions", 2 * self.numVertices, out=out)
    def setVertexVelocities(self, a): self._call("cr_set_vertex_velocities", _f64(a).ctypes.data)
    def getVertexVelocities(self, out=None):
        return self._get("cr_get_vertex_velocities", 2 * self.numVertices, out=out)
    def setVertexForces(self, a): self._call("cr_set_vertex_forces", _f64(a).ctypes.data)
    def getVertexForces(self, out=None): return self._get("cr_get_vertex_forces", 2 * self.numVertices, out=out)
    def getVertexEnergies(self): return self._get("cr_get_vertex_energies", self.numVertices)
    def getParticleEnergies(self): return self._get("cr_get_particle_energies", self.numParticles)
    def setVertexRadii(self, a): self._call("cr_set_vertex_radii", _f64(a).ctypes.data)
    def getVertexRadii(self): return self._get("cr_get_vertex_radii", self.numVertices)
    def setRestAreas(self, a): self._call("cr_set_rest_areas", _f64(a).ctypes.data)
    def getRestAreas(self): return self._get("cr_get_rest_areas", self.numParticles)
    def setRestLengths(self, a): self._call("cr_set_rest_lengths", _f64(a).ctypes.data)
    def getRestLengths(self): return self._get("cr_get_rest_lengths", self.numVertices)
    def setRestAngles(self, a): self._call("cr_set_rest_angles", _f64(a).ctypes.data)
    def getRestAngles(self): return self._get("cr_get_rest_angles", self.numVertices)
    def getAreas(self): return self._get("cr_get_areas", self.numParticles)
    def getPerimeters(self): return self._get("cr_get_perimeters", self.numParticles)
    def getSegmentLengths(self): return self._get("cr_get_segment_lengths", self.numVertices)
    def getSegmentAngles(self): return self._get("cr_get_segment_angles", self.numVertices)
    def calcParticleShape(self): self._call("cr_calc_particle_shape")
    def calcParticlePositions(self): self._call("cr_calc_particle_positions")
    def getParticlePositions(self): return self._get("cr_get_particle_positions", 2 * self.numParticles)
    def setParticlePositions(self, a): self._call("cr_set_particle_positions", _f64(a).ctypes.data)

    # ------------------------------------------------------------ neighbours
    def setDisplacementCutoff(self, cutoff, size):
        out = C.c_double()
        self._call("cr_set_displacement_cutoff", cutoff, size, C.byref(out))
        return out.value

    def calcNeighborList(self, cutDistance): self._call("cr_calc_neighbor_list", cutDistance)
    calcNeighbors = calcNeighborList
    def checkNeighbors(self): self._call("cr_check_neighbors")
    def resetLastPositions(self): self._call("cr_reset_last_positions")

    def getNeighborListSize(self):
        out = C.c_long()
        self._call("cr_get_neighbor_list_size", C.byref(out))
        return out.value

    def getNeighbors(self):
        return self._get("cr_get_neighbors", self.numVertices * self.getNeighborListSize(), np.int64)

    def getMaxNeighborList(self): return self._get("cr_get_max_neighbor_list", self.numVertices, np.int64)

    def getUpdateCount(self):
        out = C.c_long()
        self._call("cr_get_update_count", C.byref(out))
        return out.value

    def resetUpdateCount(self): self._call("cr_reset_update_count")

    # ---------------------------------------------------- forces, reductions
    def calcForceEnergy(self): self._call("cr_calc_force_energy")
    def getPotentialEnergy(self): return self._scalar("cr_get_potential_energy")
    def getKineticEnergy(self): return self._scalar("cr_get_kinetic_energy")
    def getEnergy(self): return self._scalar("cr_get_energy")
    def getTemperature(self): return self._scalar("cr_get_temperature")
    def getMaxUnbalancedForce(self): return self._scalar("cr_get_max_unbalanced_force")
    def getTotalForceMagnitude(self): return self._scalar("cr_get_total_force_magnitude")
    def getPhi(self): return self._scalar("cr_get_phi")
    def getPreferredPhi(self): return self._scalar("cr_get_preferred_phi")
    def getMeanVertexRadius(self): return self._scalar("cr_get_mean_vertex_radius")
    def getMeanParticleSize(self): return self._scalar("cr_get_mean_particle_size")
    def scaleVertices(self, scale): self._call("cr_scale_vertices", scale)

    # ------------------------------------------------------------ integrators
    def initNVE(self, T, readState=False): self._call("cr_init_nve", T, int(bool(readState)))
    def NVELoop(self, nsteps=1): self._call("cr_nve_loop", int(nsteps))
    def initNVERescale(self, T): self._call("cr_init_nve_rescale", T)
    def NVERescaleLoop(self, nsteps=1): self._call("cr_nve_rescale_loop", int(nsteps))
    def conserveMomentum(self): self._call("cr_conserve_momentum")
    def initLangevin(self, T, gamma, readState=False): self._call("cr_init_langevin", T, gamma, int(bool(readState)))
    def langevinLoop(self, nsteps=1): self._call("cr_langevin_loop", int(nsteps))

    def initFIRE(self, FIREparams, minStep, numStep, numDOF):
        self._call("cr_init_fire", _f64(FIREparams).ctypes.data, int(minStep), int(numStep), int(numDOF))

    def vertexFIRELoop(self, nsteps=1): self._call("cr_vertex_fire_loop", int(nsteps))

    def minimizeFIRE(self, tol, maxIter):
        it, f = C.c_long(), C.c_double()
        self._call("cr_fire_minimize", tol, int(maxIter), C.byref(it), C.byref(f))
        return it.value, f.value

    def getFIREState(self): return self._get("cr_get_fire_state", 3)

    # ------------------------------------------------------------ derivatives
    def hvp(self, v):
        """Hessian-vector product of the potential energy at the current positions."""
        out = np.empty(2 * self.numVertices)
        self._call("cr_hvp", _f64(v).ctypes.data, out.ctypes.data)
        return out

    def hvpDevice(self, v_ptr, hv_ptr):
        """cr_hvp_device: v and hv are device pointers (e.g. torch tensors' data_ptr())."""
        self._call("cr_hvp_device", C.c_void_p(v_ptr), C.c_void_p(hv_ptr))

    def calcPressure(self): return self._scalar("cr_calc_pressure")

    PARAMS = {"ea": 0, "el": 1, "eb": 2, "lnCalA0": 3}

    def paramDerivatives(self, param):
        """(dU, dP, dF, dP/dx) along one parameter at fixed positions."""
        dU, dP = C.c_double(), C.c_double()
        dF = np.empty(2 * self.numVertices)
        dPdx = np.empty(2 * self.numVertices)
        self._call("cr_param_derivatives", int(self.PARAMS.get(param, param)), C.byref(dU), C.byref(dP),
                   dF.ctypes.data, dPdx.ctypes.data)
        return dU.value, dP.value, dF, dPdx

    def hessianDiagBlocks(self):
        """(Nv, 3) array of the Hessian's 2 x 2 vertex blocks (xx, xy, yy)."""
        out = np.empty(3 * self.numVertices)
        self._call("cr_hessian_diag_blocks", out.ctypes.data)
        return out.reshape(-1, 3)

    def setCGPreconditioner(self, kind):
        """Preconditioner of hessianSolve: "block_jacobi" (default) or "none"."""
        self._call("cr_set_cg_preconditioner", {"none": 0, "block_jacobi": 1}.get(kind, kind))

    def hessianSolve(self, b, tol=1e-10, maxIter=100000):
        x = np.empty(2 * self.numVertices)
        it, rr = C.c_long(), C.c_double()
        self._call("cr_hessian_solve", _f64(b).ctypes.data, x.ctypes.data, float(tol), int(maxIter), C.byref(it),
                   C.byref(rr))
        return x, it.value, rr.value

    # ------------------------------------------------------------ rigid rings
    def calcRigidForceEnergy(self): self._call("cr_calc_rigid_force_energy")
    def initRigidNVE(self, T, readState=False): self._call("cr_init_rigid_nve", T, int(bool(readState)))
    def rigidNVELoop(self, nsteps=1): self._call("cr_rigid_nve_loop", int(nsteps))

    def initRigidLangevin(self, T, gamma, readState=False):
        self._call("cr_init_rigid_langevin", T, gamma, int(bool(readState)))

    def rigidLangevinLoop(self, nsteps=1): self._call("cr_rigid_langevin_loop", int(nsteps))
    def getParticleVelocities(self): return self._get("cr_get_particle_velocities", 2 * self.numParticles)
    def setParticleVelocities(self, a): self._call("cr_set_particle_velocities", _f64(a).ctypes.data)
    def getParticleAngles(self): return self._get("cr_get_particle_angles", self.numParticles)
    def setParticleAngles(self, a): self._call("cr_set_particle_angles", _f64(a).ctypes.data)

    def getParticleAngularVelocities(self):
        return self._get("cr_get_particle_angular_velocities", self.numParticles)

    def setParticleAngularVelocities(self, a):
        self._call("cr_set_particle_angular_velocities", _f64(a).ctypes.data)

    def getParticleForces(self): return self._get("cr_get_particle_forces", 2 * self.numParticles)
    def getParticleTorques(self): return self._get("cr_get_particle_torques", self.numParticles)
    def getVertexTorques(self): return self._get("cr_get_vertex_torques", self.numVertices)
    def getParticleKineticEnergy(self): return self._scalar("cr_get_particle_kinetic_energy")

    # ------------------------------------------- soft-disk pre-packing
    # The particle-level stage of compressFIRE.cpp:53-90: soft disks at the
    # particle positions, FIRE on the disks, vertices placed on the circles.
    def setParticleRadii(self, a): self._call("cr_set_particle_radii", _f64(a).ctypes.data)
    def getParticleRadii(self): return self._get("cr_get_particle_radii", self.numParticles)
    def getMeanParticleSigma(self): return self._scalar("cr_get_mean_particle_sigma")
    def getMinParticleSigma(self): return self._scalar("cr_get_min_particle_sigma")

    def setRandomParticles(self, phi0, extraRad, seed):
        """DPM2D::setRandomParticles (src/DPM2D.cu:1601-1629) on the drand48()
        stream that srand48(seed) starts."""
        self._call("cr_set_random_particles", float(phi0), float(extraRad), int(seed))

    def calcParticleNeighborList(self, cutDistance): self._call("cr_calc_particle_neighbor_list", float(cutDistance))

    def getParticleNeighborListSize(self):
        out = C.c_long()
        self._call("cr_get_particle_neighbor_list_size", C.byref(out))
        return out.value

    def getParticleNeighbors(self):
        return self._get("cr_get_particle_neighbors", self.numParticles * self.getParticleNeighborListSize(), np.int64)

    def getParticleMaxNeighborList(self):
        return self._get("cr_get_particle_max_neighbor_list", self.numParticles, np.int64)

    def calcParticleForceEnergy(self): self._call("cr_calc_particle_force_energy")
    def getParticlePotentialEnergy(self): return self._scalar("cr_get_particle_potential_energy")
    def getParticleMaxUnbalancedForce(self): return self._scalar("cr_get_particle_max_unbalanced_force")
    def resetParticleLastPositions(self): self._call("cr_reset_particle_last_positions")
    def getParticleMaxDisplacement(self): return self._scalar("cr_get_particle_max_displacement")

    def initParticleFIRE(self, params, minStep=20, numStep=0):
        """DPM2D::initFIRE + setParticleMassFIRE: params = [a_start, f_dec,
        f_inc, f_a, dt, dt_max, a]."""
        p = _f64(params)
        if p.size != 7:
            raise ValueError("FIRE takes 7 parameters")
        self._call("cr_init_particle_fire", p.ctypes.data, int(minStep), int(numStep))

    def getParticleFIREState(self):
        """(dt, a, numStep) of the particle minimiser."""
        out = self._get("cr_get_particle_fire_state", 3)
        return float(out[0]), float(out[1]), int(out[2])

    def particleFIRELoop(self, nsteps=1): self._call("cr_particle_fire_loop", int(nsteps))

    def particleFIREMinimize(self, cutDistance, tol, maxIterations):
        """The driver loop of compressFIRE.cpp:66-78; returns the iterations."""
        out = C.c_long()
        self._call("cr_particle_fire_minimize", float(cutDistance), float(tol), int(maxIterations), C.byref(out))
        return out.value

    def initVerticesOnParticles(self, draws=None):
        """DPM2D::initVerticesOnParticles; draws: 2 nv uniforms in the
        reference's drand48() call order, or None for the context's stream."""
        if draws is None:
            self._call("cr_init_vertices_on_particles", None)
        else:
            d = _f64(draws)
            if d.size != 2 * self.numVertices:
                raise ValueError("draws must hold 2 * numVertices values")
            self._call("cr_init_vertices_on_particles", d.ctypes.data)

    def softPrepack(self, phi0, extraRad=1.1, seed=1, dt=1e-2, minStep=20, cutDistance=1.0, tol0=1e-10,
                    maxIterations=5000000, draws=None):
        """compressFIRE.cpp:53-86 from setRandomParticles to
        initVerticesOnParticles: random soft disks at phi0, particle FIRE to
        max |F| < tol0 / meanParticleSigma, vertices on the disk circles.
        Returns the FIRE iterations."""
        self.setRandomParticles(phi0, extraRad, seed)
        sigma = self.getMeanParticleSize()
        step = 10 * dt * sigma
        self.setTimeStep(step)
        self.initParticleFIRE([0.2, 0.5, 1.1, 0.99, step, 10 * step, 0.2], minStep, 0)
        self.calcParticleNeighborList(cutDistance)
        self.calcParticleForceEnergy()
        self.resetParticleLastPositions()
        tol = tol0 / self.getMeanParticleSigma()
        it = self.particleFIREMinimize(cutDistance, tol, maxIterations)
        self.initVerticesOnParticles(draws)
        return it

    def setLanes(self, lanes): self._call("cr_set_lanes", int(lanes))

    def getLanes(self):
        out = C.c_int()
        self._call("cr_get_lanes", C.byref(out))
        return out.value

    def setUseGraphs(self, on): self._call("cr_set_use_graphs", int(bool(on)))

    def setMultistep(self, on): self._call("cr_set_multistep", int(bool(on)))

    def setSpinLimit(self, polls):
        """Polls a grid-barrier wait makes before giving up (0: the default 2^20;
        negative: the first poll that finds a barrier incomplete gives up)."""
        self._call("cr_set_spin_limit", C.c_longlong(int(polls)))

    def getDegraded(self):
        """True once a grid-barrier wait gave up and the context runs one launch per op."""
        out = C.c_int()
        self._call("cr_get_degraded", C.byref(out))
        return bool(out.value)

    def setPrecision(self, precision):
        """"fp64" (default, the reference's arithmetic) or "mixed" (FP32 pair
        terms on FP64-formed offsets; everything else FP64)."""
        code = {"fp64": 0, "mixed": 1}.get(precision, precision)
        self._call("cr_set_precision", int(code))

    def getPrecision(self):
        out = C.c_int()
        self._call("cr_get_precision", C.byref(out))
        return {0: "fp64", 1: "mixed"}[out.value]

    def autotune(self, reps=50):
        out = C.c_int()
        self._call("cr_autotune", int(reps), C.byref(out))
        return out.value

    def profileStepKernel(self, reps=100):
        out = C.c_double()
        self._call("cr_profile_step_kernel", int(reps), C.byref(out))
        return out.value

    def getLaunchCount(self):
        out = C.c_longlong()
        self._call("cr_get_launch_count", C.byref(out))
        return out.value

    # -------------------------------------------------------------- helpers
    @classmethod
    def from_packing(cls, pk, potential="harmonic", interaction="vertexVertex", ea=1.0, el=1.0, eb=0.01,
                     ec=1.0, LJcutoff=2.5, l1=0.0, l2=0.0, dt=None, **_):
        """Context holding a :class:`cudaring_b200.synth.Packing` with the given parameters."""
        d = cls(pk.nv_list)
        d.setBoxSize(pk.box)
        d.setPotentialType(getattr(simControl.potentialEnum, potential))
        d.setInteractionType(getattr(simControl.interactionEnum, interaction))
        d.setEnergyCosts(ea, el, eb, ec)
        d.setLJcutoff(LJcutoff)
        d.setAttractionConstants(l1, l2)
        if dt is not None:
            d.setTimeStep(dt)
        d.setVertexRadii(pk.rad)
        d.setRestAreas(pk.a0)
        d.setRestLengths(pk.l0)
        d.setRestAngles(pk.theta0)
        d.setVertexPositions(pk.pos)
        d.setVertexVelocities(pk.vel)
        return d
