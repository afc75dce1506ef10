/* cudaring.h -- C ABI of the B200-native cudaRing hot path (libcudaring.so).
 *
 * One `cr_ctx` is one 2-D periodic system of deformable (or rigid) ring
 * polymers, owned on one GPU.  Each entry point replaces the `DPM2D` /
 * `SimInterface` / `FIRE` member function of the reference (farceri/cudaRing)
 * cited beside it (file:line within that project), keeps its argument
 * meaning, and adds an `int` status return (CR_OK on success).  Host arrays
 * use the reference's layout: AoS [x0,y0,x1,y1,...] float64 for per-vertex
 * vectors, ring-contiguous counter-clockwise vertex order, int64 (`long`)
 * indices.  Setters copy synchronously; loop functions are stream-ordered on
 * the context's own stream and synchronise once before returning.
 *
 * Differences from the reference kept deliberately, all at the boundary:
 *   - loop functions take a step count (the reference advances one step per
 *     call); `cr_nve_loop(ctx, 1)` is `DPM2D::NVELoop()`;
 *   - the reference keeps one live model per process in __constant__ memory;
 *     any number of contexts may coexist here;
 *   - random numbers come from a counter-based Philox4x32-10 stream keyed by
 *     `cr_set_seed` instead of Thrust's engine reseeded from lrand48().
 */
#ifndef CUDARING_H
#define CUDARING_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cr_ctx cr_ctx;

/* Status codes. */
enum {
  CR_OK = 0,
  CR_EINVAL = 1,        /* bad argument (size mismatch, unknown enum, NULL) */
  CR_ENOMEM = 2,        /* device or host allocation failed */
  CR_ECUDA = 3,         /* CUDA runtime error; see cr_last_error */
  CR_ENONFINITE = 4,    /* a NaN/Inf force or position was produced */
  CR_ETIMEOUT = 5,      /* a bounded device wait ran out */
  CR_ENBR_OVERFLOW = 6, /* neighbour capacity exceeded and could not grow */
  CR_ESTATE = 7,        /* call out of order (e.g. loop before init) */
  CR_ENOTSUP = 8        /* option the reference has but this build does not run */
};

/* simControlStruct enums (include/DPM2D.h:22-32), same numbering. */
enum { CR_POTENTIAL_HARMONIC = 0, CR_POTENTIAL_LENNARD_JONES = 1, CR_POTENTIAL_ADHESIVE = 2, CR_POTENTIAL_WCA = 3 };
enum { CR_INTERACTION_VERTEX_VERTEX = 0, CR_INTERACTION_VERTEX_SMOOTH = 1, CR_INTERACTION_CELL_SMOOTH = 2,
       CR_INTERACTION_ALL = 3 };
enum { CR_MONOMER_HARMONIC = 0, CR_MONOMER_FENE = 1 };
enum { CR_PARTICLE_PASSIVE = 0, CR_PARTICLE_ACTIVE = 1, CR_PARTICLE_ACTIVE_SHAPE = 2 };
enum { CR_SHAPE_DEFORMABLE = 0, CR_SHAPE_RIGID = 1 };
enum { CR_NOISE_LANGEVIN = 0, CR_NOISE_BAOAB = 1, CR_NOISE_BROWNIAN = 2, CR_NOISE_DRIVEN_BROWNIAN = 3 };
enum { CR_GEOMETRY_NORMAL = 0, CR_GEOMETRY_FIXED_BOX = 1, CR_GEOMETRY_FIXED_SIDES = 2, CR_GEOMETRY_ROUND_BOX = 3 };
/* Arithmetic of the deformable-ring force kernel (no reference counterpart;
 * the reference is FP64 throughout). */
enum { CR_PRECISION_FP64 = 0, CR_PRECISION_MIXED = 1 };

/* ---- lifecycle -------------------------------------------------------- */

/* DPM2D::DPM2D (include/DPM2D.h:47) + setNumVertexInParticleList (:267) +
 * initParticleIdList (:219): numVertexInParticleList[numParticles] sets the
 * ring sizes; the context selects the current CUDA device. */
int cr_create(long numParticles, const long* numVertexInParticleList, cr_ctx** out);
int cr_destroy(cr_ctx* ctx);
/* Message of the last failing call on this context ("" if none). */
const char* cr_last_error(const cr_ctx* ctx);
/* DPM2D::getNumVertices (include/DPM2D.h:262) */
int cr_get_num_vertices(const cr_ctx* ctx, long* out);
int cr_get_num_particles(const cr_ctx* ctx, long* out);

/* ---- control switches (include/DPM2D.h:231-249) -------------------------- */
int cr_set_potential_type(cr_ctx* ctx, int potentialType);
int cr_set_interaction_type(cr_ctx* ctx, int interactionType);
int cr_set_monomer_type(cr_ctx* ctx, int monomerType);
int cr_set_particle_type(cr_ctx* ctx, int particleType);
int cr_set_noise_type(cr_ctx* ctx, int noiseType);
int cr_set_shape_type(cr_ctx* ctx, int shapeType);
/* Only CR_GEOMETRY_NORMAL (periodic) is run; walls return CR_ENOTSUP. */
int cr_set_geometry_type(cr_ctx* ctx, int geometryType);

/* ---- parameters ------------------------------------------------------- */
/* DPM2D::setBoxSize (include/DPM2D.h:275): boxSize[2] */
int cr_set_box_size(cr_ctx* ctx, const double* boxSize);
int cr_get_box_size(const cr_ctx* ctx, double* boxSize);
/* DPM2D::setEnergyCosts (include/DPM2D.h:525) */
int cr_set_energy_costs(cr_ctx* ctx, double ea, double el, double eb, double ec);
/* DPM2D::setLJcutoff (include/DPM2D.h:539): LJecut/LJfshift use the ec set
 * at the time of this call, as in the reference (src/DPM2D.cu:1923-1932). */
int cr_set_lj_cutoff(cr_ctx* ctx, double LJcutoff);
/* DPM2D::setAttractionConstants (include/DPM2D.h:535) */
int cr_set_attraction_constants(cr_ctx* ctx, double l1, double l2);
/* DPM2D::setFENEconstants (include/DPM2D.h:541) */
int cr_set_fene_constants(cr_ctx* ctx, double stiff, double ext);
/* DPM2D::setTimeStep (include/DPM2D.h:545) */
int cr_set_time_step(cr_ctx* ctx, double dt);
/* DPM2D::setSelfPropulsionParams (include/DPM2D.h:527) */
int cr_set_self_propulsion_params(cr_ctx* ctx, double driving, double taup);
/* Seed of the Philox stream used by every stochastic update. */
int cr_set_seed(cr_ctx* ctx, unsigned long long seed);

/* ---- state upload / download (host arrays, reference layout) ----------- */
/* DPM2D::setVertexPositions / getVertexPositions (include/DPM2D.h:357-358): pos[2 Nv] */
int cr_set_vertex_positions(cr_ctx* ctx, const double* pos);
int cr_get_vertex_positions(const cr_ctx* ctx, double* pos);
/* DPM2D::setVertexVelocities / getVertexVelocities (include/DPM2D.h:366-367) */
int cr_set_vertex_velocities(cr_ctx* ctx, const double* vel);
int cr_get_vertex_velocities(const cr_ctx* ctx, double* vel);
/* DPM2D::getVertexForces (include/DPM2D.h:370) */
int cr_get_vertex_forces(const cr_ctx* ctx, double* force);
int cr_set_vertex_forces(cr_ctx* ctx, const double* force);
/* Per-vertex energies (shape + vertex-vertex half-pair terms), d_energy. */
int cr_get_vertex_energies(const cr_ctx* ctx, double* energy);
/* DPM2D::getParticleEnergies (include/DPM2D.h:345): smooth-interaction ring energies */
int cr_get_particle_energies(const cr_ctx* ctx, double* pEnergy);
/* DPM2D::setVertexRadii (include/DPM2D.h:283) */
int cr_set_vertex_radii(cr_ctx* ctx, const double* rad);
int cr_get_vertex_radii(const cr_ctx* ctx, double* rad);
/* DPM2D::setRestAreas / setRestLengths / setRestAngles (include/DPM2D.h:286-292) */
int cr_set_rest_areas(cr_ctx* ctx, const double* a0);
int cr_get_rest_areas(const cr_ctx* ctx, double* a0);
int cr_set_rest_lengths(cr_ctx* ctx, const double* l0);
int cr_get_rest_lengths(const cr_ctx* ctx, double* l0);
int cr_set_rest_angles(cr_ctx* ctx, const double* theta0);
int cr_get_rest_angles(const cr_ctx* ctx, double* theta0);
/* DPM2D::getAreas / getPerimeters / getSegmentLengths / getSegmentAngles
 * (include/DPM2D.h:295-302), as of the last force evaluation. */
int cr_get_areas(const cr_ctx* ctx, double* area);
int cr_get_perimeters(const cr_ctx* ctx, double* perimeter);
int cr_get_segment_lengths(const cr_ctx* ctx, double* length);
int cr_get_segment_angles(const cr_ctx* ctx, double* theta);
/* DPM2D::calcParticlePositions + getParticlePositions (include/DPM2D.h:321, 331) */
int cr_calc_particle_positions(cr_ctx* ctx);
int cr_get_particle_positions(const cr_ctx* ctx, double* particlePos);
int cr_set_particle_positions(cr_ctx* ctx, const double* particlePos);
/* DPM2D::calcParticleShape (include/DPM2D.h:319) */
int cr_calc_particle_shape(cr_ctx* ctx);

/* ---- neighbours (src/DPM2D.cu:1300-1423, 3479-3518) -------------------- */
/* DPM2D::setDisplacementCutoff (include/DPM2D.h:447): returns cutDistance. */
int cr_set_displacement_cutoff(cr_ctx* ctx, double cutoff, double size, double* cutDistance);
/* DPM2D::calcNeighborList / calcNeighbors (include/DPM2D.h:638-640): builds
 * the list {j in another ring : d_ij/(r_i+r_j) - 1 < cutDistance} with a
 * device cell list; the set equals the reference's brute-force scan. */
int cr_calc_neighbor_list(cr_ctx* ctx, double cutDistance);
/* DPM2D::checkNeighbors (include/DPM2D.h:459): rebuild when any vertex moved
 * more than cutoff/3 since the last rebuild. */
int cr_check_neighbors(cr_ctx* ctx);
/* DPM2D::resetLastPositions (include/DPM2D.h:360) */
int cr_reset_last_positions(cr_ctx* ctx);
/* The reference's neighborListSize (power of two, only grows). */
int cr_get_neighbor_list_size(const cr_ctx* ctx, long* listSize);
/* DPM2D::getNeighbors (include/DPM2D.h:387): out[Nv * listSize] row-major,
 * ascending neighbour ids, padded with -1. */
int cr_get_neighbors(const cr_ctx* ctx, long* out);
/* DPM2D::getMaxNeighborList (include/DPM2D.h:385): out[Nv] */
int cr_get_max_neighbor_list(const cr_ctx* ctx, long* out);
/* DPM2D::getUpdateCount / resetUpdateCount (include/DPM2D.h:449-451) */
int cr_get_update_count(const cr_ctx* ctx, long* out);
int cr_reset_update_count(cr_ctx* ctx);

/* ---- forces and reductions --------------------------------------------- */
/* DPM2D::calcForceEnergy (include/DPM2D.h:547): shape + interaction (+ self
 * propulsion for active rings), overwriting forces and energies. */
int cr_calc_force_energy(cr_ctx* ctx);
/* DPM2D::getPotentialEnergy / getKineticEnergy / getEnergy / getTemperature
 * (include/DPM2D.h:403-409) */
int cr_get_potential_energy(cr_ctx* ctx, double* out);
int cr_get_kinetic_energy(cr_ctx* ctx, double* out);
int cr_get_energy(cr_ctx* ctx, double* out);
int cr_get_temperature(cr_ctx* ctx, double* out);
/* DPM2D::getMaxUnbalancedForce / getTotalForceMagnitude (include/DPM2D.h:381-383) */
int cr_get_max_unbalanced_force(cr_ctx* ctx, double* out);
int cr_get_total_force_magnitude(cr_ctx* ctx, double* out);
/* DPM2D::getPhi / getPreferredPhi (include/DPM2D.h:431-433) */
int cr_get_phi(cr_ctx* ctx, double* out);
int cr_get_preferred_phi(cr_ctx* ctx, double* out);
/* DPM2D::getMeanVertexRadius / getMeanParticleSize (include/DPM2D.h:306-312) */
int cr_get_mean_vertex_radius(cr_ctx* ctx, double* out);
int cr_get_mean_particle_size(cr_ctx* ctx, double* out);
/* DPM2D::scaleVertices (include/DPM2D.h:506): scales rings about their
 * current centroids and multiplies a0 by scale^2, l0 and rad by scale. */
int cr_scale_vertices(cr_ctx* ctx, double scale);

/* ---- integrators (src/Simulator.cu, src/DPM2D.cu:3713-3775) ------------- */
/* DPM2D::initNVE (include/DPM2D.h:684): readState != 0 keeps velocities;
 * otherwise every vertex gets its ring's N(0, sqrt(T)) velocity
 * (Langevin::injectKineticEnergy, src/Simulator.cu:32-52). */
int cr_init_nve(cr_ctx* ctx, double T, int readState);
/* DPM2D::NVELoop (include/DPM2D.h:686), nsteps times. */
int cr_nve_loop(cr_ctx* ctx, long nsteps);
/* DPM2D::initNVERescale (include/DPM2D.h:688): ring-rigid thermal
 * velocities scaled to exactly T; each NVERescaleLoop step (:690) first
 * scales all velocities back to T (NVERescale, src/Simulator.cu:215-238). */
int cr_init_nve_rescale(cr_ctx* ctx, double T);
int cr_nve_rescale_loop(cr_ctx* ctx, long nsteps);
/* SimInterface::conserveMomentum (include/Simulator.h:51): removes the mean
 * vertex velocity (deformable rings, src/Simulator.cu:91-108) or the mean
 * ring velocity over all rings (rigid rings, src/Simulator.cu:309-312). */
int cr_conserve_momentum(cr_ctx* ctx);
/* DPM2D::initLangevin (include/DPM2D.h:680): the noise type selects
 * Langevin, BAOAB, Brownian or driven Brownian (src/DPM2D.cu:3713-3753). */
int cr_init_langevin(cr_ctx* ctx, double T, double gamma, int readState);
/* DPM2D::langevinLoop (include/DPM2D.h:682), nsteps times. */
int cr_langevin_loop(cr_ctx* ctx, long nsteps);

/* ---- FIRE (src/FIRE.cu:29-41, 302-411) ---------------------------------- */
/* DPM2D::initFIRE (include/DPM2D.h:665): params[7] = {a_start, f_dec, f_inc,
 * f_a, dt, dt_max, a}. */
int cr_init_fire(cr_ctx* ctx, const double* params, long minStep, long numStep, long numDOF);
/* DPM2D::vertexFIRELoop (include/DPM2D.h:673), nsteps times. */
int cr_vertex_fire_loop(cr_ctx* ctx, long nsteps);
/* The driver loop of compressFIRE.cpp:109-117: FIRE iterations until
 * getMaxUnbalancedForce() <= tol or maxIter iterations; reports both. */
int cr_fire_minimize(cr_ctx* ctx, double tol, long maxIter, long* iterations, double* maxForce);
/* FIRE scalars {dt, a, numStep} after the last iteration. */
int cr_get_fire_state(cr_ctx* ctx, double* out3);

/* ---- rigid rings (src/DPM2D.cu:2128-2179, src/Simulator.cu:241-371) ----- */
/* DPM2D::calcRigidForceEnergy (include/DPM2D.h:567): vertex-vertex forces,
 * per-vertex torque about the ring centroid, ring force, torque / moment of
 * inertia (the angular acceleration), moment of inertia and energy. */
int cr_calc_rigid_force_energy(cr_ctx* ctx);
/* DPM2D::initRigidNVE / rigidNVELoop (include/DPM2D.h:697-699): ring
 * velocities N(0, sqrt(T)) with zero mean unless readState; angles and
 * angular velocities start at zero. */
int cr_init_rigid_nve(cr_ctx* ctx, double T, int readState);
int cr_rigid_nve_loop(cr_ctx* ctx, long nsteps);
/* DPM2D::initRigidLangevin / rigidLangevinLoop (include/DPM2D.h:693-695).
 * Deliberate fix: the ring velocity takes noise*xi - gamma*v with noise =
 * sqrt(2 T gamma / dt); the reference adds unscaled N(0,1) draws
 * (src/Simulator.cu:272-289).  Active rigid rings (particle type active) are
 * pushed along a self-propulsion angle that diffuses with 1/taup. */
int cr_init_rigid_langevin(cr_ctx* ctx, double T, double gamma, int readState);
int cr_rigid_langevin_loop(cr_ctx* ctx, long nsteps);
/* Ring state (include/DPM2D.h:339-354): velocities [2 Np], angles [Np],
 * angular velocities [Np], forces [2 Np], torques [Np] (angular
 * accelerations), vertex torques [Nv]. */
int cr_get_particle_velocities(const cr_ctx* ctx, double* out);
int cr_set_particle_velocities(cr_ctx* ctx, const double* in);
int cr_get_particle_angles(const cr_ctx* ctx, double* out);
int cr_set_particle_angles(cr_ctx* ctx, const double* in);
int cr_get_particle_angular_velocities(const cr_ctx* ctx, double* out);
int cr_set_particle_angular_velocities(cr_ctx* ctx, const double* in);
int cr_get_particle_forces(const cr_ctx* ctx, double* out);
int cr_get_particle_torques(const cr_ctx* ctx, double* out);
int cr_get_vertex_torques(const cr_ctx* ctx, double* out);
/* DPM2D::getParticleKineticEnergy (include/DPM2D.h:415): 1/2 sum |v_ring|^2 */
int cr_get_particle_kinetic_energy(cr_ctx* ctx, double* out);

/* ---- soft-disk pre-packing (compressFIRE.cpp:53-90) --------------------- */
/* The particle-level stage before vertex FIRE: every ring is a soft disk of
 * radius particleRad at its particle position (cr_set/get_particle_positions),
 * minimised by FIRE, after which the vertices are placed on circles about the
 * disk centres.  Forces use the potential set by cr_set_potential_type with
 * radSum = r_i + r_j; forces, velocities and energies per particle are read
 * with cr_get_particle_forces / _velocities / _energies. */
/* DPM2D::setParticleRadii / getParticleRadii (src/DPM2D.cu:814-822) */
int cr_set_particle_radii(cr_ctx* ctx, const double* particleRad);
int cr_get_particle_radii(const cr_ctx* ctx, double* particleRad);
/* DPM2D::getMeanParticleSigma / getMinParticleSigma (src/DPM2D.cu:762-768);
 * the minimum starts from 1, as the reference's reduction does. */
int cr_get_mean_particle_sigma(cr_ctx* ctx, double* out);
int cr_get_min_particle_sigma(cr_ctx* ctx, double* out);
/* DPM2D::setRandomParticles (src/DPM2D.cu:1601-1629): box 1 x 1, rest areas,
 * lengths and vertex radii scaled by sqrt(preferred phi / phi0), disk
 * centres uniform in the box and radii extraRad * sqrt(2 a0 / (nv sin(2 pi / nv))),
 * drawing from the drand48() stream that srand48(seed) starts. */
int cr_set_random_particles(cr_ctx* ctx, double phi0, double extraRad, long seed);
/* DPM2D::calcParticleNeighborList (src/DPM2D.cu:3521-3545): j != i is listed
 * when -(1 - d_ij / (2 r_i)) < cutDistance (the reference's particle rule
 * sums the listing particle's own radius twice, include/cudaKernel.cuh:289-296,
 * 1765-1789).  Size, counts and rows (ascending, -1 padded) as for vertices. */
int cr_calc_particle_neighbor_list(cr_ctx* ctx, double cutDistance);
int cr_get_particle_neighbor_list_size(const cr_ctx* ctx, long* out);
int cr_get_particle_max_neighbor_list(const cr_ctx* ctx, long* partMaxNeighborList);
int cr_get_particle_neighbors(const cr_ctx* ctx, long* partNeighborList);
/* DPM2D::calcParticleForceEnergy for the periodic box (src/DPM2D.cu:3611-3622;
 * kernelCalcParticleInteraction, include/cudaKernel.cuh:1185-1219) */
int cr_calc_particle_force_energy(cr_ctx* ctx);
/* DPM2D::getParticlePotentialEnergy / getParticleMaxUnbalancedForce
 * (src/DPM2D.cu:1097-1099, 3633-3638) */
int cr_get_particle_potential_energy(cr_ctx* ctx, double* out);
int cr_get_particle_max_unbalanced_force(cr_ctx* ctx, double* out);
/* DPM2D::resetParticleLastPositions / getParticleMaxDisplacement
 * (src/DPM2D.cu:838-840, 1435-1441) */
int cr_reset_particle_last_positions(cr_ctx* ctx);
int cr_get_particle_max_displacement(cr_ctx* ctx, double* out);
/* DPM2D::initFIRE + setParticleMassFIRE (src/DPM2D.cu:3660-3684): p7 =
 * {a_start, f_dec, f_inc, f_a, dt, dt_max, a}, masses pi / r^2 per particle. */
int cr_init_particle_fire(cr_ctx* ctx, const double* p7, long minStep, long numStep);
/* {dt, a, numStep} of the particle minimiser (FIRE.h:31-42) */
int cr_get_particle_fire_state(cr_ctx* ctx, double* out3);
/* DPM2D::particleFIRELoop (src/DPM2D.cu:3692-3694; FIRE::minimizerParticleLoop,
 * src/FIRE.cu:156-171), nsteps iterations; the particle list is not rebuilt. */
int cr_particle_fire_loop(cr_ctx* ctx, long nsteps);
/* The driver loop of compressFIRE.cpp:66-78: iterations until max |F_d| <= tol
 * or maxIterations, the particle list rebuilt (and the last positions reset)
 * after any iteration in which a particle moved more than
 * (1 + cutDistance) * getMinParticleSigma / 3 since the last build.  Call it,
 * as the driver does, after building the list and computing the forces.
 * Runs on the device in captured chunks of 64 iterations. */
int cr_particle_fire_minimize(cr_ctx* ctx, double cutDistance, double tol, long maxIterations, long* iterations);
/* DPM2D::initVerticesOnParticles (src/DPM2D.cu:1678-1691): vertex v of ring q
 * at R (cos 2 pi v / nv, sin 2 pi v / nv) + particlePos_q + 1e-3 l0_v (u, u'),
 * R = sqrt(2 a0 / (nv sin(2 pi / nv))), v the global vertex index; velocities,
 * forces and energies zeroed, the vertex list marked stale.  draws: the 2 nv
 * uniforms u in the reference's drand48() call order, or NULL for the
 * context's Philox stream. */
int cr_init_vertices_on_particles(cr_ctx* ctx, const double* draws);

/* ---- run statistics and measurement ------------------------------------ */
/* Kernels this context has run since creation (direct launches and
 * graph-node kernels per replay). */
int cr_get_launch_count(const cr_ctx* ctx, long long* out);
/* The context's CUDA stream (cudaStream_t), for recording timing events. */
int cr_get_stream(const cr_ctx* ctx, void** out);
/* Average device time of the fused step kernel (the integrator's force +
 * update op) over `reps` back-to-back launches on scratch copies of the
 * state, timed with CUDA events on the context stream; state is unchanged. */
int cr_profile_step_kernel(cr_ctx* ctx, long reps, double* ms_per_launch);

/* ---- tuning (no reference counterpart: launch shape of the fused kernel) -- */
/* Lanes per vertex in the pair phase of the fused kernel (1, 2, 4 or 8);
 * tiles hold 128, 96, 64 or 32 vertices of whole rings respectively. */
int cr_set_lanes(cr_ctx* ctx, int lanes);
int cr_get_lanes(const cr_ctx* ctx, int* lanes);
/* 1: step sequences run as captured CUDA graphs (default), every op that
 * moved positions followed by the one-launch rebuild check; 0: direct
 * launches with a host check after each op. */
int cr_set_use_graphs(cr_ctx* ctx, int on);
/* 1 (default): the middle steps of NVE, Langevin and BAOAB runs of
 * deformable rings run in a multi-step kernel (up to 64 steps per launch,
 * grid barriers between steps) when the GPU holds all of its CTAs at once
 * and one or two lanes per vertex are in use; 0: one launch per step.  FP64
 * results are identical; mixed-precision results agree to FP32 rounding.
 * The kernel's grid barriers need all of its CTAs resident (so does the
 * one-launch neighbour-list build).  With other work running on the same
 * GPU a barrier may give up (cr_set_spin_limit); the context then goes back
 * to the state the call started from, switches to one launch per op with the
 * multi-kernel list build for the rest of its life, and runs the call again
 * (cr_get_degraded reports it). */
int cr_set_multistep(cr_ctx* ctx, int on);
/* No reference counterpart.  Polls a grid-barrier wait makes before giving
 * up (default 2^20, about a second; 0 restores the default; a negative
 * value: the first poll that finds a barrier incomplete gives up, which
 * every wait but the last CTA's does).  For GPUs shared with other work and
 * for tests of the fallback above. */
int cr_set_spin_limit(cr_ctx* ctx, long long polls);
/* No reference counterpart.  *out = 1 once a grid-barrier wait of this
 * context gave up and it runs one launch per op. */
int cr_get_degraded(const cr_ctx* ctx, int* out);
/* Times the fused step kernel for every lane count whose tile holds the
 * largest ring (cr_profile_step_kernel, `reps` launches each) and keeps the
 * fastest; reports the choice.  Needs a neighbour list. */
int cr_autotune(cr_ctx* ctx, long reps, int* lanes_out);
/* CR_PRECISION_FP64 (default): every term in FP64, matching the reference.
 * CR_PRECISION_MIXED: positions, velocities, integration, the shape terms
 * and all reductions stay FP64; the vertex-vertex and vertex-segment pair
 * terms run in FP32 on minimum-image offsets formed in FP64 and rounded
 * once, with FP32 force accumulation per vertex.  Applies to the force
 * evaluation, the fused step kernel and FIRE of deformable rings. */
int cr_set_precision(cr_ctx* ctx, int precision);
int cr_get_precision(const cr_ctx* ctx, int* precision);

/* ---- neighbour list without allocation -----------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves (a host framework that hands out only fixed, pre-sized
 * buffers; code that must not call cudaMalloc/cudaFree because they
 * synchronise the whole device and stall its other streams): builds the
 * same neighbour list as cr_calc_neighbor_list from caller-owned device
 * arrays, keeping every temporary in one static device array of the library,
 * so it calls no cudaMalloc, cudaFree or allocating library routine.
 *   pos[2 Nv] (double, AoS), rad[Nv], ring_of[Nv] (int32 ring index): device
 *   boxSize[2]: host; maxRad >= every radius; cutDistance as returned by
 *   cr_set_displacement_cutoff; neighbors: device int32 [capacity][Nv]
 *   (slot-major: neighbour s of vertex v at neighbors[s * Nv + v]); counts:
 *   device int32 [Nv]; *maxCount: host, largest count; stream: cudaStream_t
 *   (NULL = legacy default stream); the call synchronises that stream.
 * Limits: Nv <= CR_NOALLOC_MAX_VERTICES, else CR_EINVAL before any buffer
 * is touched; the cell grid is coarsened to at most CR_NOALLOC_MAX_CELLS
 * cells (same list); CR_ENBR_OVERFLOW when a count exceeds capacity (counts
 * and *maxCount are still complete).  The first call on a device looks up the
 * scratch array's address (once per device) and keeps it for the process:
 * make that call before any stream capture, and do not use the entry point on
 * a device after cudaDeviceReset.  All calls share that array: calls that
 * overlap on the GPU race and must be serialised. */
#define CR_NOALLOC_MAX_VERTICES 65536
#define CR_NOALLOC_MAX_CELLS 65536
int cr_neighbor_list_noalloc(const double* pos, const double* rad, const int* ring_of, long numVertices,
                             const double* boxSize, double maxRad, double cutDistance, long capacity,
                             int* neighbors, int* counts, long* maxCount, void* stream);

/* ---- derivatives ---------------------------------------------------------
 * No reference counterpart (the reference has no derivatives beyond forces).
 * Evaluated at the current positions with the current neighbour list, for
 * deformable rings (harmonic or FENE monomers; vertex-vertex or smooth
 * vertex-segment interaction; rigid rings return CR_ENOTSUP).  U is the total
 * potential energy. */
enum { CR_PARAM_EA = 0, CR_PARAM_EL = 1, CR_PARAM_EB = 2, CR_PARAM_LN_CALA0 = 3 };
/* Hessian-vector product hv = (d^2 U / dx^2) v, v and hv of 2 Nv values */
int cr_hvp(cr_ctx* ctx, const double* v, double* hv);
/* the same with v and hv in device memory of the context's device */
int cr_hvp_device(cr_ctx* ctx, const double* v_dev, double* hv_dev);
/* pressure P = -dU/dA for an affine dilation of positions and box (the
 * virial pressure of every interaction and shape term; the reference's
 * stress kernel, include/cudaKernel.cuh:1513-1568, covers pair terms only) */
int cr_calc_pressure(cr_ctx* ctx, double* P);
/* derivatives along one parameter at fixed positions: dU, dP (scalars), dF
 * = dForce/dparam and dPdx = dP/dx (2 Nv each; any output may be NULL).
 * CR_PARAM_LN_CALA0 differentiates along ln(calA0), with rest lengths and
 * vertex radii proportional to sqrt(calA0) (DPM2D.cu:1577-1581 conventions). */
int cr_param_derivatives(cr_ctx* ctx, int param, double* dU, double* dP, double* dF, double* dPdx);
/* conjugate-gradient solve of H x = b (H the Hessian at the current
 * positions) on the complement of the uniform translations, to relative
 * residual tol; preconditioned (cr_set_cg_preconditioner) */
int cr_hessian_solve(cr_ctx* ctx, const double* b, double* x, double tol, long maxIter, long* iterations,
                     double* relres);
/* No reference counterpart.  Preconditioner of cr_hessian_solve: 1
 * (default) block-Jacobi, the inverse 2 x 2 diagonal Hessian block of every
 * vertex (its diagonal's magnitudes where the block is not positive
 * definite); 0 none. */
int cr_set_cg_preconditioner(cr_ctx* ctx, int kind);
/* No reference counterpart.  The 2 x 2 diagonal blocks of the Hessian,
 * d2U / dx_v dx_v: out[3 v .. 3 v + 2] = (xx, xy, yy) for every vertex. */
int cr_hessian_diag_blocks(cr_ctx* ctx, double* out);

/* ---- batches of independent systems -------------------------------------
 * No single reference counterpart: the reference holds one system per process
 * (its parameters live in __constant__ symbols, include/cudaKernel.cuh:17-67)
 * and its drivers loop over packings one at a time (compressFIRE.cpp).  A
 * batch holds S systems of deformable rings with their own boxes, ring counts
 * and packing fractions in concatenated arrays (system s's rings and
 * vertices follow system s-1's, in the order of numParticles[] and
 * numVertexInParticleList[]), and runs every op as one launch over all of
 * them; each system keeps its own neighbour list, FIRE scalars, convergence
 * and rebuild flags.  Energy costs, potential and interaction are shared.
 * Arrays are in the single-system layout, concatenated over systems. */
typedef struct cr_batch cr_batch;
int cr_batch_create(long numSystems, const long* numParticles, const long* numVertexInParticleList, cr_batch** out);
int cr_batch_destroy(cr_batch* b);
const char* cr_batch_last_error(const cr_batch* b);
int cr_batch_get_sizes(const cr_batch* b, long* numSystems, long* numParticles, long* numVertices);
int cr_batch_set_potential_type(cr_batch* b, int potential);
int cr_batch_set_interaction_type(cr_batch* b, int interaction);
int cr_batch_set_energy_costs(cr_batch* b, double ea, double el, double eb, double ec);
int cr_batch_set_lj_cutoff(cr_batch* b, double LJcutoff);
int cr_batch_set_attraction_constants(cr_batch* b, double l1, double l2);
int cr_batch_set_precision(cr_batch* b, int precision);
/* lanes per vertex of the batched tile kernel: 1, 2 or 4 (with that lane
 * count's default tile: 128, 96 or 64 vertices) */
int cr_batch_set_lanes(cr_batch* b, int lanes);
int cr_batch_get_lanes(const cr_batch* b, int* lanes);
/* Tile shape of the batched tile kernel: (lanes per vertex, threads per CTA)
 * in (1, 128), (1, 192), (2, 128), (2, 192), (4, 256); a tile holds
 * threads / lanes vertices of whole rings of one system.  Rings longer than
 * 128 vertices need (1, 192). */
int cr_batch_set_tile_shape(cr_batch* b, int lanes, int block);
int cr_batch_get_tile_shape(const cr_batch* b, int* lanes, int* block);
/* times the batched FIRE force kernel for each admissible tile shape and keeps the fastest */
int cr_batch_autotune(cr_batch* b, long reps, int* lanes_out);
int cr_batch_profile_fire_tile(cr_batch* b, long reps, double* ms_per_launch);
/* boxSizes[2 S] = {Lx_0, Ly_0, Lx_1, ...} */
int cr_batch_set_box_sizes(cr_batch* b, const double* boxSizes);
int cr_batch_get_box_sizes(const cr_batch* b, double* boxSizes);
int cr_batch_set_vertex_positions(cr_batch* b, const double* pos);
int cr_batch_get_vertex_positions(cr_batch* b, double* pos);
int cr_batch_set_vertex_velocities(cr_batch* b, const double* vel);
int cr_batch_get_vertex_velocities(cr_batch* b, double* vel);
int cr_batch_get_vertex_forces(cr_batch* b, double* force);
int cr_batch_get_vertex_energies(cr_batch* b, double* energy);
int cr_batch_set_vertex_radii(cr_batch* b, const double* rad);
int cr_batch_get_vertex_radii(cr_batch* b, double* rad);
int cr_batch_set_rest_areas(cr_batch* b, const double* a0);
int cr_batch_get_rest_areas(cr_batch* b, double* a0);
int cr_batch_set_rest_lengths(cr_batch* b, const double* l0);
int cr_batch_get_rest_lengths(cr_batch* b, double* l0);
int cr_batch_set_rest_angles(cr_batch* b, const double* theta0);
/* DPM2D::setDisplacementCutoff per system with size_ = 2 <r> of that system;
 * returns the shared cutDistance */
int cr_batch_set_displacement_cutoff(cr_batch* b, double cutoff_, double* cutDistance);
int cr_batch_calc_neighbor_lists(cr_batch* b);
int cr_batch_calc_force_energy(cr_batch* b);
/* per-system results, arrays of S */
int cr_batch_get_potential_energies(cr_batch* b, double* U);
int cr_batch_get_max_unbalanced_forces(cr_batch* b, double* maxF);
int cr_batch_get_phis(cr_batch* b, double* phi);
int cr_batch_get_preferred_phis(cr_batch* b, double* phi);
int cr_batch_get_mean_particle_sizes(cr_batch* b, double* sigma);
/* 1: the system takes part in the batch's ops, 0: it is frozen */
int cr_batch_set_active(cr_batch* b, const int* active);
/* DPM2D::initFIRE for every system; dt (nullable) gives per-system time
 * steps, dt_max scaled with them */
int cr_batch_init_fire(cr_batch* b, const double* FIREparams7, const double* dt, long minStep);
/* FIRE iterations until max |F_i,d| <= tol[s] in every system or maxIter */
int cr_batch_fire_minimize(cr_batch* b, const double* tol, long maxIter, long* iterations, double* maxForce);
/* DPM2D::scaleVertices with one factor per system */
int cr_batch_scale_vertices(cr_batch* b, const double* scale);
/* Quasi-static compression to jamming (compressFIRE.cpp:101-205) of every
 * system.  state[s]: 1 jammed, 2 step limit, 3 compression step halved below
 * min_dphi (phi within min_dphi of jamming). */
typedef struct cr_compress_params {
  double dphi;          /* starting packing-fraction step */
  double min_dphi;      /* stop a system once its halved step falls below this */
  double fire_dt;       /* FIRE time step in units of the mean particle size */
  double tol0;          /* force tolerance times the mean particle size */
  double energy_tol;    /* criterion 1: potential energy per ring threshold */
  long max_fire_iters;  /* FIRE iterations per compression step */
  long max_steps;       /* compression steps */
  int criterion;        /* 0: maximum force (the reference's), 1: energy */
} cr_compress_params;
int cr_batch_compress(cr_batch* b, const cr_compress_params* params, double* phi, long* steps, int* state,
                      long* fireIterations);
/* The same protocol with the host between steps and between chunks of 64
 * FIRE iterations (cr_batch_compress runs the whole loop as one CUDA graph,
 * conditional WHILE nodes over the steps and the chunks); both give the same
 * states. */
int cr_batch_compress_stepwise(cr_batch* b, const cr_compress_params* params, double* phi, long* steps, int* state,
                               long* fireIterations);
int cr_batch_get_launch_count(const cr_batch* b, long long* out);
/* No reference counterpart.  1 (default): FIRE iterations of batches whose
 * tiles the GPU holds at once run in a persistent kernel (FP64; tile shapes
 * (1, 128) and (2, 192)), up to 64 iterations per launch with grid barriers
 * in place of kernel boundaries, the same iterates as one launch per op; 0:
 * one launch per op.  A grid-barrier wait that gives up (cr_set_spin_limit
 * semantics, batch status) switches the batch to one launch per op. */
int cr_batch_set_persistent(cr_batch* b, int on);
/* Entries per vertex the batch's neighbour lists hold (grown on overflow). */
int cr_batch_get_list_capacity(const cr_batch* b, int* out);

#ifdef __cplusplus
}
#endif
#endif /* CUDARING_H */
