// cudaring/DPM2D.hpp -- header-only C++ facade over include/cudaring.h.
//
// Reproduces the hot-path member functions of the reference's DPM2D class
// (include/DPM2D.h of farceri/cudaRing) so driver code written against it
// (runNVE.cpp, compressFIRE.cpp style loops) compiles with few changes:
//   cudaring::DPM2D dpm(numParticles, nDim, numVertexPerParticle);
//   dpm.setPotentialType(...); ...
//   cudaring::ioDPMFile io(&dpm); io.readPackingFromDirectory(dir, numParticles, nDim);
//   dpm.setEnergyCosts(ea, el, eb, ec); ...
//   double cut = dpm.setDisplacementCutoff(0.5, 2 * dpm.getMeanVertexRadius());
//   dpm.calcNeighbors(cut); dpm.calcForceEnergy(); dpm.initNVE(T, readState);
//   while (step != maxStep) { dpm.NVELoop(); ... }
// (ioDPMFile is in cudaring/FileIO.hpp.)  Host vectors are
// std::vector<double> / std::vector<long> in the reference's layout.  Failing
// calls throw cudaring::Error carrying the status code.
//
// The reference constructor sizes the system as nParticles rings of
// nVertexPerParticle vertices; setNumVertexInParticleList (called by the
// packing reader) re-sizes it.  The C ABI fixes the ring sizes when a context
// is created, so the facade records every control switch and parameter set
// so far and replays them on the new context when the ring sizes change.
#pragma once
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../cudaring.h"

namespace cudaring {

class Error : public std::runtime_error {
 public:
  Error(const std::string& what, int code) : std::runtime_error(what), code(code) {}
  int code;
};

class DPM2D {
 public:
  // DPM2D::DPM2D(long nParticles, long dim, long nVertexPerParticle)
  // (include/DPM2D.h:47, src/DPM2D.cu:41-95): nParticles rings of
  // nVertexPerParticle vertices with the reference's default constants
  // (ea 1e5, el 20, eb 10, ec 1, dt 1e-3, unit box).  Only dim == 2 runs.
  DPM2D(long nParticles, long dim, long nVertexPerParticle) {
    if (dim != 2) throw Error("DPM2D: only nDim == 2 is supported", CR_ENOTSUP);
    if (nParticles <= 0 || nVertexPerParticle < 3) throw Error("DPM2D: bad system size", CR_EINVAL);
    create(std::vector<long>((size_t)nParticles, nVertexPerParticle));
  }
  explicit DPM2D(const std::vector<long>& numVertexInParticleList) { create(numVertexInParticleList); }
  ~DPM2D() {
    if (ctx_) cr_destroy(ctx_);
  }
  DPM2D(const DPM2D&) = delete;
  DPM2D& operator=(const DPM2D&) = delete;

  long nDim = 2, numParticles = 0, numVertices = 0;
  cr_ctx* handle() { return ctx_; }

  // sizes (include/DPM2D.h:219-273)
  long getNDim() const { return nDim; }
  long getNumParticles() const { return numParticles; }
  long getNumVertices() const { return numVertices; }
  std::vector<long> getNumVertexInParticleList() const { return nvList_; }
  // DPM2D::setNumVertexInParticleList: new ring sizes; the context is
  // re-created (state cleared) and the recorded switches and parameters are
  // applied to it again
  void setNumVertexInParticleList(const std::vector<long>& list) {
    if (list == nvList_) return;
    cr_ctx* old = ctx_;
    ctx_ = nullptr;
    create(list);
    if (old) cr_destroy(old);
    replay();
  }
  // the reference's per-array initialisers: the context allocates everything
  // when it is created, so these only check the sizes they are given
  void setNumVertices(long n) {
    if (n != numVertices) throw Error("setNumVertices: size differs from the ring list", CR_EINVAL);
  }
  void initParticleIdList() {}
  void initShapeVariables(long nv, long np) { checkSizes(nv, np, "initShapeVariables"); }
  void initDynamicalVariables(long nv) { setNumVertices(nv); }
  void initNeighbors(long nv) { setNumVertices(nv); }
  void setLengthScale() {}
  // neighbour lists are the only neighbour mode (simControlStruct::neighborEnum::neighbor = 0)
  void setNeighborType(int v) {
    if (v != 0) throw Error("setNeighborType: only the neighbour-list mode is supported", CR_ENOTSUP);
  }

  // switches (include/DPM2D.h:231-249)
  void setPotentialType(int v) { record([=](cr_ctx* c) { return cr_set_potential_type(c, v); }, "setPotentialType"); }
  void setInteractionType(int v) {
    record([=](cr_ctx* c) { return cr_set_interaction_type(c, v); }, "setInteractionType");
  }
  void setMonomerType(int v) { record([=](cr_ctx* c) { return cr_set_monomer_type(c, v); }, "setMonomerType"); }
  void setParticleType(int v) { record([=](cr_ctx* c) { return cr_set_particle_type(c, v); }, "setParticleType"); }
  void setNoiseType(int v) { record([=](cr_ctx* c) { return cr_set_noise_type(c, v); }, "setNoiseType"); }
  void setShapeType(int v) { record([=](cr_ctx* c) { return cr_set_shape_type(c, v); }, "setShapeType"); }
  void setGeometryType(int v) { record([=](cr_ctx* c) { return cr_set_geometry_type(c, v); }, "setGeometryType"); }

  // parameters
  void setBoxSize(const std::vector<double>& b) {
    if (b.size() < 2) throw Error("setBoxSize: two lengths expected", CR_EINVAL);
    const double lx = b[0], ly = b[1];
    record([=](cr_ctx* c) { const double v[2] = {lx, ly}; return cr_set_box_size(c, v); }, "setBoxSize");
  }
  std::vector<double> getBoxSize() {
    std::vector<double> out(2);
    ok(cr_get_box_size(ctx_, out.data()), "getBoxSize");
    return out;
  }
  void setEnergyCosts(double ea, double el, double eb, double ec) {
    record([=](cr_ctx* c) { return cr_set_energy_costs(c, ea, el, eb, ec); }, "setEnergyCosts");
  }
  void setLJcutoff(double v) { record([=](cr_ctx* c) { return cr_set_lj_cutoff(c, v); }, "setLJcutoff"); }
  void setAttractionConstants(double l1, double l2) {
    record([=](cr_ctx* c) { return cr_set_attraction_constants(c, l1, l2); }, "setAttractionConstants");
  }
  void setFENEconstants(double s, double e) {
    record([=](cr_ctx* c) { return cr_set_fene_constants(c, s, e); }, "setFENEconstants");
  }
  double setTimeStep(double dt) {
    record([=](cr_ctx* c) { return cr_set_time_step(c, dt); }, "setTimeStep");
    return dt;
  }
  void setSelfPropulsionParams(double f0, double taup) {
    record([=](cr_ctx* c) { return cr_set_self_propulsion_params(c, f0, taup); }, "setSelfPropulsionParams");
  }
  // seed of the context's Philox streams (the reference seeds srand48 from the clock)
  void setSeed(unsigned long long seed) { record([=](cr_ctx* c) { return cr_set_seed(c, seed); }, "setSeed"); }

  // state
  void setVertexPositions(const std::vector<double>& a) { ok(cr_set_vertex_positions(ctx_, a.data()), "setVertexPositions"); }
  std::vector<double> getVertexPositions() { return get2(cr_get_vertex_positions, "getVertexPositions"); }
  void setVertexVelocities(const std::vector<double>& a) { ok(cr_set_vertex_velocities(ctx_, a.data()), "setVertexVelocities"); }
  std::vector<double> getVertexVelocities() { return get2(cr_get_vertex_velocities, "getVertexVelocities"); }
  std::vector<double> getVertexForces() { return get2(cr_get_vertex_forces, "getVertexForces"); }
  void setVertexRadii(const std::vector<double>& a) { ok(cr_set_vertex_radii(ctx_, a.data()), "setVertexRadii"); }
  std::vector<double> getVertexRadii() { return getv(cr_get_vertex_radii, numVertices, "getVertexRadii"); }
  void setRestAreas(const std::vector<double>& a) { ok(cr_set_rest_areas(ctx_, a.data()), "setRestAreas"); }
  std::vector<double> getRestAreas() { return getv(cr_get_rest_areas, numParticles, "getRestAreas"); }
  void setRestLengths(const std::vector<double>& a) { ok(cr_set_rest_lengths(ctx_, a.data()), "setRestLengths"); }
  std::vector<double> getRestLengths() { return getv(cr_get_rest_lengths, numVertices, "getRestLengths"); }
  void setRestAngles(const std::vector<double>& a) { ok(cr_set_rest_angles(ctx_, a.data()), "setRestAngles"); }
  std::vector<double> getRestAngles() { return getv(cr_get_rest_angles, numVertices, "getRestAngles"); }
  // ring shapes (DPM2D::calcParticleShape, getAreas, getPerimeters, getParticleShapes)
  void calcParticleShape() { ok(cr_calc_particle_shape(ctx_), "calcParticleShape"); }
  std::vector<double> getAreas() { return getv(cr_get_areas, numParticles, "getAreas"); }
  std::vector<double> getPerimeters() { return getv(cr_get_perimeters, numParticles, "getPerimeters"); }
  std::vector<double> getParticleShapes() {
    calcParticleShape();
    const std::vector<double> a = getAreas(), p = getPerimeters();
    std::vector<double> out((size_t)(3 * numParticles));
    for (long q = 0; q < numParticles; q++) {
      out[3 * q] = a[q];
      out[3 * q + 1] = p[q];
      out[3 * q + 2] = p[q] * p[q] / (4.0 * 3.14159265358979323846 * a[q]);
    }
    return out;
  }
  void calcParticlePositions() { ok(cr_calc_particle_positions(ctx_), "calcParticlePositions"); }
  std::vector<double> getParticlePositions() {
    calcParticlePositions();
    return getv(cr_get_particle_positions, 2 * numParticles, "getParticlePositions");
  }

  // neighbours
  double setDisplacementCutoff(double cutoff, double size) {
    double c = 0;
    ok(cr_set_displacement_cutoff(ctx_, cutoff, size, &c), "setDisplacementCutoff");
    return c;
  }
  void calcNeighborList(double cutDistance) { ok(cr_calc_neighbor_list(ctx_, cutDistance), "calcNeighborList"); }
  void calcNeighbors(double cutDistance) { calcNeighborList(cutDistance); }
  void checkNeighbors() { ok(cr_check_neighbors(ctx_), "checkNeighbors"); }
  std::vector<long> getNeighbors() {
    long ls = 0;
    ok(cr_get_neighbor_list_size(ctx_, &ls), "getNeighbors");
    std::vector<long> out((size_t)(numVertices * ls));
    ok(cr_get_neighbors(ctx_, out.data()), "getNeighbors");
    return out;
  }
  std::vector<long> getMaxNeighborList() {
    std::vector<long> out((size_t)numVertices);
    ok(cr_get_max_neighbor_list(ctx_, out.data()), "getMaxNeighborList");
    return out;
  }
  long getUpdateCount() {
    long u = 0;
    ok(cr_get_update_count(ctx_, &u), "getUpdateCount");
    return u;
  }
  void resetUpdateCount() { ok(cr_reset_update_count(ctx_), "resetUpdateCount"); }

  // forces and reductions
  void calcForceEnergy() { ok(cr_calc_force_energy(ctx_), "calcForceEnergy"); }
  double getPotentialEnergy() { return scalar(cr_get_potential_energy, "getPotentialEnergy"); }
  double getKineticEnergy() { return scalar(cr_get_kinetic_energy, "getKineticEnergy"); }
  double getEnergy() { return scalar(cr_get_energy, "getEnergy"); }
  double getTemperature() { return scalar(cr_get_temperature, "getTemperature"); }
  double getMaxUnbalancedForce() { return scalar(cr_get_max_unbalanced_force, "getMaxUnbalancedForce"); }
  double getTotalForceMagnitude() { return scalar(cr_get_total_force_magnitude, "getTotalForceMagnitude"); }
  double getPhi() { return scalar(cr_get_phi, "getPhi"); }
  double getPreferredPhi() { return scalar(cr_get_preferred_phi, "getPreferredPhi"); }
  double getMeanVertexRadius() { return scalar(cr_get_mean_vertex_radius, "getMeanVertexRadius"); }
  double getMeanParticleSize() { return scalar(cr_get_mean_particle_size, "getMeanParticleSize"); }
  void scaleVertices(double s) { ok(cr_scale_vertices(ctx_, s), "scaleVertices"); }

  // integrators (one step per call by default, as in the reference)
  void initNVE(double T, bool readState) { ok(cr_init_nve(ctx_, T, readState ? 1 : 0), "initNVE"); }
  void NVELoop(long nsteps = 1) { ok(cr_nve_loop(ctx_, nsteps), "NVELoop"); }
  void initNVERescale(double T) { ok(cr_init_nve_rescale(ctx_, T), "initNVERescale"); }
  void NVERescaleLoop(long nsteps = 1) { ok(cr_nve_rescale_loop(ctx_, nsteps), "NVERescaleLoop"); }
  void conserveMomentum() { ok(cr_conserve_momentum(ctx_), "conserveMomentum"); }
  void initLangevin(double T, double gamma, bool readState) {
    ok(cr_init_langevin(ctx_, T, gamma, readState ? 1 : 0), "initLangevin");
  }
  void langevinLoop(long nsteps = 1) { ok(cr_langevin_loop(ctx_, nsteps), "langevinLoop"); }
  void initFIRE(std::vector<double>& params, long minStep, long numStep, long numDOF) {
    ok(cr_init_fire(ctx_, params.data(), minStep, numStep, numDOF), "initFIRE");
  }
  void vertexFIRELoop(long nsteps = 1) { ok(cr_vertex_fire_loop(ctx_, nsteps), "vertexFIRELoop"); }

  // soft-disk pre-packing (compressFIRE.cpp:53-90)
  void setRandomParticles(double phi0, double extraRad, long seed) {
    ok(cr_set_random_particles(ctx_, phi0, extraRad, seed), "setRandomParticles");
  }
  void calcParticleNeighborList(double cutDistance) {
    ok(cr_calc_particle_neighbor_list(ctx_, cutDistance), "calcParticleNeighborList");
  }
  void calcParticleForceEnergy() { ok(cr_calc_particle_force_energy(ctx_), "calcParticleForceEnergy"); }
  double getParticlePotentialEnergy() { return scalar(cr_get_particle_potential_energy, "getParticlePotentialEnergy"); }
  double getParticleMaxUnbalancedForce() {
    return scalar(cr_get_particle_max_unbalanced_force, "getParticleMaxUnbalancedForce");
  }
  double getMeanParticleSigma() { return scalar(cr_get_mean_particle_sigma, "getMeanParticleSigma"); }
  double getMinParticleSigma() { return scalar(cr_get_min_particle_sigma, "getMinParticleSigma"); }
  void resetParticleLastPositions() { ok(cr_reset_particle_last_positions(ctx_), "resetParticleLastPositions"); }
  double getParticleMaxDisplacement() { return scalar(cr_get_particle_max_displacement, "getParticleMaxDisplacement"); }
  // DPM2D::initFIRE followed by setParticleMassFIRE, for particle FIRE
  void initParticleFIRE(std::vector<double>& params, long minStep, long numStep) {
    ok(cr_init_particle_fire(ctx_, params.data(), minStep, numStep), "initParticleFIRE");
  }
  void particleFIRELoop(long nsteps = 1) { ok(cr_particle_fire_loop(ctx_, nsteps), "particleFIRELoop"); }
  long particleFIREMinimize(double cutDistance, double tol, long maxIterations) {
    long it = 0;
    ok(cr_particle_fire_minimize(ctx_, cutDistance, tol, maxIterations, &it), "particleFIREMinimize");
    return it;
  }
  void initVerticesOnParticles(const double* draws = nullptr) {
    ok(cr_init_vertices_on_particles(ctx_, draws), "initVerticesOnParticles");
  }

 private:
  cr_ctx* ctx_ = nullptr;
  std::vector<long> nvList_;
  std::vector<std::function<int(cr_ctx*)>> settings_;  // switches and parameters, in call order

  void create(const std::vector<long>& list) {
    int rc = cr_create((long)list.size(), list.data(), &ctx_);
    if (rc != CR_OK) throw Error("cr_create failed", rc);
    nvList_ = list;
    numParticles = (long)list.size();
    cr_get_num_vertices(ctx_, &numVertices);
  }
  void record(std::function<int(cr_ctx*)> set, const char* what) {
    ok(set(ctx_), what);
    settings_.push_back(std::move(set));
  }
  void replay() {
    for (auto& set : settings_) ok(set(ctx_), "replaying a setting on the re-sized system");
  }
  void checkSizes(long nv, long np, const char* what) {
    if (nv != numVertices || np != numParticles) throw Error(std::string(what) + ": size differs from the ring list", CR_EINVAL);
  }
  void ok(int rc, const char* what) {
    if (rc != CR_OK) throw Error(std::string(what) + ": " + cr_last_error(ctx_), rc);
  }
  std::vector<double> getv(int (*fn)(const cr_ctx*, double*), long n, const char* what) {
    std::vector<double> out((size_t)n);
    ok(fn(ctx_, out.data()), what);
    return out;
  }
  std::vector<double> get2(int (*fn)(const cr_ctx*, double*), const char* what) {
    std::vector<double> out((size_t)(2 * numVertices));
    ok(fn(ctx_, out.data()), what);
    return out;
  }
  double scalar(int (*fn)(cr_ctx*, double*), const char* what) {
    double v = 0;
    ok(fn(ctx_, &v), what);
    return v;
  }
};

}  // namespace cudaring
