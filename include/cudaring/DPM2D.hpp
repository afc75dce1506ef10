// cudaring/DPM2D.hpp -- header-only C++ facade over include/cudaring.h.
//
// Reproduces the hot-path member functions of the reference's DPM2D class
// (include/DPM2D.h of farceri/cudaRing) so driver code written against it
// (runNVE.cpp, compressFIRE.cpp style loops) compiles with few changes:
//   cudaring::DPM2D dpm(numVertexInParticleList);
//   dpm.setBoxSize(box); dpm.setEnergyCosts(ea, el, eb, ec); ...
//   double cut = dpm.setDisplacementCutoff(0.5, 2 * dpm.getMeanVertexRadius());
//   dpm.calcNeighbors(cut); dpm.calcForceEnergy(); dpm.initNVE(T, false);
//   while (step != maxStep) { dpm.NVELoop(); ... }
// Host vectors are std::vector<double> / std::vector<long> in the reference's
// layout.  Failing calls throw cudaring::Error carrying the status code.
#pragma once
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
  explicit DPM2D(const std::vector<long>& numVertexInParticleList) {
    int rc = cr_create((long)numVertexInParticleList.size(), numVertexInParticleList.data(), &ctx_);
    if (rc != CR_OK) throw Error("cr_create failed", rc);
    numParticles = (long)numVertexInParticleList.size();
    cr_get_num_vertices(ctx_, &numVertices);
  }
  ~DPM2D() {
    if (ctx_) cr_destroy(ctx_);
  }
  DPM2D(const DPM2D&) = delete;
  DPM2D& operator=(const DPM2D&) = delete;

  long numParticles = 0, numVertices = 0;
  cr_ctx* handle() { return ctx_; }

  // switches (include/DPM2D.h:231-249)
  void setPotentialType(int v) { ok(cr_set_potential_type(ctx_, v), "setPotentialType"); }
  void setInteractionType(int v) { ok(cr_set_interaction_type(ctx_, v), "setInteractionType"); }
  void setMonomerType(int v) { ok(cr_set_monomer_type(ctx_, v), "setMonomerType"); }
  void setParticleType(int v) { ok(cr_set_particle_type(ctx_, v), "setParticleType"); }
  void setNoiseType(int v) { ok(cr_set_noise_type(ctx_, v), "setNoiseType"); }

  // parameters
  void setBoxSize(const std::vector<double>& b) { ok(cr_set_box_size(ctx_, b.data()), "setBoxSize"); }
  void setEnergyCosts(double ea, double el, double eb, double ec) {
    ok(cr_set_energy_costs(ctx_, ea, el, eb, ec), "setEnergyCosts");
  }
  void setLJcutoff(double c) { ok(cr_set_lj_cutoff(ctx_, c), "setLJcutoff"); }
  void setAttractionConstants(double l1, double l2) { ok(cr_set_attraction_constants(ctx_, l1, l2), "setAttractionConstants"); }
  void setFENEconstants(double s, double e) { ok(cr_set_fene_constants(ctx_, s, e), "setFENEconstants"); }
  double setTimeStep(double dt) {
    ok(cr_set_time_step(ctx_, dt), "setTimeStep");
    return dt;
  }
  void setSelfPropulsionParams(double f0, double taup) {
    ok(cr_set_self_propulsion_params(ctx_, f0, taup), "setSelfPropulsionParams");
  }

  // state
  void setVertexPositions(const std::vector<double>& a) { ok(cr_set_vertex_positions(ctx_, a.data()), "setVertexPositions"); }
  std::vector<double> getVertexPositions() { return get2(cr_get_vertex_positions, "getVertexPositions"); }
  void setVertexVelocities(const std::vector<double>& a) { ok(cr_set_vertex_velocities(ctx_, a.data()), "setVertexVelocities"); }
  std::vector<double> getVertexVelocities() { return get2(cr_get_vertex_velocities, "getVertexVelocities"); }
  std::vector<double> getVertexForces() { return get2(cr_get_vertex_forces, "getVertexForces"); }
  void setVertexRadii(const std::vector<double>& a) { ok(cr_set_vertex_radii(ctx_, a.data()), "setVertexRadii"); }
  void setRestAreas(const std::vector<double>& a) { ok(cr_set_rest_areas(ctx_, a.data()), "setRestAreas"); }
  void setRestLengths(const std::vector<double>& a) { ok(cr_set_rest_lengths(ctx_, a.data()), "setRestLengths"); }
  void setRestAngles(const std::vector<double>& a) { ok(cr_set_rest_angles(ctx_, a.data()), "setRestAngles"); }

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
  void ok(int rc, const char* what) {
    if (rc != CR_OK) throw Error(std::string(what) + ": " + cr_last_error(ctx_), rc);
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
