// Reference-kernel host driver (oracle/_ref).
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's own `include/DPM2D.h` and `include/cudaKernel.cuh` (read from
// the reference checkout at build time, never copied) behind `shim.h`, giving
// a shared library whose entry points run the reference's kernels, unchanged,
// as host loops (`#pragma omp parallel for` over the kernel index).  It is
// used (a) to generate the golden fixtures under tests/golden/, (b) to pin the
// C restatement in oracle/oracle.c, and (c) as the timed CPU baseline.
//
// The reference's host orchestration lives in DPM2D.cu / Simulator.cu /
// FIRE.cu as Thrust calls; those few lines are restated here as host loops,
// each block citing the reference lines it follows.  The reference keeps one
// live model per process in `__constant__` symbols (cudaKernel.cuh:17-67);
// under the shim those become plain globals, so this driver is single-model
// too.
#include "shim.h"
#include "DPM2D.h"
#include "cudaKernel.cuh"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>
#include <omp.h>

thread_local crShimDim3 blockIdx, threadIdx, blockDim;

namespace {

#define REF_RUN(count, call)                                   \
  do {                                                         \
    const long n_ = (count);                                   \
    _Pragma("omp parallel for schedule(static)")               \
    for (long i_ = 0; i_ < n_; i_++) {                         \
      blockDim.x = 1; threadIdx.x = 0; blockIdx.x = i_;        \
      call;                                                    \
    }                                                          \
  } while (0)

struct RefModel {
  long np = 0, nv = 0;
  std::vector<long> nvList, firstVertex, particleId;
  std::vector<double> boxSize{1.0, 1.0};
  std::vector<double> pos, vel, force, energy, lastPos, rad, l0, theta0, a0;
  std::vector<double> area, perimeter, theta, length, particlePos, particleEnergy;
  std::vector<long> neighborList, maxNeighborList;
  long neighborListSize = 0;
  double ea = 1e5, el = 20, eb = 10, ec = 1, l1 = 0, l2 = 0;
  double LJcutoff = 0, LJecut = 0, LJfshift = 0, stiff = 0, extSq = 0, dt = 1e-3;
  double cutoff = 0, cutDistance = 1;
  long updateCount = 0;
  simControlStruct sc{};
  // FIRE state (FIRE.h:31-42)
  double a_start = 0.2, f_dec = 0.5, f_inc = 1.1, f_a = 0.99, fire_dt = 0, fire_dt_max = 0, fire_a = 0.2;
  long minStep = 20, numStep = 0;
  // rigid state
  std::vector<double> torque, particleForce, particleTorque, momentOfInertia;
  std::vector<double> particleVel, particleAngle, particleAngvel, particleLastPos, particleLastAngle;
  // soft-disk pre-packing state: particle radii, list, FIRE masses
  std::vector<double> particleRad, particleMass;
  std::vector<long> partNeighborList, partMaxNeighborList;
  long partNeighborListSize = 0;
};

RefModel M;

void sync_symbols() {
  d_simControl = M.sc;
  d_boxSizePtr = M.boxSize.data();
  d_nDim = 2;
  d_numParticles = M.np;
  d_numVertices = M.nv;
  d_numVertexPerParticle = M.np ? M.nvList[0] : 0;
  d_numVertexInParticleListPtr = M.nvList.data();
  d_firstVertexInParticleIdPtr = M.firstVertex.data();
  d_particleIdListPtr = M.particleId.data();
  d_dt = M.dt; d_rho0 = 1.0;
  d_ea = M.ea; d_el = M.el; d_eb = M.eb; d_ec = M.ec;
  d_l1 = M.l1; d_l2 = M.l2;
  d_LJcutoff = M.LJcutoff; d_LJecut = M.LJecut; d_LJfshift = M.LJfshift;
  d_stiff = M.stiff; d_extSq = M.extSq;
  d_neighborListPtr = M.neighborList.data();
  d_maxNeighborListPtr = M.maxNeighborList.data();
  d_neighborListSize = M.neighborListSize;
  d_partNeighborListPtr = M.partNeighborList.data();
  d_partMaxNeighborListPtr = M.partMaxNeighborList.data();
  d_partNeighborListSize = M.partNeighborListSize;
}

// DPM2D::calcNeighborList (DPM2D.cu:3479-3507): fill, run, grow to the next
// power of two and re-run when the list overflowed.
void calc_neighbor_list(double cutDistance) {
  std::fill(M.maxNeighborList.begin(), M.maxNeighborList.end(), 0L);
  std::fill(M.neighborList.begin(), M.neighborList.end(), -1L);
  sync_symbols();
  REF_RUN(M.nv, kernelCalcNeighborList(M.pos.data(), M.rad.data(), cutDistance));
  long maxNeighbors = -1;
  for (long v = 0; v < M.nv; v++) maxNeighbors = std::max(maxNeighbors, M.maxNeighborList[v]);
  if (maxNeighbors > M.neighborListSize) {
    M.neighborListSize = (long)std::pow(2, std::ceil(std::log2((double)maxNeighbors)));
    M.neighborList.assign(M.nv * M.neighborListSize, -1L);
    sync_symbols();
    REF_RUN(M.nv, kernelCalcNeighborList(M.pos.data(), M.rad.data(), cutDistance));
  }
}

// DPM2D::checkDisplacement (DPM2D.cu:1390-1406) with shift == false.
void check_neighbors() {
  std::vector<int> flag(M.nv, 0);
  sync_symbols();
  REF_RUN(M.nv, kernelCheckVertexDisplacement(M.pos.data(), M.lastPos.data(), flag.data(), M.cutoff));
  long sum = 0;
  for (int f : flag) sum += f;
  if (sum != 0) {
    calc_neighbor_list(M.cutDistance);
    M.lastPos = M.pos;
    M.updateCount += 1;
  }
}

// DPM2D::addSelfPropulsion (DPM2D.cu:1995-2035) with the per-ring angle
// increments supplied by the caller (the reference draws them from Thrust).
void add_self_propulsion(double driving, const double* dAngle) {
  const double PI_ = PI;
  for (long p = 0; p < M.np; p++) {
    double a = M.particleAngle[p] + dAngle[p];
    a = a + PI_;
    a = a - 2.0 * PI_ * std::floor(a / (2.0 * PI_));
    a = a - PI_;
    M.particleAngle[p] = a;
  }
  for (long v = 0; v < M.nv; v++) {
    long p = M.particleId[v];
    for (long dim = 0; dim < 2; dim++)
      M.force[v * 2 + dim] += driving * ((1 - dim) * std::cos(M.particleAngle[p]) + dim * std::sin(M.particleAngle[p]));
  }
}

// DPM2D::calcShapeForceEnergy + calcForceEnergyGPU (DPM2D.cu:1976-1993,
// 2058-2104) for periodic geometry.
void calc_force_energy() {
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticleShape(M.pos.data(), M.length.data(), M.theta.data(), M.area.data(), M.perimeter.data()));
  REF_RUN(M.np, kernelCalcParticlePositions(M.pos.data(), M.particlePos.data()));
  REF_RUN(M.nv, kernelCalcShapeForceEnergy(M.a0.data(), M.area.data(), M.particlePos.data(), M.l0.data(), M.theta0.data(),
                                           M.theta.data(), M.pos.data(), M.force.data(), M.energy.data()));
  std::fill(M.particleEnergy.begin(), M.particleEnergy.end(), 0.0);
  switch (M.sc.interactionType) {
    case simControlStruct::interactionEnum::vertexVertex:
      REF_RUN(M.nv, kernelCalcVertexInteraction(M.rad.data(), M.pos.data(), M.force.data(), M.energy.data()));
      break;
    case simControlStruct::interactionEnum::all:
      REF_RUN(M.nv, kernelCalcAllToAllVertexInteraction(M.rad.data(), M.pos.data(), M.force.data(), M.energy.data()));
      break;
    default:
      REF_RUN(M.nv, kernelCalcSmoothInteraction(M.rad.data(), M.pos.data(), M.force.data(), M.particleEnergy.data()));
      break;
  }
}

void update_vertex_vel(double timeStep) {
  sync_symbols();
  REF_RUN(M.nv, kernelUpdateVertexVel(M.vel.data(), M.force.data(), timeStep));
}
void update_vertex_pos(double timeStep) {
  sync_symbols();
  REF_RUN(M.nv, kernelUpdateVertexPos(M.pos.data(), M.vel.data(), timeStep));
}

}  // namespace

extern "C" {

int ref_num_threads(void) { return omp_get_max_threads(); }

int ref_create(long np, const long* nvList) {
  M = RefModel();
  M.np = np;
  M.nvList.assign(nvList, nvList + np);
  M.firstVertex.resize(np);
  long count = 0;
  for (long p = 0; p < np; p++) {  // DPM2D::initParticleIdList (DPM2D.cu:282-300)
    M.firstVertex[p] = count;
    for (long k = 0; k < nvList[p]; k++) M.particleId.push_back(p);
    count += nvList[p];
  }
  M.nv = count;
  M.pos.assign(2 * count, 0.0); M.vel.assign(2 * count, 0.0); M.force.assign(2 * count, 0.0);
  M.energy.assign(count, 0.0); M.lastPos.assign(2 * count, 0.0);
  M.rad.assign(count, 0.0); M.l0.assign(count, 0.0); M.theta0.assign(count, 0.0); M.a0.assign(np, 0.0);
  M.area.assign(np, 0.0); M.perimeter.assign(np, 0.0); M.theta.assign(count, 0.0); M.length.assign(count, 0.0);
  M.particlePos.assign(2 * np, 0.0); M.particleEnergy.assign(np, 0.0);
  M.neighborList.assign(count, -1L); M.maxNeighborList.assign(count, 0L); M.neighborListSize = 0;
  M.torque.assign(count, 0.0); M.particleForce.assign(2 * np, 0.0); M.particleTorque.assign(np, 0.0);
  M.momentOfInertia.assign(np, 0.0); M.particleVel.assign(2 * np, 0.0); M.particleAngle.assign(np, 0.0);
  M.particleAngvel.assign(np, 0.0); M.particleLastPos.assign(2 * np, 0.0); M.particleLastAngle.assign(np, 0.0);
  M.particleRad.assign(np, 0.0); M.particleMass.assign(2 * np, 1.0);
  M.partNeighborList.assign(np, -1L); M.partMaxNeighborList.assign(np, 0L); M.partNeighborListSize = 0;
  M.sc.simulationType = simControlStruct::simulationEnum::gpu;
  M.sc.geometryType = simControlStruct::geometryEnum::normal;
  M.sc.particleType = simControlStruct::particleEnum::passive;
  M.sc.shapeType = simControlStruct::shapeEnum::deformable;
  M.sc.noiseType = simControlStruct::noiseEnum::langevin;
  M.sc.potentialType = simControlStruct::potentialEnum::harmonic;
  M.sc.interactionType = simControlStruct::interactionEnum::vertexVertex;
  M.sc.neighborType = simControlStruct::neighborEnum::neighbor;
  M.sc.monomerType = simControlStruct::monomerEnum::harmonic;
  return 0;
}

long ref_num_vertices(void) { return M.nv; }

void ref_set_box(double lx, double ly) { M.boxSize = {lx, ly}; }

void ref_set_types(int potential, int interaction, int monomer, int particle) {
  M.sc.potentialType = (simControlStruct::potentialEnum)potential;
  M.sc.interactionType = (simControlStruct::interactionEnum)interaction;
  M.sc.monomerType = (simControlStruct::monomerEnum)monomer;
  M.sc.particleType = (simControlStruct::particleEnum)particle;
}

void ref_set_energy_costs(double ea, double el, double eb, double ec) { M.ea = ea; M.el = el; M.eb = eb; M.ec = ec; }

// DPM2D::setLJcutoff (DPM2D.cu:1923-1932)
void ref_set_lj_cutoff(double c) {
  M.LJcutoff = c;
  double ratio6 = 1 / std::pow(c, 6);
  M.LJecut = 4 * M.ec * (ratio6 * ratio6 - ratio6);
  M.LJfshift = 24 * M.ec * (2 * ratio6 - 1) * ratio6 / c;
}
void ref_get_lj_constants(double* out) { out[0] = M.LJecut; out[1] = M.LJfshift; }

void ref_set_attraction(double l1, double l2) { M.l1 = l1; M.l2 = l2; }
void ref_set_fene(double stiff, double ext) { M.stiff = stiff; M.extSq = ext * ext; }
void ref_set_time_step(double dt) { M.dt = dt; }

void ref_set_state(const double* pos, const double* vel, const double* rad, const double* l0,
                   const double* theta0, const double* a0) {
  if (pos) std::copy(pos, pos + 2 * M.nv, M.pos.begin());
  if (vel) std::copy(vel, vel + 2 * M.nv, M.vel.begin());
  if (rad) std::copy(rad, rad + M.nv, M.rad.begin());
  if (l0) std::copy(l0, l0 + M.nv, M.l0.begin());
  if (theta0) std::copy(theta0, theta0 + M.nv, M.theta0.begin());
  if (a0) std::copy(a0, a0 + M.np, M.a0.begin());
}

// DPM2D::setDisplacementCutoff (DPM2D.cu:1300-1329)
double ref_set_displacement_cutoff(double cutoff_, double size_) {
  switch (M.sc.potentialType) {
    case simControlStruct::potentialEnum::harmonic: M.cutDistance = 1; break;
    case simControlStruct::potentialEnum::lennardJones: M.cutDistance = M.LJcutoff; break;
    case simControlStruct::potentialEnum::wca: M.cutDistance = WCAcut; break;
    case simControlStruct::potentialEnum::adhesive: M.cutDistance = 1 + M.l2; break;
  }
  M.cutDistance += cutoff_;
  M.cutoff = cutoff_ * size_;
  return M.cutDistance;
}

void ref_calc_neighbor_list(double cutDistance) { calc_neighbor_list(cutDistance); }
void ref_reset_last_positions(void) { M.lastPos = M.pos; }
void ref_check_neighbors(void) { check_neighbors(); }
long ref_update_count(void) { return M.updateCount; }
long ref_neighbor_list_size(void) { return M.neighborListSize; }
void ref_get_neighbors(long* out) { std::copy(M.neighborList.begin(), M.neighborList.end(), out); }
void ref_get_max_neighbor_list(long* out) { std::copy(M.maxNeighborList.begin(), M.maxNeighborList.end(), out); }

void ref_calc_force_energy(void) { calc_force_energy(); }

// field ids: 0 pos, 1 vel, 2 force, 3 energy, 4 particleEnergy, 5 area,
// 6 perimeter, 7 theta, 8 length, 9 particlePos, 10 lastPos, 11 torque,
// 12 particleForce, 13 particleTorque, 14 particleAngle, 15 momentOfInertia,
// 16 particleVel, 17 particleAngvel
void ref_get(int field, double* out) {
  const std::vector<double>* src = nullptr;
  switch (field) {
    case 0: src = &M.pos; break;            case 1: src = &M.vel; break;
    case 2: src = &M.force; break;          case 3: src = &M.energy; break;
    case 4: src = &M.particleEnergy; break; case 5: src = &M.area; break;
    case 6: src = &M.perimeter; break;      case 7: src = &M.theta; break;
    case 8: src = &M.length; break;         case 9: src = &M.particlePos; break;
    case 10: src = &M.lastPos; break;       case 11: src = &M.torque; break;
    case 12: src = &M.particleForce; break; case 13: src = &M.particleTorque; break;
    case 14: src = &M.particleAngle; break; case 15: src = &M.momentOfInertia; break;
    case 16: src = &M.particleVel; break;   case 17: src = &M.particleAngvel; break;
    default: return;
  }
  std::copy(src->begin(), src->end(), out);
}

void ref_set_particle_state(const double* pPos, const double* pVel, const double* pAngle, const double* pAngvel) {
  if (pPos) std::copy(pPos, pPos + 2 * M.np, M.particlePos.begin());
  if (pVel) std::copy(pVel, pVel + 2 * M.np, M.particleVel.begin());
  if (pAngle) std::copy(pAngle, pAngle + M.np, M.particleAngle.begin());
  if (pAngvel) std::copy(pAngvel, pAngvel + M.np, M.particleAngvel.begin());
}

// DPM2D::getPotentialEnergy (DPM2D.cu:1062-1080)
double ref_potential_energy(void) {
  double e = 0;
  for (double x : M.energy) e += x;
  if (M.sc.interactionType == simControlStruct::interactionEnum::vertexSmooth ||
      M.sc.interactionType == simControlStruct::interactionEnum::cellSmooth) {
    for (double x : M.particleEnergy) e += x;
  } else if (M.sc.interactionType != simControlStruct::interactionEnum::vertexVertex) {
    return 0;
  }
  return e;
}

// DPM2D::getKineticEnergy (DPM2D.cu:1082-1087)
double ref_kinetic_energy(void) {
  double k = 0;
  for (double v : M.vel) k += v * v;
  return 0.5 * k;
}

// DPM2D::getMaxUnbalancedForce (DPM2D.cu:997-1005)
double ref_max_unbalanced_force(void) {
  double m = -1;
  for (double f : M.force) m = std::max(m, f * f);
  return std::sqrt(m);
}

// DPM2D::getTotalForceMagnitude (DPM2D.cu:986-994)
double ref_total_force_magnitude(void) {
  double s = 0;
  for (double f : M.force) s += f * f;
  return std::sqrt(s / (M.nv * 2));
}

// DPM2D::getPhi (DPM2D.cu:1202-1220): uses the current areas.
double ref_phi(void) {
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticleShape(M.pos.data(), M.length.data(), M.theta.data(), M.area.data(), M.perimeter.data()));
  double phi = 0;
  for (double a : M.area) phi += a;
  std::vector<double> vertexArea(M.np);
  REF_RUN(M.np, kernelCalcVertexArea(M.rad.data(), vertexArea.data()));
  double va = 0;
  for (double a : vertexArea) va += a;
  phi += PI * va;
  return phi / (M.boxSize[0] * M.boxSize[1]);
}

// NVE::integrate (Simulator.cu:206-212) with DPM2D::checkNeighbors and
// shift == false, repeated nsteps times.
void ref_nve_loop(long nsteps) {
  for (long s = 0; s < nsteps; s++) {
    update_vertex_vel(0.5 * M.dt);
    update_vertex_pos(M.dt);
    check_neighbors();
    calc_force_energy();
    update_vertex_vel(0.5 * M.dt);
  }
}

// NVERescale::integrate / injectKineticEnergy (Simulator.cu:215-238): scale
// every velocity by sqrt(Tinject / T), T = 2K / (2 Nv) (DPM2D.cu getTemperature),
// then one NVE step.
void ref_nve_rescale_loop(long nsteps, double Tinject) {
  for (long s = 0; s < nsteps; s++) {
    double vv = 0.0;
    for (long i = 0; i < 2 * M.nv; i++) vv += M.vel[i] * M.vel[i];
    const double T = vv / (2.0 * M.nv);
    const double scale = sqrt(Tinject / T);
    for (long i = 0; i < 2 * M.nv; i++) M.vel[i] *= scale;
    update_vertex_vel(0.5 * M.dt);
    update_vertex_pos(M.dt);
    check_neighbors();
    calc_force_energy();
    update_vertex_vel(0.5 * M.dt);
  }
}

// Langevin::integrate (Simulator.cu:23-30).  `xi` holds nsteps * np * 2
// standard-normal draws (the reference draws them from Thrust); step s uses
// xi[s*np*2 .. (s+1)*np*2).  noise = sqrt(2 T gamma / dt) (DPM2D.cu:3718).
// For active particles `dpsi` holds nsteps * np angle increments.
void ref_langevin_loop(long nsteps, double gamma, double noise, const double* xi,
                       double driving, const double* dpsi) {
  for (long s = 0; s < nsteps; s++) {
    update_vertex_vel(0.5 * M.dt);
    update_vertex_pos(M.dt);
    check_neighbors();
    calc_force_energy();
    if (M.sc.particleType == simControlStruct::particleEnum::active)
      add_self_propulsion(driving, dpsi + s * M.np);
    const double* r = xi + s * M.np * 2;
    for (long v = 0; v < M.nv; v++) {  // langevinAddThermostatForces (Simulator.cu:68-73)
      long p = M.particleId[v];
      for (long dim = 0; dim < 2; dim++)
        M.force[v * 2 + dim] += noise * r[p * 2 + dim] - gamma * M.vel[v * 2 + dim];
    }
    update_vertex_vel(0.5 * M.dt);
  }
}

// Brownian::integrate (Simulator.cu:147-177) and DrivenBrownian (180-203):
// v = (F + noise * xi_ring) / gamma; x += dt v.  xi == NULL gives the driven
// (noise-free) form.
void ref_brownian_loop(long nsteps, double gamma, double noise, const double* xi,
                       double driving, const double* dpsi) {
  for (long s = 0; s < nsteps; s++) {
    check_neighbors();
    calc_force_energy();
    if (M.sc.particleType == simControlStruct::particleEnum::active)
      add_self_propulsion(driving, dpsi + s * M.np);
    for (long v = 0; v < M.nv; v++) {
      long p = M.particleId[v];
      for (long dim = 0; dim < 2; dim++) {
        double f = M.force[v * 2 + dim];
        M.vel[v * 2 + dim] = xi ? (f + noise * xi[s * M.np * 2 + p * 2 + dim]) / gamma : f / gamma;
      }
    }
    update_vertex_pos(M.dt);
  }
}

// BAOAB::integrate (Simulator.cu:112-144); gammaFactor = exp(-gamma dt),
// noise = sqrt(1 - exp(-2 gamma dt)) sqrt(T) (DPM2D.cu:3722-3724).
void ref_baoab_loop(long nsteps, double gammaFactor, double noise, const double* xi) {
  for (long s = 0; s < nsteps; s++) {
    update_vertex_vel(0.5 * M.dt);
    update_vertex_pos(0.5 * M.dt);
    const double* r = xi + s * M.np * 2;
    for (long v = 0; v < M.nv; v++) {
      long p = M.particleId[v];
      for (long dim = 0; dim < 2; dim++)
        M.vel[v * 2 + dim] = gammaFactor * M.vel[v * 2 + dim] + noise * r[p * 2 + dim];
    }
    update_vertex_pos(0.5 * M.dt);
    check_neighbors();
    calc_force_energy();
    update_vertex_vel(0.5 * M.dt);
  }
}

// FIRE::initMinimizer (FIRE.cu:29-41)
void ref_fire_init(const double* p7, long minStep, long numStep) {
  M.a_start = p7[0]; M.f_dec = p7[1]; M.f_inc = p7[2]; M.f_a = p7[3];
  M.fire_dt = p7[4]; M.fire_dt_max = p7[5]; M.fire_a = p7[6];
  M.minStep = minStep; M.numStep = numStep;
}

void ref_fire_state(double* out) {
  out[0] = M.fire_dt; out[1] = M.fire_a; out[2] = (double)M.numStep;
}

// FIRE::minimizerVertexLoop (FIRE.cu:397-411) repeated nsteps times.
void ref_fire_loop(long nsteps) {
  for (long s = 0; s < nsteps; s++) {
    // checkFIREParams (FIRE.cu:338-371)
    double vDotF = 0;
    for (long i = 0; i < 2 * M.nv; i++) vDotF += M.vel[i] * M.force[i];
    if (vDotF > 0) {
      M.numStep++;
      if (M.numStep > M.minStep) {
        M.fire_dt = std::min(M.fire_dt * M.f_inc, M.fire_dt_max);
        M.fire_a *= M.f_a;
      }
    } else {
      M.numStep = 0;
      M.fire_dt = std::max(M.fire_dt * M.f_dec, M.fire_dt_max / 10);
      M.fire_a = M.a_start;
      double h = 0.5 * M.fire_dt;
      for (long i = 0; i < 2 * M.nv; i++) M.pos[i] -= h * M.vel[i];
      std::fill(M.vel.begin(), M.vel.end(), 0.0);
    }
    // updateVertexVelocity (FIRE.cu:320-335)
    for (long i = 0; i < 2 * M.nv; i++) M.vel[i] += 0.5 * M.fire_dt * M.force[i];
    // bendVertexVelocityTowardsForce (FIRE.cu:374-394)
    double vv = 0, ff = 0;
    for (long i = 0; i < 2 * M.nv; i++) { vv += M.vel[i] * M.vel[i]; ff += M.force[i] * M.force[i]; }
    if (ff > 0) {
      double ratio = std::sqrt(vv / ff);
      for (long i = 0; i < 2 * M.nv; i++) M.vel[i] = (1 - M.fire_a) * M.vel[i] + M.fire_a * M.force[i] * ratio;
    }
    // updateVertexPosition (FIRE.cu:302-317)
    for (long i = 0; i < 2 * M.nv; i++) M.pos[i] += M.fire_dt * M.vel[i];
    check_neighbors();
    calc_force_energy();
    for (long i = 0; i < 2 * M.nv; i++) M.vel[i] += 0.5 * M.fire_dt * M.force[i];
  }
}

// DPM2D::scaleVertices (DPM2D.cu:1802-1811) using the current particlePos.
void ref_scale_vertices(double scale) {
  sync_symbols();
  REF_RUN(M.np, kernelScaleVertexPositions(M.particlePos.data(), M.pos.data(), scale));
  for (double& a : M.a0) a *= scale * scale;
  for (double& a : M.area) a *= scale * scale;
  for (double& l : M.l0) l *= scale;
  for (double& r : M.rad) r *= scale;
}

void ref_calc_particle_positions(void) {
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticlePositions(M.pos.data(), M.particlePos.data()));
}

// DPM2D::calcRigidForceEnergy for vertexVertex (DPM2D.cu:2128-2142, 2106-2114,
// 2144-2166): vertex force + torque, moment of inertia, per-ring sums.
void ref_calc_rigid_force_energy(void) {
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticlePositions(M.pos.data(), M.particlePos.data()));
  REF_RUN(M.nv, kernelCalcVertexForceTorque(M.rad.data(), M.pos.data(), M.particlePos.data(), M.force.data(),
                                            M.torque.data(), M.energy.data()));
  REF_RUN(M.np, kernelCalcTorqueAndMomentOfInertia(M.pos.data(), M.particlePos.data(), M.force.data(), M.torque.data(),
                                                   M.momentOfInertia.data()));
  REF_RUN(M.np, kernelCalcParticleRigidForceEnergy(M.force.data(), M.torque.data(), M.energy.data(),
                                                   M.momentOfInertia.data(), M.particleForce.data(),
                                                   M.particleTorque.data(), M.particleEnergy.data()));
}

// DPM2D::translateVertices / rotateVertices (DPM2D.cu:1834-1848).
static void translate_rotate(void) {
  sync_symbols();
  REF_RUN(M.np, kernelTranslateVertices(M.particlePos.data(), M.particleLastPos.data(), M.pos.data()));
  REF_RUN(M.np, kernelRotateVertices(M.particlePos.data(), M.particleAngle.data(), M.particleLastAngle.data(), M.pos.data()));
}

// RigidNVE::integrate (Simulator.cu:316-371) repeated nsteps times.
void ref_rigid_nve_loop(long nsteps) {
  for (long s = 0; s < nsteps; s++) {
    M.particleLastPos = M.particlePos;
    M.particleLastAngle = M.particleAngle;
    for (long p = 0; p < M.np; p++) {
      for (long dim = 0; dim < 2; dim++) M.particleVel[p * 2 + dim] += 0.5 * M.dt * M.particleForce[p * 2 + dim];
      M.particleAngvel[p] += 0.5 * M.dt * M.particleTorque[p];
    }
    for (long p = 0; p < M.np; p++) {
      for (long dim = 0; dim < 2; dim++) M.particlePos[p * 2 + dim] += M.dt * M.particleVel[p * 2 + dim];
      M.particleAngle[p] += M.dt * M.particleAngvel[p];
    }
    translate_rotate();
    check_neighbors();
    ref_calc_rigid_force_energy();
    for (long p = 0; p < M.np; p++) {
      for (long dim = 0; dim < 2; dim++) M.particleVel[p * 2 + dim] += 0.5 * M.dt * M.particleForce[p * 2 + dim];
      M.particleAngvel[p] += 0.5 * M.dt * M.particleTorque[p];
    }
  }
}

// ------------------------------------------------------- soft-disk pre-packing
// The soft-particle stage before vertex FIRE (compressFIRE.cpp:53-90): random
// disks, particle neighbour list, particle forces, particle FIRE, vertices
// placed on the particle circles.

void ref_set_soft_particles(const double* pPos, const double* pRad) {
  if (pPos) std::copy(pPos, pPos + 2 * M.np, M.particlePos.begin());
  if (pRad) std::copy(pRad, pRad + M.np, M.particleRad.begin());
}

void ref_get_particle_radii(double* out) { std::copy(M.particleRad.begin(), M.particleRad.end(), out); }
void ref_get_geometry(double* out) {  // a0[np], l0[nv], rad[nv], box[2]
  std::copy(M.a0.begin(), M.a0.end(), out);
  std::copy(M.l0.begin(), M.l0.end(), out + M.np);
  std::copy(M.rad.begin(), M.rad.end(), out + M.np + M.nv);
  out[M.np + 2 * M.nv] = M.boxSize[0];
  out[M.np + 2 * M.nv + 1] = M.boxSize[1];
}

// DPM2D::calcParticleNeighborList (DPM2D.cu:3521-3545)
void ref_calc_particle_neighbor_list(double cutDistance) {
  std::fill(M.partMaxNeighborList.begin(), M.partMaxNeighborList.end(), 0L);
  std::fill(M.partNeighborList.begin(), M.partNeighborList.end(), -1L);
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticleNeighborList(M.particlePos.data(), M.particleRad.data(), cutDistance));
  long maxNeighbors = -1;
  for (long p = 0; p < M.np; p++) maxNeighbors = std::max(maxNeighbors, M.partMaxNeighborList[p]);
  if (maxNeighbors > M.partNeighborListSize) {
    M.partNeighborListSize = (long)std::pow(2, std::ceil(std::log2((double)maxNeighbors)));
    M.partNeighborList.assign(M.np * M.partNeighborListSize, -1L);
    sync_symbols();
    REF_RUN(M.np, kernelCalcParticleNeighborList(M.particlePos.data(), M.particleRad.data(), cutDistance));
  }
}
long ref_particle_neighbor_list_size(void) { return M.partNeighborListSize; }
void ref_get_particle_neighbors(long* out) { std::copy(M.partNeighborList.begin(), M.partNeighborList.end(), out); }
void ref_get_particle_max_neighbor_list(long* out) {
  std::copy(M.partMaxNeighborList.begin(), M.partMaxNeighborList.end(), out);
}

// DPM2D::calcParticleForceEnergy for periodic geometry (DPM2D.cu:3611-3622, 3582-3588)
void ref_calc_particle_force_energy(void) {
  sync_symbols();
  REF_RUN(M.np, kernelCalcParticleInteraction(M.particleRad.data(), M.particlePos.data(), M.particleForce.data(),
                                              M.particleEnergy.data()));
}

// DPM2D::getParticleMaxUnbalancedForce (DPM2D.cu:3633-3638)
double ref_particle_max_unbalanced_force(void) {
  double m = -1;
  for (double f : M.particleForce) m = std::max(m, f * f);
  return std::sqrt(m);
}
double ref_particle_potential_energy(void) {
  double e = 0;
  for (double x : M.particleEnergy) e += x;
  return e;
}
void ref_reset_particle_last_positions(void) { M.particleLastPos = M.particlePos; }
// DPM2D::getParticleMaxDisplacement (DPM2D.cu:1435-1441)
double ref_particle_max_displacement(void) {
  sync_symbols();
  std::vector<double> disp(M.np, 0.0);
  REF_RUN(M.np, kernelCalcParticleDisplacement(M.particlePos.data(), M.particleLastPos.data(), disp.data()));
  double m = -1;
  for (double d : disp) m = std::max(m, d);
  return m;
}

// DPM2D::initFIRE (DPM2D.cu:3660-3674) + DPM2D::setParticleMassFIRE (:3676-3684)
void ref_particle_fire_init(const double* p7, long minStep, long numStep) {
  ref_fire_init(p7, minStep, numStep);
  M.particleLastPos = M.particlePos;
  for (long p = 0; p < M.np; p++)
    for (long dim = 0; dim < 2; dim++) M.particleMass[p * 2 + dim] = PI / (M.particleRad[p] * M.particleRad[p]);
}

// FIRE::minimizerParticleLoop (FIRE.cu:156-171) repeated nsteps times, with
// FIRE::updateParticlePositionAndVelocity (:45-71), updateParticleVelocity
// (:74-97) and bendParticleVelocityTowardsForce (:100-141).  The reference's
// checkParticleNeighbors call inside the loop rebuilds the *vertex* list
// (DPM2D.cu:1425-1433), which no particle force reads; it is left out.
void ref_particle_fire_loop(long nsteps) {
  const long n2 = 2 * M.np;
  for (long s = 0; s < nsteps; s++) {
    for (long p = 0; p < M.np; p++) {
      double totalForce = 0;
      for (long dim = 0; dim < 2; dim++) {
        const long i = p * 2 + dim;
        M.particleVel[i] += 0.5 * M.fire_dt * M.particleForce[i] / M.particleMass[i];
        M.particlePos[i] += M.fire_dt * M.particleVel[i];
        totalForce += M.particleForce[i];
      }
      if (totalForce == 0)
        for (long dim = 0; dim < 2; dim++) M.particleVel[p * 2 + dim] = 0;
    }
    ref_calc_particle_force_energy();
    for (long p = 0; p < M.np; p++) {
      double totalForce = 0;
      for (long dim = 0; dim < 2; dim++) {
        const long i = p * 2 + dim;
        M.particleVel[i] += 0.5 * M.fire_dt * M.particleForce[i] / M.particleMass[i];
        totalForce += M.particleForce[i];
      }
      if (totalForce == 0)
        for (long dim = 0; dim < 2; dim++) M.particleVel[p * 2 + dim] = 0;
    }
    double vDotF = 0;
    for (long i = 0; i < n2; i++) vDotF += M.particleVel[i] * M.particleForce[i];
    if (vDotF < 0) {
      std::fill(M.particleVel.begin(), M.particleVel.end(), 0.0);
      M.numStep = 0;
      M.fire_dt = std::max(M.fire_dt * M.f_dec, M.fire_dt_max / 10);
      M.fire_a = M.a_start;
    } else if (M.numStep > M.minStep) {
      M.fire_dt = std::min(M.fire_dt * M.f_inc, M.fire_dt_max);
      M.fire_a *= M.f_a;
    }
    double vv = 0, ff = 0;
    for (long i = 0; i < n2; i++) { vv += M.particleVel[i] * M.particleVel[i]; ff += M.particleForce[i] * M.particleForce[i]; }
    if (ff == 0) {
      std::fill(M.particleVel.begin(), M.particleVel.end(), 0.0);
    } else {
      const double ratio = std::sqrt(vv / ff);
      const double a = M.fire_a;
      for (long i = 0; i < n2; i++) M.particleVel[i] = (1 - a) * M.particleVel[i] + a * M.particleForce[i] * ratio;
    }
    M.numStep++;
  }
}

// compressFIRE.cpp:66-78: particle FIRE to max |F| <= tol, the particle list
// rebuilt whenever 3 * (largest displacement since the last build) exceeds
// (1 + cutDistance) * (smallest particle radius).  Returns the iterations.
long ref_particle_fire_minimize(double cutDistance, double tol, long maxIterations) {
  double minRad = 1.0;  // DPM2D::getMinParticleSigma (DPM2D.cu:766-768)
  for (double r : M.particleRad) minRad = std::min(minRad, r);
  const double cutoff = (1 + cutDistance) * minRad;
  long iteration = 0;
  while (ref_particle_max_unbalanced_force() > tol && iteration != maxIterations) {
    ref_particle_fire_loop(1);
    if (3 * ref_particle_max_displacement() > cutoff) {
      ref_calc_particle_neighbor_list(cutDistance);
      M.particleLastPos = M.particlePos;
    }
    iteration += 1;
  }
  return iteration;
}

// DPM2D::initVerticesOnParticles (DPM2D.cu:1678-1691) with the 2 * nv
// drand48() draws supplied in call order (x then y of each vertex).
void ref_init_vertices_on_particles(const double* draws) {
  for (long v = 0; v < M.nv; v++) {
    const long p = M.particleId[v];
    const long n = M.nvList[p];
    const double rad = std::sqrt((2. * M.a0[p]) / (n * std::sin(2. * PI / n)));
    M.pos[v * 2] = rad * std::cos((2. * PI * v) / n) + M.particlePos[p * 2] + 1e-03 * M.l0[v] * draws[2 * v];
    M.pos[v * 2 + 1] = rad * std::sin((2. * PI * v) / n) + M.particlePos[p * 2 + 1] + 1e-03 * M.l0[v] * draws[2 * v + 1];
  }
  std::fill(M.vel.begin(), M.vel.end(), 0.0);
  std::fill(M.force.begin(), M.force.end(), 0.0);
  std::fill(M.energy.begin(), M.energy.end(), 0.0);
}

// DPM2D::getPreferredPhi (DPM2D.cu:1222-1238) for the periodic box.
static double preferred_phi(void) {
  double phi = 0;
  for (double a : M.a0) phi += a;
  std::vector<double> vertexArea(M.np, 0.0);
  sync_symbols();
  REF_RUN(M.np, kernelCalcVertexArea(M.rad.data(), vertexArea.data()));
  double va = 0;
  for (double x : vertexArea) va += x;
  phi += PI * va;
  return phi / (M.boxSize[0] * M.boxSize[1]);
}

// DPM2D::getPreferredPhi (DPM2D.cu:1222-1238), exported.
double ref_preferred_phi(void) { return preferred_phi(); }

// DPM2D::setRandomParticles (DPM2D.cu:1601-1629) with the drand48() stream
// of srand48(seed): erand48 on the state srand48 would set.
void ref_set_random_particles(double phi0, double extraRad, long seed) {
  unsigned short xs[3] = {0x330E, (unsigned short)(seed & 0xFFFF), (unsigned short)((seed >> 16) & 0xFFFF)};
  const double scale = std::sqrt(preferred_phi() / phi0);
  M.boxSize = {1.0, 1.0};
  for (long p = 0; p < M.np; p++) {
    M.a0[p] /= (scale * scale);
    M.area[p] = M.a0[p];
    for (long dim = 0; dim < 2; dim++) M.particlePos[p * 2 + dim] = M.boxSize[dim] * erand48(xs);
    M.particleRad[p] = extraRad * std::sqrt((2. * M.a0[p]) / (M.nvList[p] * std::sin(2. * PI / M.nvList[p])));
  }
  for (long v = 0; v < M.nv; v++) {
    M.l0[v] /= scale;
    M.rad[v] /= scale;
  }
}

// the drand48() draws that follow n earlier ones on srand48(seed)
void ref_drand48_stream(long seed, long skip, long n, double* out) {
  unsigned short xs[3] = {0x330E, (unsigned short)(seed & 0xFFFF), (unsigned short)((seed >> 16) & 0xFFFF)};
  for (long i = 0; i < skip; i++) erand48(xs);
  for (long i = 0; i < n; i++) out[i] = erand48(xs);
}

}  // extern "C"
