// Host-side declarations of the kernel launchers (internal to libcudaring).
#pragma once
#include <cuda_runtime.h>

#include "cr_common.cuh"

namespace cr {

struct StepArgs;

struct LaunchCfg {
  cudaStream_t stream;
  int grid;    // number of tiles / CTAs
  int lanes;   // lanes per vertex in the pair phase (1, 2, 4, 8)
  int precision = CR_PRECISION_FP64;  // CR_PRECISION_* (deformable tile kernel)
  bool pdl = false;   // programmatic dependent launch (inside step graphs)
  int block = 0;      // batch tiles: threads per CTA (0: the lane count's default, batch_tile_block)
};

// cr_tile.cu
void launch_tile(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                 const StepArgs& s);
int tile_vertices(int lanes);
// cr_tile_batch.cu: the same kernel over the tiles of many systems (tile.x =
// system, s.bsys the per-system table).  Tile shapes (lanes per vertex,
// threads per CTA): (1, 128), (1, 192), (2, 128), (2, 192), (4, 256); a
// tile holds threads / lanes vertices.
int batch_tile_block(int lanes, int block);   // the shape's CTA size (0: the lane count's default), or 0 if unsupported
void launch_tile_batch(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                       const StepArgs& s);
// Multi-step kernel (k_tile_steps): up to s.persist_max middle steps per
// launch with grid barriers between them; one or two lanes per vertex.  The
// grid must be resident at once: tile_steps_max_blocks() CTAs at most.
using TileStepsFn = void (*)(SysParams, SysArrays, StepArgs);
TileStepsFn tile_steps_fn_fp64(int pot, int inter, int lanes);
TileStepsFn tile_steps_fn_mixed(int pot, int inter, int lanes);
int tile_steps_max_blocks(int pot, int inter, int lanes, int precision);
cudaError_t launch_tile_steps(const LaunchCfg& c, int pot, int inter, const SysParams& p, const SysArrays& a,
                              const StepArgs& s);
// cr_tile_mixed.cu (expects p with its FP32 constants filled)
void launch_tile_mixed(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                       const StepArgs& s);

// cr_misc.cu
struct FireParams {
  double a_start, f_dec, f_inc, f_a, dt_max;
  long long min_step;
  double tol;
};
void launch_drift(cudaStream_t st, const SysParams& p, const SysArrays& a, const StepArgs& s, int nblocks);
void launch_fire_pre(cudaStream_t st, const SysParams& p, const SysArrays& a, const StepArgs& s,
                     const FireParams& fp, double* fire_state, int nblocks);
void launch_reduce(cudaStream_t st, int nv, int np, const double2* vel, const double2* force, const double* energy,
                   const double* p_energy, int use_p_energy, double* partials, DevStatus* status, int nblocks);
void launch_affine_vel(cudaStream_t st, int n, double2* vel, double scale, double2 shift);
void launch_inject_ke(cudaStream_t st, int nv, const int* ring_of, double2* vel, double amplitude,
                      unsigned long long seed, unsigned long long stream);
void launch_scale_vertices(cudaStream_t st, int nv, int np, const int* ring_of, const double2* ppos, double2* pos,
                           double* a0, double* area, double* l0, double* rad, double scale);
void launch_advance_angles(cudaStream_t st, int np, double* angle, double amp, unsigned long long seed,
                           unsigned long long stream);
void launch_vertex_area(cudaStream_t st, int np, const int* ring_first, const int* ring_nv, const double* rad,
                        double* out);

// cr_rigid.cu
struct RigidArgs {
  double2* p_vel;      // ring velocity (half-step velocity between ops of a sequence)
  double* p_angle;     // ring orientation angle
  double* p_angvel;    // ring angular velocity
  double2* p_force;    // ring force (sum over vertices, plus thermostat / propulsion terms)
  double* p_torque;    // ring torque / moment of inertia (angular acceleration)
  double* p_moi;       // ring moment of inertia (unit vertex mass)
  double* v_torque;    // per-vertex torque about the centroid
  double* sp_angle;    // self-propulsion angle of active rigid rings
};
void launch_rigid(const LaunchCfg& c, int pot, int mode, const SysParams& p, const SysArrays& a, const StepArgs& s,
                  const RigidArgs& r);
void launch_rigid_drift(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s,
                        const RigidArgs& r);
void launch_rigid_inject(cudaStream_t st, int np, double2* p_vel, double amp, unsigned long long seed,
                         unsigned long long stream);

// cr_diff.cu: forces and energies in hyper-dual arithmetic (cr_hd.cuh)
struct DiffArgs {
  SysParams p;
  const double2* pos;
  const double2* t1;   // position tangent e1 (nullable)
  const double2* t2;   // position tangent e2 (nullable)
  double s1, s2;       // box tangents: L (1 + s1 e1 + s2 e2)
  double pe1[3], pe2[3];  // tangents of ea, el, eb
  double c1, c2;       // tangents of ln(calA0): l0, rad ~ sqrt(calA0)
  const double* rad;
  const double* l0;
  const double* theta0;
  const double* a0;
  const int2* vtopo;
  const int* nbr;
  const int* nbr_cnt;
  int nbr_cap;
  double* force_out;   // [nv][8]: Fx (a, b, c, d), Fy (a, b, c, d)
  double* energy_out;  // [nv][4]
  double* ring_area;   // [np][4] scratch: hyper-dual ring areas (filled by the launch)
  const int* skip;     // nullable: nothing is evaluated while *skip != 0
  // 1: each thread seeds its own vertex only (x tangent e1, y tangent e2;
  // t1, t2 null), so the e1 and e2 parts of the force on v are the columns
  // of -H_vv, the vertex's 2 x 2 diagonal block of the Hessian
  int diag;
};
void launch_diff(cudaStream_t st, int pot, int inter, const DiffArgs& g, const int* ring_first, const int* ring_nv);
// Device-resident conjugate-gradient iterations on the projected Hessian
// (cr_hessian_solve): every scalar stays on the device, so a run of
// iterations is one captured graph with no host synchronisation.
struct CgState {
  double rr, bb, tol;     // |r|^2, |b|^2, relative tolerance
  double alpha, beta;     // step and direction coefficients of the iteration
  double mx, my;          // mean of H p over the vertices (removed: translations)
  long long iters, max_iters;
  int done;               // converged, iteration limit, or non-positive curvature
  int bad;                // 1: a non-positive curvature p.Hp was met
  double rz;              // r.z with z = M^-1 r (the preconditioned residual; = |r|^2 without one)
  double zx, zy;          // mean of z over the vertices (removed: translations)
};
struct CgArgs {
  int nv;
  double* x;
  double* r;
  double* p;
  double* hp;
  const double* fhd;  // hyper-dual forces of the H p launch
  CgState* st;
  double* partials;   // [nblk][8]
  int nblk;
  double* z;          // preconditioned residual M^-1 r
  const double* minv; // [nv][3] inverse diagonal blocks (a, b, d of [[a, b], [b, d]]); null: no preconditioner
};
void launch_cg_iteration(cudaStream_t st, const CgArgs& a);
// Block-Jacobi preconditioner from a diag-mode hyper-dual launch: minv[v] the
// inverse of the vertex's 2 x 2 Hessian block (its positive part where the
// block is not positive definite); z = M^-1 r.
void launch_cg_prec(cudaStream_t st, int nv, const double* fhd, double* minv);
void launch_cg_apply(cudaStream_t st, int nv, const double* minv, const double* r, double* z);
int cg_blocks(int nv);
void launch_dot_partials(cudaStream_t st, int n, const double* a, const double* b, double* out, int nblocks);
void launch_axpby(cudaStream_t st, int n, double a, const double* x, double b, double* y);
void launch_extract_hv(cudaStream_t st, int nv, const double* fhd, double* hv);
void launch_sub_mean(cudaStream_t st, int nv, double* x, double mx, double my);

// cr_nbr.cu
// Vertex ids a cell bucket of the one-launch build holds; a build that finds
// a fuller cell sorts by cell instead (same list).
constexpr int kCellBucket = 16;
// ints of the cell_cnt allocation for the bucket form over `ncells` cells
inline size_t cell_count_words(int ncells) { return 2 * (size_t)ncells + 2; }
struct CellGrid {
  int ncx, ncy;       // cells per dimension (>= 3 each), or 0 for brute force
  double cx, cy;      // cell sizes
};
struct NbrArgs {
  const double2* pos;
  const double* rad;
  const int* ring_of;
  int* nbr;           // [cap][nv]
  int* nbr_cnt;
  int cap;
  double cut_distance;
  double2* last_pos;  // set to pos by the build
  // cell scratch
  int* cell_of;
  int* slot;
  int* cell_cnt;      // [ncells], zero between builds
  int* cell_start;    // [ncells + 1]
  int* cell_vid;      // [nv]
  double2* cell_pos;  // [nv]
  double* cell_rad;   // [nv]
  int* cell_ring;     // [nv]
  // optional companion list: per entry the packed ring-predecessor offsets
  // of the neighbour (see SysArrays::nbr_pq); written when nbr_pq is set
  const int* pq_pack = nullptr;  // [nv] per-vertex packed offsets
  int* nbr_pq = nullptr;         // [cap][nv]
  int* cell_pq = nullptr;        // [nv] cell-sorted copy of pq_pack
  DevStatus* status;
  int count_op;       // 1: the build is one op of a step sequence (ops_done += 1)
  int count_update;   // 1: a displacement-triggered rebuild (DPM2D::updateCount += 1)
  int* block_sum = nullptr;  // [grid] per-CTA cell totals of the one-launch build
  // bucket form of the one-launch build (all set, or bucket null): cell_cnt
  // then holds two count arrays of cell_stride entries and two control words
  // (which array is current, and whether a cell overflowed its bucket); each
  // cell's bucket holds up to kCellBucket members, with their data
  int* bucket = nullptr;           // [ncells][kCellBucket] vertex ids
  double2* bucket_pos = nullptr;   // positions
  double* bucket_rad = nullptr;    // radii
  int* bucket_ring = nullptr;      // rings
  int* bucket_pq = nullptr;        // packed ring-predecessor offsets (with nbr_pq)
  int cell_stride = 0;
  // 1: the pair's radius sum is twice the listing vertex's own radius (the
  // particle list rule of kernelCalcParticleNeighborList, whose
  // extractOtherParticle returns the particle's own radius,
  // include/cudaKernel.cuh:289-296, 1765-1789)
  int self_rsum = 0;
};
void launch_nbr_build(cudaStream_t st, const SysParams& p, const CellGrid& g, const NbrArgs& n);
// The whole build in one launch of `blocks` CTAs (at most nbr_fused_max_blocks()).
// force = 0: return at once unless the status block armed a rebuild (and no
// abort or convergence is pending), so it can follow every step op in a graph.
// pdl: programmatic dependent launch after the step kernel (inside graphs).
void launch_nbr_fused(cudaStream_t st, const SysParams& p, const CellGrid& g, const NbrArgs& n, int blocks,
                      int force, bool pdl = false);
// CTAs of the one-launch build that the current device holds at once.
int nbr_fused_max_blocks();
// Grid of the one-launch build for nv vertices.
int nbr_fused_blocks(int nv, int max_blocks);

// ------------------------------------------------ soft-disk pre-packing (cr_soft.cu)
// FIRE scalars of the particle minimiser (FIRE.h:31-42) plus the bend that the
// last force op computed and the next move op applies.
struct SoftFire {
  double dt, dt_max, a, a_start, f_dec, f_inc, f_a;
  double ratio;    // sqrt(|v|^2 / |F|^2) of the pending bend
  double tol;      // convergence: max |F_d| <= tol
  double max_f2;   // max F_d^2 after the last force op
  long long min_step, num_step, iters;
  int zero;        // the pending bend zeroes every velocity
  int pending;     // a bend is waiting
  int converged;
  int pad;
};
struct SoftArgs {
  double2* pos;       // particle positions
  double2* vel;
  double2* force;
  double* energy;     // per particle
  const double* rad;  // particle radii
  const int* nbr;     // [cap][np] slot-major particle list
  const int* cnt;
  int cap;
  double2* last_pos;  // positions at the last list build
  double cutoff;      // rebuild when 3 |x - last| > cutoff
  SoftFire* fire;
  DevStatus* status;
  double* partials;   // [blocks][4]
};
int soft_blocks(int np);
void launch_soft_force(cudaStream_t st, int pot, const SysParams& p, const SoftArgs& a, bool fire);
void launch_soft_move(cudaStream_t st, const SysParams& p, const SoftArgs& a, int check);
void launch_soft_bend(cudaStream_t st, int np, const SoftArgs& a);
void launch_soft_vertices(cudaStream_t st, int nv, const int* ring_of, const int* ring_nv, const double* a0,
                          const double* l0, const double2* ppos, const double* draws, unsigned long long seed,
                          unsigned long long stream, double2* pos, double2* vel, double2* force, double* energy);
// building blocks shared with the batched build (cr_batch.cu)
void launch_cell_scan(cudaStream_t st, int ncells, int* cell_cnt, int* cell_start);
void launch_cell_sort(cudaStream_t st, int ncells, int nv, const NbrArgs& n);

}  // namespace cr
