// Shared device definitions for the cudaRing-B200 hot path (sm_100a).
//
// Layout in HBM (one system):
//   pos, vel, force : double2[Nv]  ring-contiguous, counter-clockwise rings
//   rad, l0, theta0 : double[Nv];  a0 : double[Np]
//   ring_of         : int32[Nv];   ring_first, ring_nv : int32[Np]
//   pp_of           : int2[Nv]     (previous, second-previous vertex of the ring)
//   vtopo           : int2[Nv]     (ring, k | nv << 16)
//   nbr             : int32[cap][Nv] column-major (slot-major) neighbour list,
//                     nbr_cnt int32[Nv]; vertex ids in internal order
//   nbr_pq          : int32[cap][Nv] packed ring-predecessor offsets of each
//                     listed neighbour (lets a gather issue the neighbour's
//                     own and its predecessors' loads together)
//   tiles           : int4[T]      (first ring, end ring, first vertex, end vertex)
// All arithmetic on the plain path is FP64, as in the reference.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cudaring.h"

namespace cr {

// Programmatic dependent launch.  A kernel launched with launch_k(pdl = true)
// may be scheduled while the kernel before it in the stream is finishing;
// pdl_wait() blocks until that kernel has completed and its writes are
// visible (a no-op for an ordinary launch), so it comes before any read of
// data the previous kernel writes.  pdl_trigger() lets the next kernel be
// scheduled early; without it the next kernel starts when this one exits.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                            Args&&... args) {
  if (!pdl) {
    kernel<<<grid, block, 0, st>>>(static_cast<KArgs>(args)...);
    return cudaSuccess;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

constexpr double kPi = 3.141592653589793238462643383279502884197;
constexpr double kWCAcut = 1.122462048;  // include/defs.h:17 of the reference

enum Pot : int { POT_HARMONIC = 0, POT_LJ = 1, POT_ADHESIVE = 2, POT_WCA = 3 };
enum Inter : int { INT_VV = 0, INT_SMOOTH = 1 };

// Scalars of one system, passed by value to every kernel (__grid_constant__).
struct SysParams {
  int nv;        // vertices
  int np;        // rings
  double lx, ly, inv_lx, inv_ly;
  double ea, el, eb, ec, l1, l2;
  double lj_cutoff, lj_ecut, lj_fshift;
  double stiff, ext_sq;
  int monomer;   // 0 harmonic, 1 FENE
  int potential; // Pot
  // FP32 copies of the pair constants for the mixed-precision pair terms,
  // filled from the FP64 values when a mixed-precision kernel is launched
  float f_ec, f_l1, f_l2, f_lj_cutoff, f_lj_ecut, f_lj_fshift;
  // mixed precision: a smooth unit whose vertex lies within f_near * radSum
  // of its segment is evaluated in FP64 (0: none)
  float f_near;
};

inline SysParams with_f32_constants(SysParams p) {
  p.f_ec = (float)p.ec;
  p.f_l1 = (float)p.l1;
  p.f_l2 = (float)p.l2;
  p.f_lj_cutoff = (float)p.lj_cutoff;
  p.f_lj_ecut = (float)p.lj_ecut;
  p.f_lj_fshift = (float)p.lj_fshift;
  // Near-contact units of the steep potentials carry the FP32 error: around
  // the Lennard-Jones minimum (radSum * 2^(1/6)) the force falls by ~57
  // epsilon/sigma per sigma and 2 r^12 - r^6 cancels, so one FP32 rounding of
  // the distance or of r^6 moves a unit force by ~1e-6 of the net force.
  // Units closer than 1.2 radSum are therefore evaluated in FP64 (every WCA
  // unit: its whole range is that steep); harmonic and adhesive forces are
  // linear in the overlap and stay FP32.
  p.f_near = p.potential == 1 ? 1.2f : (p.potential == 3 ? 1.2f : 0.0f);
  return p;
}

// Device pointers of one system (internal order).
struct SysArrays {
  const double2* pos;   // read positions for this evaluation
  const double* rad;
  const double* l0;
  const double* theta0;
  const double* a0;
  const int* ring_of;
  const int* ring_first;
  const int* ring_nv;
  const int2* pp_of;
  const int* nbr;       // [cap][nv]
  const int* nbr_cnt;
  const int4* tiles;
  int nbr_cap;
  // per vertex: {ring, k | nv << 16}, k the vertex's index inside its ring
  const int2* vtopo;
  // per list entry (same [cap][nv] layout as nbr): the neighbour j's ring
  // predecessors as offsets from j, (prev(j) - j) in the low 16 bits and
  // (prev(prev(j)) - j) in the high 16 bits, both signed
  const int* nbr_pq;
};

__host__ __device__ inline int pq_pack_of(int dq, int dqq) { return (dq & 0xffff) | (int)((unsigned)dqq << 16); }
__device__ __forceinline__ int pq_first(int pk) { return (int)(short)(pk & 0xffff); }
__device__ __forceinline__ int pq_second(int pk) { return pk >> 16; }

// Minimum-image difference, reference pbcDistance (include/cudaKernel.cuh:70-74)
// with delta/size replaced by delta*(1/size) and round-half-away by
// round-half-even (one rounding instruction); the two agree except when
// delta/size lies within one ulp of a half-integer, i.e. |delta| ~ L/2, far
// outside every interaction and list range.
__device__ __forceinline__ double pbc1(double d, double size, double inv) {
  return d - size * rint(d * inv);
}
// B: anything with lx, ly, inv_lx, inv_ly (SysParams, or Box for one system
// of a batch)
template <class B>
__device__ __forceinline__ double2 pbc2(const B& p, double2 a, double2 b) {
  return make_double2(pbc1(a.x - b.x, p.lx, p.inv_lx), pbc1(a.y - b.y, p.ly, p.inv_ly));
}

// Periodic box of one system of a batch.
struct Box {
  double lx, ly, inv_lx, inv_ly;
};

// Pair magnitude for the vertex-vertex path: returns gradMultiple g (force on
// "this" is g * delta / d) and sets the half-pair energy.  Restates
// calcContactInteraction / calcLJInteraction / calcAdhesiveInteraction /
// calcWCAInteraction (include/cudaKernel.cuh:531-668) and, for the smooth
// path, calcGradMultipleAndEnergy (:806-858); the two differ only in how
// ratio^12 is formed (pow(r,6)^2 vs pow(r,12)), which is a rounding-level
// difference, so one form serves both.
template <int POT>
__device__ __forceinline__ double pair_gm(const SysParams& p, double d, double rsum, double& ep) {
  if constexpr (POT == POT_HARMONIC) {
    double ov = 1.0 - d / rsum;
    if (ov > 0.0) {
      ep = (0.5 * p.ec * ov * ov) * 0.5;
      return p.ec * ov / rsum;
    }
    return 0.0;
  } else if constexpr (POT == POT_LJ) {
    if (d <= p.lj_cutoff * rsum) {
      double ratio = rsum / d;
      double r2 = ratio * ratio;
      double r6 = r2 * r2 * r2;
      double r12 = r6 * r6;
      double fshift = p.lj_fshift / rsum;
      ep = 0.5 * (4.0 * p.ec * (r12 - r6) - p.lj_ecut - fabs(fshift) * (d - p.lj_cutoff * rsum));
      return 24.0 * p.ec * (2.0 * r12 - r6) / d - fshift;
    }
    return 0.0;
  } else if constexpr (POT == POT_ADHESIVE) {
    double ov = 1.0 - d / rsum;
    if (d < (1.0 + p.l2) * rsum) {
      if (d < (1.0 + p.l1) * rsum) {
        ep = 0.5 * p.ec * (ov * ov - p.l1 * p.l2) * 0.5;
        return p.ec * ov / rsum;
      }
      double k = p.ec * p.l1 / (p.l2 - p.l1);
      ep = -(0.5 * k * (ov + p.l2) * (ov + p.l2)) * 0.5;
      return -k * (ov + p.l2) / rsum;
    }
    return 0.0;
  } else {  // WCA
    if (d <= kWCAcut * rsum) {
      double ratio = rsum / d;
      double r2 = ratio * ratio;
      double r6 = r2 * r2 * r2;
      double r12 = r6 * r6;
      ep = 0.5 * p.ec * (4.0 * (r12 - r6) + 1.0);
      return 24.0 * p.ec * (2.0 * r12 - r6) / d;
    }
    return 0.0;
  }
}

// Runtime -> compile-time dispatch over the potential.
template <template <int> class F, typename... Args>
inline void dispatch_pot(int pot, Args&&... args) {
  switch (pot) {
    case POT_HARMONIC: F<POT_HARMONIC>::run(args...); break;
    case POT_LJ: F<POT_LJ>::run(args...); break;
    case POT_ADHESIVE: F<POT_ADHESIVE>::run(args...); break;
    default: F<POT_WCA>::run(args...); break;
  }
}

// Device-side status block shared by every kernel of one context.
struct DevStatus {
  int rebuild;        // displacement check fired since the last rebuild
  int overflow;       // a list build found more neighbours than capacity
  int abort;          // set on overflow/timeouts: later ops of a launch become no-ops
  int nonfinite;      // a NaN/Inf force or position was seen
  long long ops_done; // completed step operations (for resume after abort)
  long long update_count;  // neighbour-list rebuilds (DPM2D::updateCount)
  int max_count;      // largest neighbour count of the last build
  unsigned int done_ctr;   // last-block counter for in-kernel final reductions
  int converged;      // FIRE: max |F| component below tolerance
  int max_ever;       // largest neighbour count of any build
  long long fire_iters;    // FIRE iterations actually performed
  long long rng_step;      // integrator steps since init: noise of step s uses Philox streams 2s, 2s+1
  double sums[8];     // final reductions written by the last block
  unsigned int bar_count;  // grid barrier of the one-launch build: arrivals
  int stalled;        // a grid-barrier wait gave up (the build did not finish)
  // multi-step kernel (k_tile_steps): barrier arrivals, the rotation base of
  // its three per-step flag slots (bit 1: a rebuild is due, bit 2: a
  // non-finite force), and the middle steps of the sequence still to run
  unsigned long long pbar;
  int pflag[3];
  long long pbase;
  long long steps_left;
  // persistent batched FIRE: the last launch left with its force op due
  int bpending;
  // polls a grid-barrier wait makes before it gives up (0: 2^20, about a
  // second; negative: none, the first poll that finds the barrier incomplete
  // gives up)
  long long spin_limit;
};

__device__ __forceinline__ long long barrier_poll_limit(const DevStatus* st) {
  const long long lim = *(const volatile long long*)&st->spin_limit;
  return lim > 0 ? lim : (lim == 0 ? (1LL << 20) : 0);
}

}  // namespace cr
