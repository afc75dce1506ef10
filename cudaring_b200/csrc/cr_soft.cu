// Soft-disk pre-packing: the particle-level stage that precedes vertex FIRE
// (compressFIRE.cpp:53-90).  Every ring is a soft disk of radius
// particleRad at its particle position; the disks are minimised by FIRE with
// per-particle masses pi / r^2, then each ring's vertices are placed on a
// circle about its particle position.
//
//   k_soft_force<POT, FIRE>  kernelCalcParticleInteraction
//                            (include/cudaKernel.cuh:1185-1219): per particle,
//                            over its list, the vertex pair terms with radSum
//                            = r_i + r_j.  FIRE = true adds the second half
//                            kick of FIRE::updateParticleVelocity
//                            (src/FIRE.cu:74-97) and per-CTA sums of v.F,
//                            |v|^2, |F|^2 and max F_d^2; the last CTA does
//                            bendParticleVelocityTowardsForce's scalar part
//                            (src/FIRE.cu:100-141) and the convergence test
//                            of the driver loop (compressFIRE.cpp:66).
//   k_soft_move              the velocity bend left pending by the last force
//                            op, then updateParticlePositionAndVelocity
//                            (src/FIRE.cu:45-71) and the driver's displacement
//                            test (compressFIRE.cpp:72-76) into status.rebuild
//   k_soft_bend              a pending bend alone (end of a call)
//   k_soft_vertices          DPM2D::initVerticesOnParticles (src/DPM2D.cu:1678-1691)
//
// The particle list is built by the one-launch cell-list build of cr_nbr.cu
// with the particle list rule (self_rsum).
#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

namespace {

constexpr int kSoftBlock = 256;

// fixed-order CTA sum / max over the block, result on thread 0
__device__ __forceinline__ double block_sum_d(double x, double* s) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = x;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kSoftBlock / 32; w++) t += s[w];
  return t;
}
__device__ __forceinline__ double block_max_d(double x, double* s) {
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = x;
  __syncthreads();
  double t = -1.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kSoftBlock / 32; w++) t = fmax(t, s[w]);
  return t;
}

// v -> the bend of bendParticleVelocityTowardsForce (src/FIRE.cu:120-139)
__device__ __forceinline__ double2 bend(double2 v, double2 f, const SoftFire& fr) {
  if (fr.zero) return make_double2(0.0, 0.0);
  const double a = fr.a;
  return make_double2((1 - a) * v.x + a * f.x * fr.ratio, (1 - a) * v.y + a * f.y * fr.ratio);
}

}  // namespace

template <int POT, bool FIRE>
__global__ void __launch_bounds__(kSoftBlock) k_soft_force(const __grid_constant__ SysParams p,
                                                           const __grid_constant__ SoftArgs a) {
  __shared__ double s_red[kSoftBlock / 32];
  DevStatus* st = a.status;
  if (FIRE) {
    const volatile SoftFire* vf = a.fire;
    if (vf->converged || ((volatile DevStatus*)st)->abort) return;  // uniform: no CTA takes part below
  }
  const int i = blockIdx.x * kSoftBlock + threadIdx.x;
  double vf_ = 0.0, vv = 0.0, ff = 0.0, fm = -1.0;
  if (i < p.np) {
    const double2 xi = a.pos[i];
    const double ri = a.rad[i];
    double2 f = make_double2(0.0, 0.0);
    double e = 0.0;
    const int cnt = min(a.cnt[i], a.cap);
    for (int k = 0; k < cnt; k++) {
      const int j = a.nbr[(size_t)k * p.np + i];
      pair_own<POT>(p, pbc2(p, xi, a.pos[j]), ri + a.rad[j], f, e);
    }
    a.force[i] = f;
    a.energy[i] = e;
    if (FIRE) {
      const double dt = a.fire->dt;
      const double m = kPi / (ri * ri);  // DPM2D::setParticleMassFIRE (src/DPM2D.cu:3676-3684)
      double2 v = a.vel[i];
      v.x += 0.5 * dt * f.x / m;
      v.y += 0.5 * dt * f.y / m;
      double total = 0;
      total += f.x;
      total += f.y;
      if (total == 0) v = make_double2(0.0, 0.0);
      a.vel[i] = v;
      vf_ = v.x * f.x + v.y * f.y;
      vv = v.x * v.x + v.y * v.y;
      ff = f.x * f.x + f.y * f.y;
      fm = fmax(f.x * f.x, f.y * f.y);
    }
  }
  if (!FIRE) return;
  const double b0 = block_sum_d(vf_, s_red);
  const double b1 = block_sum_d(vv, s_red);
  const double b2 = block_sum_d(ff, s_red);
  const double b3 = block_max_d(fm, s_red);
  if (threadIdx.x == 0) {
    double* q = a.partials + 4 * blockIdx.x;
    q[0] = b0;
    q[1] = b1;
    q[2] = b2;
    q[3] = b3;
  }
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      __threadfence();
      double vdotf = 0.0, v2 = 0.0, f2 = 0.0, fmax2 = -1.0;
      for (unsigned int b = 0; b < gridDim.x; b++) {
        const volatile double* q = a.partials + 4 * b;
        vdotf += q[0];
        v2 += q[1];
        f2 += q[2];
        fmax2 = fmax(fmax2, q[3]);
      }
      SoftFire& fr = *a.fire;
      int zero = 0;
      if (vdotf < 0) {
        zero = 1;
        fr.num_step = 0;
        fr.dt = fmax(fr.dt * fr.f_dec, fr.dt_max / 10);
        fr.a = fr.a_start;
      } else if (fr.num_step > fr.min_step) {
        fr.dt = fmin(fr.dt * fr.f_inc, fr.dt_max);
        fr.a *= fr.f_a;
      }
      if (f2 == 0) zero = 1;
      fr.zero = zero;
      fr.ratio = zero ? 0.0 : sqrt(v2 / f2);
      fr.pending = 1;
      fr.num_step += 1;
      fr.iters += 1;
      fr.max_f2 = fmax2;
      if (!(sqrt(fmax2) > fr.tol)) fr.converged = 1;
      st->done_ctr = 0;
    }
  }
}

__global__ void __launch_bounds__(kSoftBlock) k_soft_move(const __grid_constant__ SysParams p,
                                                          const __grid_constant__ SoftArgs a, int check) {
  DevStatus* st = a.status;
  if (((volatile DevStatus*)st)->abort) return;  // resumed by the host after it regrows the list
  const SoftFire fr = *a.fire;  // written by earlier kernels only
  const int i = blockIdx.x * kSoftBlock + threadIdx.x;
  if (i < p.np) {
    double2 v = a.vel[i];
    const double2 f = a.force[i];
    if (fr.pending) v = bend(v, f, fr);
    if (!fr.converged) {
      const double dt = fr.dt;
      const double m = kPi / (a.rad[i] * a.rad[i]);
      double2 x = a.pos[i];
      v.x += 0.5 * dt * f.x / m;
      x.x += dt * v.x;
      v.y += 0.5 * dt * f.y / m;
      x.y += dt * v.y;
      double total = 0;
      total += f.x;
      total += f.y;
      if (total == 0) v = make_double2(0.0, 0.0);
      a.pos[i] = x;
      if (check && 3.0 * dist_of(pbc2(p, x, a.last_pos[i])) > a.cutoff) st->rebuild = 1;
    }
    a.vel[i] = v;
  }
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      a.fire->pending = 0;
      st->done_ctr = 0;
    }
  }
}

__global__ void __launch_bounds__(kSoftBlock) k_soft_bend(int np, const __grid_constant__ SoftArgs a) {
  const SoftFire fr = *a.fire;  // written by earlier kernels only
  if (!fr.pending) return;
  const int i = blockIdx.x * kSoftBlock + threadIdx.x;
  if (i < np) a.vel[i] = bend(a.vel[i], a.force[i], fr);
  if (is_last_block(a.status)) {
    if (threadIdx.x == 0) {
      a.fire->pending = 0;
      a.status->done_ctr = 0;
    }
  }
}

// rad = sqrt(2 a0 / (n sin(2 pi / n))), angle 2 pi v / n with v the global
// vertex index, jitter 1e-3 * l0 * u with u the caller's draws (x then y of
// each vertex) or Philox uniforms.
__global__ void __launch_bounds__(kSoftBlock) k_soft_vertices(int nv, const int* ring_of, const int* ring_nv,
                                                              const double* a0, const double* l0, const double2* ppos,
                                                              const double* draws, unsigned long long seed,
                                                              unsigned long long stream, double2* pos, double2* vel,
                                                              double2* force, double* energy) {
  const int v = blockIdx.x * kSoftBlock + threadIdx.x;
  if (v >= nv) return;
  const int q = ring_of[v];
  const int n = ring_nv[q];
  const double rad = sqrt((2. * a0[q]) / (n * sin(2. * kPi / n)));
  const double ang = (2. * kPi * v) / n;
  double2 u;
  if (draws) u = make_double2(draws[2 * v], draws[2 * v + 1]);
  else u = philox_uniform2(seed, stream, (unsigned long long)v);
  const double2 c = ppos[q];
  pos[v] = make_double2(rad * cos(ang) + c.x + 1e-03 * l0[v] * u.x, rad * sin(ang) + c.y + 1e-03 * l0[v] * u.y);
  vel[v] = make_double2(0.0, 0.0);
  force[v] = make_double2(0.0, 0.0);
  energy[v] = 0.0;
}

namespace {
template <int POT>
struct SoftForceL {
  static void run(cudaStream_t st, const SysParams& p, const SoftArgs& a, bool fire) {
    const int nb = (p.np + kSoftBlock - 1) / kSoftBlock;
    if (fire) k_soft_force<POT, true><<<nb, kSoftBlock, 0, st>>>(p, a);
    else k_soft_force<POT, false><<<nb, kSoftBlock, 0, st>>>(p, a);
  }
};
}  // namespace

int soft_blocks(int np) { return (np + kSoftBlock - 1) / kSoftBlock; }

void launch_soft_force(cudaStream_t st, int pot, const SysParams& p, const SoftArgs& a, bool fire) {
  dispatch_pot<SoftForceL>(pot, st, p, a, fire);
}

void launch_soft_move(cudaStream_t st, const SysParams& p, const SoftArgs& a, int check) {
  k_soft_move<<<soft_blocks(p.np), kSoftBlock, 0, st>>>(p, a, check);
}

void launch_soft_bend(cudaStream_t st, int np, const SoftArgs& a) {
  k_soft_bend<<<soft_blocks(np), kSoftBlock, 0, st>>>(np, a);
}

void launch_soft_vertices(cudaStream_t st, int nv, const int* ring_of, const int* ring_nv, const double* a0,
                          const double* l0, const double2* ppos, const double* draws, unsigned long long seed,
                          unsigned long long stream, double2* pos, double2* vel, double2* force, double* energy) {
  k_soft_vertices<<<(nv + kSoftBlock - 1) / kSoftBlock, kSoftBlock, 0, st>>>(nv, ring_of, ring_nv, a0, l0, ppos, draws,
                                                                          seed, stream, pos, vel, force, energy);
}

}  // namespace cr
