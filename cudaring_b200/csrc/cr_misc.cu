// Per-vertex update kernels and reductions around the tiled force kernel.
#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

// Early-exit prologue shared by op kernels: when the sequence was aborted or
// FIRE converged, every CTA still takes part in the last-block protocol.
__device__ __forceinline__ bool op_skipped(const StepArgs& s) {
  DevStatus* st = s.status;
  if (!(st->abort | st->converged)) return false;
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      st->done_ctr = 0;
      if (s.use_cond) cudaGraphSetConditional(s.cond, 0u);
    }
  }
  return true;
}

__device__ __forceinline__ void op_finish(const StepArgs& s) {
  DevStatus* st = s.status;
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      __threadfence();
      st->ops_done += 1;
      st->done_ctr = 0;
      if (s.use_cond) cudaGraphSetConditional(s.cond, st->rebuild ? 1u : 0u);
    }
  }
}

// First half kick + drift that opens an NVE / Langevin / BAOAB sequence:
// kernelUpdateVertexVel(dt/2) then kernelUpdateVertexPos(dt)
// (include/cudaKernel.cuh:1980-1996, src/Simulator.cu:23-30, 112-119); with
// rescale_T set it opens every NVERescale step.
__global__ void __launch_bounds__(256) k_drift(const __grid_constant__ SysParams p,
                                               const __grid_constant__ SysArrays a,
                                               const __grid_constant__ StepArgs s) {
  if (op_skipped(s)) return;
  DevStatus* st = s.status;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < p.nv) {
    const double2 x = a.pos[v];
    const double2 f = s.force[v];
    double2 vh = s.vel[v];
    if (s.rescale_T > 0.0) {
      // NVERescale::injectKineticEnergy (src/Simulator.cu:224-238): T from the
      // sum of v^2 that the previous op reduced, T = sum v^2 / (2 Nv)
      const double scale = sqrt(s.rescale_T / (st->sums[S_VV] / (2.0 * p.nv)));
      vh = make_double2(vh.x * scale, vh.y * scale);
    }
    vh = make_double2(vh.x + s.hdt * f.x, vh.y + s.hdt * f.y);
    double2 xn;
    if (s.kind == KIND_BAOAB) {
      xn = make_double2(x.x + s.hdt * vh.x, x.y + s.hdt * vh.y);
      const unsigned long long step = (unsigned long long)st->rng_step;
      const double2 z = philox_normal2(s.seed, 2ull * step, (unsigned long long)a.ring_of[v]);
      vh = make_double2(s.gamma_factor * vh.x + s.noise * z.x, s.gamma_factor * vh.y + s.noise * z.y);
      xn = make_double2(xn.x + s.hdt * vh.x, xn.y + s.hdt * vh.y);
    } else {
      xn = make_double2(x.x + s.dt * vh.x, x.y + s.dt * vh.y);
    }
    s.pos_out[v] = xn;
    s.vel[v] = vh;
    if (3.0 * dist_of(pbc2(p, xn, s.last_pos[v])) > s.disp_cutoff) st->rebuild = 1;
  }
  op_finish(s);
}

// FIRE iteration up to the position update (FIRE::minimizerVertexLoop,
// src/FIRE.cu:397-406): checkFIREParams (:338-371) from P = v.F, the
// half kick (:320-335), bendVertexVelocityTowardsForce (:374-394) and
// updateVertexPosition (:302-317).  |v|^2 after the half kick is formed from
// the three sums of the previous force op:  |v + h F|^2 = vv + 2h vF + h^2 FF.
__global__ void __launch_bounds__(256) k_fire_pre(const __grid_constant__ SysParams p,
                                                  const __grid_constant__ SysArrays a,
                                                  const __grid_constant__ StepArgs s,
                                                  const __grid_constant__ FireParams fp, double* fire_state) {
  if (op_skipped(s)) return;
  DevStatus* st = s.status;
  const long long it = st->fire_iters;
  const double* cur = fire_state + (it & 1) * 4;
  double dt = cur[0], alpha = cur[1];
  long long nstep = (long long)cur[2];
  const double P = st->sums[S_VF], vv = st->sums[S_VV], ff = st->sums[S_FF];
  bool rollback = false;
  if (P > 0) {
    nstep++;
    if (nstep > fp.min_step) {
      dt = fmin(dt * fp.f_inc, fp.dt_max);
      alpha *= fp.f_a;
    }
  } else {
    nstep = 0;
    dt = fmax(dt * fp.f_dec, fp.dt_max / 10);
    alpha = fp.a_start;
    rollback = true;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double* nxt = fire_state + ((it + 1) & 1) * 4;
    nxt[0] = dt;
    nxt[1] = alpha;
    nxt[2] = (double)nstep;
  }
  const double h = 0.5 * dt;
  const double vpost2 = rollback ? (h * h) * ff : vv + dt * P + (h * h) * ff;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < p.nv) {
    double2 x = a.pos[v];
    double2 vel = s.vel[v];
    const double2 f = s.force[v];
    if (rollback) {
      x = make_double2(x.x - h * vel.x, x.y - h * vel.y);
      vel = make_double2(0.0, 0.0);
    }
    vel = make_double2(vel.x + h * f.x, vel.y + h * f.y);
    if (ff > 0) {
      const double ratio = sqrt(vpost2 / ff);
      vel = make_double2((1 - alpha) * vel.x + alpha * f.x * ratio, (1 - alpha) * vel.y + alpha * f.y * ratio);
    }
    x = make_double2(x.x + dt * vel.x, x.y + dt * vel.y);
    s.pos_out[v] = x;
    s.vel[v] = vel;
    if (3.0 * dist_of(pbc2(p, x, s.last_pos[v])) > s.disp_cutoff) st->rebuild = 1;
  }
  op_finish(s);
}

// Sums for the getters and for the first FIRE check: PE, |v|^2, v.F, |F|^2,
// max F_d^2 (DPM2D::getPotentialEnergy .. getMaxUnbalancedForce,
// src/DPM2D.cu:986-1087), written to status->sums by the last CTA.
__global__ void __launch_bounds__(256) k_reduce(int nv, int np, const double2* vel, const double2* force,
                                                const double* energy, const double* p_energy, int use_p_energy,
                                                double* partials, DevStatus* st) {
  // compensated per-thread sums (two_sum_add), then the compensated CTA tree
  double acc[NSUM] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, cmp[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const double2 u = vel[v], f = force[v];
    two_sum_add(acc[S_PE], cmp[S_PE], energy[v]);
    two_sum_add(acc[S_VV], cmp[S_VV], u.x * u.x + u.y * u.y);
    two_sum_add(acc[S_VF], cmp[S_VF], u.x * f.x + u.y * f.y);
    two_sum_add(acc[S_FF], cmp[S_FF], f.x * f.x + f.y * f.y);
    acc[S_FMAX2] = fmax(acc[S_FMAX2], fmax(f.x * f.x, f.y * f.y));
    if (!(isfinite(f.x) && isfinite(f.y))) acc[S_NONFINITE] = 1.0;
  }
  if (use_p_energy)
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x)
      two_sum_add(acc[S_PE], cmp[S_PE], p_energy[q]);
#pragma unroll
  for (int q = 0; q < 4; q++) acc[q] += cmp[q];
  __shared__ double s_red[8][NSUM];
  block_partials<256>(acc, s_red, partials + (size_t)blockIdx.x * NSUM);
  if (is_last_block(st)) {
    reduce_partials(partials, gridDim.x, st->sums);
    __syncthreads();
    if (threadIdx.x == 0) st->done_ctr = 0;
  }
}

// v <- scale * v + shift for n double2 velocities (exact temperature after a
// thermal draw; momentum removal).
__global__ void k_affine_vel(int n, double2* vel, double scale, double2 shift) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < n) {
    const double2 u = vel[v];
    vel[v] = make_double2(scale * u.x + shift.x, scale * u.y + shift.y);
  }
}

// Langevin::injectKineticEnergy (src/Simulator.cu:32-52): every vertex takes
// its ring's N(0, amplitude) velocity.
__global__ void k_inject_ke(int nv, const int* ring_of, double2* vel, double amplitude, unsigned long long seed,
                            unsigned long long stream) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    const double2 z = philox_normal2(seed, stream, (unsigned long long)ring_of[v]);
    vel[v] = make_double2(amplitude * z.x, amplitude * z.y);
  }
}

// DPM2D::scaleVertices (src/DPM2D.cu:1802-1811) with kernelScaleVertexPositions
// (include/cudaKernel.cuh:1644-1658): raw (not minimum-image) offsets from the
// stored ring centroid.
__global__ void k_scale_vertices(int nv, int np, const int* ring_of, const double2* ppos, double2* pos, double* a0,
                                 double* area, double* l0, double* rad, double scale) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    const double2 c = ppos[ring_of[v]];
    double2 x = pos[v];
    x.x += (scale - 1) * (x.x - c.x);
    x.y += (scale - 1) * (x.y - c.y);
    pos[v] = x;
    l0[v] *= scale;
    rad[v] *= scale;
  }
  if (v < np) {
    a0[v] *= scale * scale;
    area[v] *= scale * scale;
  }
}

// addSelfPropulsion's angle update (src/DPM2D.cu:2007-2017).
__global__ void k_advance_angles(int np, double* angle, double amp, unsigned long long seed,
                                 unsigned long long stream) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < np) {
    const double2 z = philox_normal2(seed, stream, (unsigned long long)q);
    double psi = angle[q] + amp * z.x;
    psi = psi + kPi;
    psi = psi - 2.0 * kPi * floor(psi / (2.0 * kPi));
    angle[q] = psi - kPi;
  }
}

// kernelCalcVertexArea (include/cudaKernel.cuh:1636-1642)
__global__ void k_vertex_area(int np, const int* ring_first, const int* ring_nv, const double* rad, double* out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < np) {
    const double r = rad[ring_first[q]];
    out[q] = r * r * (0.5 * ring_nv[q] - 1);
  }
}

// ---------------------------------------------------------------- launchers

void launch_drift(cudaStream_t st, const SysParams& p, const SysArrays& a, const StepArgs& s, int nblocks) {
  k_drift<<<nblocks, 256, 0, st>>>(p, a, s);
}
void launch_fire_pre(cudaStream_t st, const SysParams& p, const SysArrays& a, const StepArgs& s,
                     const FireParams& fp, double* fire_state, int nblocks) {
  k_fire_pre<<<nblocks, 256, 0, st>>>(p, a, s, fp, fire_state);
}
void launch_reduce(cudaStream_t st, int nv, int np, const double2* vel, const double2* force, const double* energy,
                   const double* p_energy, int use_p_energy, double* partials, DevStatus* status, int nblocks) {
  k_reduce<<<nblocks, 256, 0, st>>>(nv, np, vel, force, energy, p_energy, use_p_energy, partials, status);
}
void launch_affine_vel(cudaStream_t st, int n, double2* vel, double scale, double2 shift) {
  k_affine_vel<<<(n + 255) / 256, 256, 0, st>>>(n, vel, scale, shift);
}
void launch_inject_ke(cudaStream_t st, int nv, const int* ring_of, double2* vel, double amplitude,
                      unsigned long long seed, unsigned long long stream) {
  k_inject_ke<<<(nv + 255) / 256, 256, 0, st>>>(nv, ring_of, vel, amplitude, seed, stream);
}
void launch_scale_vertices(cudaStream_t st, int nv, int np, const int* ring_of, const double2* ppos, double2* pos,
                           double* a0, double* area, double* l0, double* rad, double scale) {
  const int n = nv > np ? nv : np;
  k_scale_vertices<<<(n + 255) / 256, 256, 0, st>>>(nv, np, ring_of, ppos, pos, a0, area, l0, rad, scale);
}
void launch_advance_angles(cudaStream_t st, int np, double* angle, double amp, unsigned long long seed,
                           unsigned long long stream) {
  k_advance_angles<<<(np + 255) / 256, 256, 0, st>>>(np, angle, amp, seed, stream);
}
void launch_vertex_area(cudaStream_t st, int np, const int* ring_first, const int* ring_nv, const double* rad,
                        double* out) {
  k_vertex_area<<<(np + 255) / 256, 256, 0, st>>>(np, ring_first, ring_nv, rad, out);
}

}  // namespace cr
