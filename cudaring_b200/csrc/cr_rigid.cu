// Rigid rings (DPM2D::calcRigidForceEnergy, RigidNVE, RigidLangevin).
//
// One CTA per tile of whole rings, as in k_tile:
//   1. centroid of each ring from offsets to its first vertex (calcParticlePos,
//      include/cudaKernel.cuh:365-388) by a per-ring tree in shared memory;
//   2. vertex-vertex pair forces, own side only (kernelCalcVertexForceTorque,
//      :1412-1450), L lanes per vertex;
//   3. per-vertex torque about the centroid and the ring sums: force, torque /
//      moment of inertia, moment of inertia, energy
//      (kernelCalcTorqueAndMomentOfInertia / kernelCalcParticleRigidForceEnergy,
//      :1452-1492);
//   4. MODE_STEP: the ring's velocity and angular velocity complete the step
//      (RigidNVE::updateVelocity, src/Simulator.cu:348-369) and, for advancing
//      ops, take the next half kick, move the centroid and the angle
//      (updatePosition, :329-346) and every vertex is translated and rotated
//      about the new centroid (kernelTranslateVertices / kernelRotateVertices,
//      include/cudaKernel.cuh:1678-1713) into the other position buffer.
// Ring mass is 1 and the torque term is the angular acceleration, as in the
// reference.  The Langevin form here is a correct one (friction and noise
// noise*xi - gamma*v on the ring velocity with noise = sqrt(2 T gamma / dt));
// the reference's RigidLangevin adds unscaled N(0,1) draws to the velocity.
#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

// PREC_MIXED: the vertex pair terms in FP32 on FP64-formed offsets (as the
// deformable kernel's mixed path), accumulated per vertex in FP32; torques,
// ring sums and integration stay FP64.
template <int POT, int MODE, int BLOCK, int L, int PREC>
__global__ void __launch_bounds__(BLOCK) k_rigid(const __grid_constant__ SysParams p,
                                                 const __grid_constant__ SysArrays a,
                                                 const __grid_constant__ StepArgs s,
                                                 const __grid_constant__ RigidArgs r) {
  constexpr int TV = BLOCK / L;
  __shared__ double2 s_pos[TV];
  __shared__ double2 s_u[TV];     // offsets from the ring's first vertex -> centroid
  __shared__ double2 s_f[TV];     // pair force
  __shared__ double s_e[TV];
  __shared__ double2 s_rf[TV];    // ring sums
  __shared__ double s_rt[TV], s_rm[TV], s_re[TV];
  __shared__ double2 s_c[TV];     // centroid per vertex slot (valid at the ring's first vertex)
  __shared__ double2 s_shift[TV]; // ring translation for this op (first vertex slot)
  __shared__ double s_dang[TV];   // ring rotation for this op (first vertex slot)
  __shared__ double s_red[BLOCK / 32][NSUM];

  DevStatus* st = s.status;
  if (MODE == MODE_STEP && (st->abort | st->converged)) {
    if (is_last_block(st)) {
      if (threadIdx.x == 0) {
        st->done_ctr = 0;
        if (s.use_cond) cudaGraphSetConditional(s.cond, 0u);
      }
    }
    return;
  }
  const int4 tile = a.tiles[blockIdx.x];
  const int v0 = tile.z, nvt = tile.w - tile.z;
  const int t = threadIdx.x;
  int ring = -1, k = 0, lf = 0, nvr = 1;
  if (t < nvt) {
    const int v = v0 + t;
    ring = a.ring_of[v];
    nvr = a.ring_nv[ring];
    lf = a.ring_first[ring] - v0;
    k = t - lf;
    s_pos[t] = a.pos[v];
  }
  __syncthreads();
  if (t < nvt) s_u[t] = pbc2(p, s_pos[t], s_pos[lf]);
  for (int stride = 1; stride < TV; stride <<= 1) {
    __syncthreads();
    if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) {
      s_u[t].x += s_u[t + stride].x;
      s_u[t].y += s_u[t + stride].y;
    }
  }
  __syncthreads();
  if (t < nvt && k == 0) {
    const double2 x0 = s_pos[t];
    s_c[t] = make_double2(x0.x + s_u[t].x / nvr, x0.y + s_u[t].y / nvr);
  }

  // pair forces
  {
    const int lv = t / L, lane = t % L;
    using T = typename std::conditional<PREC == PREC_MIXED, float, double>::type;
    typename Vec2<T>::type fi{0, 0};
    double ei = 0.0;
    if (lv < nvt) {
      const int i = v0 + lv;
      const double2 xi = s_pos[lv];
      const double ri = a.rad[i];
      const int cnt = min(a.nbr_cnt[i], a.nbr_cap);
      for (int sl = lane; sl < cnt; sl += L) {
        const int j = __ldg(a.nbr + (size_t)sl * p.nv + i);
        if constexpr (PREC == PREC_MIXED) pair_own_f<POT>(p, f2(pbc2(p, xi, a.pos[j])), (float)(ri + __ldg(a.rad + j)), fi, ei);
        else pair_own<POT>(p, pbc2(p, xi, a.pos[j]), ri + __ldg(a.rad + j), fi, ei);
      }
    }
#pragma unroll
    for (int o = L >> 1; o > 0; o >>= 1) {
      fi.x += __shfl_xor_sync(0xffffffffu, fi.x, o);
      fi.y += __shfl_xor_sync(0xffffffffu, fi.y, o);
      ei += __shfl_xor_sync(0xffffffffu, ei, o);
    }
    if (lane == 0 && lv < nvt) {
      s_f[lv] = make_double2(fi.x, fi.y);
      s_e[lv] = ei;
    }
  }
  __syncthreads();

  // torque about the centroid and ring sums
  double2 F = make_double2(0.0, 0.0), rel = make_double2(0.0, 0.0);
  double tau = 0.0;
  if (t < nvt) {
    F = s_f[t];
    rel = pbc2(p, s_pos[t], s_c[lf]);
    tau = rel.x * F.y - rel.y * F.x;
    s_rf[t] = F;
    s_rt[t] = tau;
    s_rm[t] = rel.x * rel.x + rel.y * rel.y;
    s_re[t] = s_e[t];
  }
  for (int stride = 1; stride < TV; stride <<= 1) {
    __syncthreads();
    if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) {
      s_rf[t].x += s_rf[t + stride].x;
      s_rf[t].y += s_rf[t + stride].y;
      s_rt[t] += s_rt[t + stride];
      s_rm[t] += s_rm[t + stride];
      s_re[t] += s_re[t + stride];
    }
  }
  __syncthreads();

  if constexpr (MODE == MODE_FORCE) {
    if (t < nvt) {
      const int v = v0 + t;
      s.force[v] = F;
      s.energy[v] = s_e[t];
      r.v_torque[v] = tau;
      if (k == 0) {
        s.ppos_out[ring] = s_c[t];
        r.p_force[ring] = s_rf[t];
        r.p_torque[ring] = s_rt[t] / s_rm[t];
        r.p_moi[ring] = s_rm[t];
        s.p_energy[ring] = s_re[t];
      }
    }
    return;
  } else {
    double sums[NSUM] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const unsigned long long step = (unsigned long long)st->rng_step;
    if (t < nvt && k == 0) {
      double2 Fp = s_rf[t];
      const double alpha = s_rt[t] / s_rm[t];
      if (s.active) {
        // self-propulsion of the ring along its own diffusing angle
        double psi = r.sp_angle[ring];
        const double2 z = philox_normal2(s.seed, 2ull * step + 1ull, (unsigned long long)ring);
        psi += s.sp_amp * z.x;
        psi = psi + kPi;
        psi = psi - 2.0 * kPi * floor(psi / (2.0 * kPi));
        psi = psi - kPi;
        r.sp_angle[ring] = psi;
        double sn, cs;
        sincos(psi, &sn, &cs);
        Fp.x += s.driving * cs;
        Fp.y += s.driving * sn;
      }
      const double2 vh = r.p_vel[ring];
      const double wh = r.p_angvel[ring];
      if (s.kind == KIND_LANGEVIN) {
        const double2 z = philox_normal2(s.seed, 2ull * step, (unsigned long long)ring);
        Fp.x += s.noise * z.x - s.gamma * vh.x;
        Fp.y += s.noise * z.y - s.gamma * vh.y;
      }
      const double2 vn = make_double2(vh.x + s.hdt * Fp.x, vh.y + s.hdt * Fp.y);
      const double wn = wh + s.hdt * alpha;
      if (s.advance) {
        const double2 v2 = make_double2(vn.x + s.hdt * Fp.x, vn.y + s.hdt * Fp.y);
        const double w2 = wn + s.hdt * alpha;
        r.p_vel[ring] = v2;
        r.p_angvel[ring] = w2;
        r.p_angle[ring] += s.dt * w2;
        s_shift[t] = make_double2(s.dt * v2.x, s.dt * v2.y);
        s_dang[t] = s.dt * w2;
      } else {
        r.p_vel[ring] = vn;
        r.p_angvel[ring] = wn;
        r.p_force[ring] = Fp;
        r.p_torque[ring] = alpha;
        r.p_moi[ring] = s_rm[t];
        s.p_energy[ring] = s_re[t];
        s.ppos_out[ring] = s_c[t];
      }
      if (s.accumulate) {
        sums[S_PE] = s_re[t];
        sums[S_VV] = vn.x * vn.x + vn.y * vn.y;
        sums[S_VF] = vn.x * Fp.x + vn.y * Fp.y;
        sums[S_FF] = Fp.x * Fp.x + Fp.y * Fp.y;
        sums[S_FMAX2] = fmax(Fp.x * Fp.x, Fp.y * Fp.y);
      }
      if (!(isfinite(Fp.x) && isfinite(Fp.y) && isfinite(alpha))) sums[S_NONFINITE] = 1.0;
    }
    __syncthreads();
    if (t < nvt) {
      const int v = v0 + t;
      if (s.advance) {
        // kernelTranslateVertices then kernelRotateVertices about the new centroid
        const double2 sh = s_shift[lf];
        const double da = s_dang[lf];
        const double2 cn = make_double2(s_c[lf].x + sh.x, s_c[lf].y + sh.y);
        double2 x = make_double2(s_pos[t].x + sh.x, s_pos[t].y + sh.y);
        const double2 d = pbc2(p, x, cn);
        double sn, cs;
        sincos(da, &sn, &cs);
        x.x += (d.x * cs - d.y * sn) - d.x;
        x.y += (d.x * sn + d.y * cs) - d.y;
        s.pos_out[v] = x;
        if (3.0 * dist_of(pbc2(p, x, s.last_pos[v])) > s.disp_cutoff) st->rebuild = 1;
      } else {
        s.force[v] = F;
        s.energy[v] = s_e[t];
        r.v_torque[v] = tau;
      }
    }
    block_partials<BLOCK>(sums, s_red, s.partials + (size_t)blockIdx.x * NSUM);
    if (is_last_block(st)) {
      reduce_partials(s.partials, gridDim.x, st->sums);
      __syncthreads();
      if (t == 0) {
        __threadfence();
        if (st->sums[S_NONFINITE] != 0.0) {
          st->nonfinite = 1;
          st->abort = 1;
        }
        st->ops_done += 1;
        st->rng_step += 1;
        st->done_ctr = 0;
        if (s.use_cond) cudaGraphSetConditional(s.cond, st->rebuild ? 1u : 0u);
      }
    }
  }
}

// First half kick + move that opens a rigid NVE / Langevin sequence, from the
// stored ring forces (RigidNVE::integrate up to the force call).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_rigid_drift(const __grid_constant__ SysParams p,
                                                       const __grid_constant__ SysArrays a,
                                                       const __grid_constant__ StepArgs s,
                                                       const __grid_constant__ RigidArgs r) {
  __shared__ double2 s_shift[BLOCK];
  __shared__ double2 s_cn[BLOCK];
  __shared__ double s_dang[BLOCK];
  DevStatus* st = s.status;
  if (st->abort | st->converged) {
    if (is_last_block(st)) {
      if (threadIdx.x == 0) {
        st->done_ctr = 0;
        if (s.use_cond) cudaGraphSetConditional(s.cond, 0u);
      }
    }
    return;
  }
  const int4 tile = a.tiles[blockIdx.x];
  const int v0 = tile.z, nvt = tile.w - tile.z;
  const int t = threadIdx.x;
  int ring = -1, lf = 0;
  if (t < nvt) {
    ring = a.ring_of[v0 + t];
    lf = a.ring_first[ring] - v0;
    if (t == lf) {
      const double2 Fp = r.p_force[ring];
      const double alpha = r.p_torque[ring];
      const double2 v2 = make_double2(r.p_vel[ring].x + s.hdt * Fp.x, r.p_vel[ring].y + s.hdt * Fp.y);
      const double w2 = r.p_angvel[ring] + s.hdt * alpha;
      const double2 c = s.ppos_out[ring];
      r.p_vel[ring] = v2;
      r.p_angvel[ring] = w2;
      r.p_angle[ring] += s.dt * w2;
      s_shift[t] = make_double2(s.dt * v2.x, s.dt * v2.y);
      s_cn[t] = make_double2(c.x + s.dt * v2.x, c.y + s.dt * v2.y);
      s_dang[t] = s.dt * w2;
    }
  }
  __syncthreads();
  if (t < nvt) {
    const int v = v0 + t;
    const double2 sh = s_shift[lf];
    const double2 cn = s_cn[lf];
    double2 x = a.pos[v];
    x.x += sh.x;
    x.y += sh.y;
    const double2 d = pbc2(p, x, cn);
    double sn, cs;
    sincos(s_dang[lf], &sn, &cs);
    x.x += (d.x * cs - d.y * sn) - d.x;
    x.y += (d.x * sn + d.y * cs) - d.y;
    s.pos_out[v] = x;
    if (3.0 * dist_of(pbc2(p, x, s.last_pos[v])) > s.disp_cutoff) st->rebuild = 1;
  }
  if (is_last_block(st)) {
    if (t == 0) {
      __threadfence();
      st->ops_done += 1;
      st->done_ctr = 0;
      if (s.use_cond) cudaGraphSetConditional(s.cond, st->rebuild ? 1u : 0u);
    }
  }
}

// Ring velocities N(0, sqrt(T)) with the mean removed
// (RigidLangevin::injectKineticEnergy + kernelConserveParticleMomentum,
// src/Simulator.cu:255-262, over all rings).
__global__ void k_rigid_inject(int np, double2* p_vel, double amp, unsigned long long seed, unsigned long long stream) {
  __shared__ double2 s_sum[256];
  double2 acc = make_double2(0.0, 0.0);
  for (int q = threadIdx.x; q < np; q += blockDim.x) {
    const double2 z = philox_normal2(seed, stream, (unsigned long long)q);
    acc.x += amp * z.x;
    acc.y += amp * z.y;
  }
  s_sum[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s_sum[threadIdx.x].x += s_sum[threadIdx.x + o].x;
      s_sum[threadIdx.x].y += s_sum[threadIdx.x + o].y;
    }
    __syncthreads();
  }
  const double2 mean = make_double2(s_sum[0].x / np, s_sum[0].y / np);
  for (int q = threadIdx.x; q < np; q += blockDim.x) {
    const double2 z = philox_normal2(seed, stream, (unsigned long long)q);
    p_vel[q] = make_double2(amp * z.x - mean.x, amp * z.y - mean.y);
  }
}

template <int POT, int MODE, int PREC>
static void launch_rigid_p(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s,
                           const RigidArgs& r) {
  if (c.lanes == 1) k_rigid<POT, MODE, 128, 1, PREC><<<c.grid, 128, 0, c.stream>>>(p, a, s, r);
  else if (c.lanes == 4) k_rigid<POT, MODE, 256, 4, PREC><<<c.grid, 256, 0, c.stream>>>(p, a, s, r);
  else if (c.lanes == 8) k_rigid<POT, MODE, 256, 8, PREC><<<c.grid, 256, 0, c.stream>>>(p, a, s, r);
  else k_rigid<POT, MODE, 192, 2, PREC><<<c.grid, 192, 0, c.stream>>>(p, a, s, r);  // tiles of up to 96 vertices
}

template <int POT, int MODE>
static void launch_rigid_t(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s,
                           const RigidArgs& r) {
  if (c.precision == CR_PRECISION_MIXED) launch_rigid_p<POT, MODE, PREC_MIXED>(c, p, a, s, r);
  else launch_rigid_p<POT, MODE, PREC_FP64>(c, p, a, s, r);
}

void launch_rigid(const LaunchCfg& c, int pot, int mode, const SysParams& p_in, const SysArrays& a,
                  const StepArgs& s, const RigidArgs& r) {
  const SysParams p = with_f32_constants(p_in);  // the FP32 pair terms read them
#define CR_RIGID_CASE(P)                                              \
  case P:                                                             \
    if (mode == MODE_FORCE) launch_rigid_t<P, MODE_FORCE>(c, p, a, s, r); \
    else launch_rigid_t<P, MODE_STEP>(c, p, a, s, r);                 \
    break;
  switch (pot) {
    CR_RIGID_CASE(POT_HARMONIC)
    CR_RIGID_CASE(POT_LJ)
    CR_RIGID_CASE(POT_ADHESIVE)
    CR_RIGID_CASE(POT_WCA)
    default: break;
  }
#undef CR_RIGID_CASE
}

void launch_rigid_drift(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s,
                        const RigidArgs& r) {
  // every tile holds at most 128 vertices (tile_vertices)
  k_rigid_drift<128><<<c.grid, 128, 0, c.stream>>>(p, a, s, r);
}

void launch_rigid_inject(cudaStream_t st, int np, double2* p_vel, double amp, unsigned long long seed,
                         unsigned long long stream) {
  k_rigid_inject<<<1, 256, 0, st>>>(np, p_vel, amp, seed, stream);
}

}  // namespace cr
