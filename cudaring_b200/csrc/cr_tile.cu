// Tiled force + integrator kernel (see cr_tile.cuh for the phase structure).
#include "cr_tile.cuh"
#include "cr_launch.h"

namespace cr {

// Occupancy target in threads per SM: 512 leaves 128 registers per thread,
// where the smooth-interaction body compiles without spills.
constexpr int kTileThreadsPerSM = 512;

template <int POT, int INTER, int MODE, int BLOCK, int L>
__global__ void __launch_bounds__(BLOCK, kTileThreadsPerSM / BLOCK) k_tile(const __grid_constant__ SysParams p,
                                                const __grid_constant__ SysArrays a,
                                                const __grid_constant__ StepArgs s) {
  constexpr int TV = BLOCK / L;
  __shared__ double2 s_pos[TV];
  __shared__ double2 s_seg[TV];     // pbc(pos[next] - pos[v])
  __shared__ double s_theta[TV];
  __shared__ double s_r0[TV];       // shoelace terms -> ring area
  __shared__ double s_r1[TV];       // segment lengths -> perimeter
  __shared__ double2 s_r2[TV];      // offsets from the first vertex -> centroid
  __shared__ double2 s_fpair[TV];   // pair force on v
  __shared__ double2 s_fprev[TV];   // smooth: force on prev(v) gathered by v
  __shared__ double s_epair[TV];
  __shared__ int s_lp[TV], s_ln[TV], s_lf[TV], s_nv[TV];
  __shared__ double s_red[BLOCK / 32][NSUM];

  DevStatus* st = s.status;
  if (MODE == MODE_STEP && (st->abort | st->converged)) {
    // keep the last-block protocol intact so later ops see a consistent counter
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

  // ---- phase 1: geometry --------------------------------------------------
  int ring = -1, k = 0, lf = 0, nvr = 1;
  if (t < nvt) {
    const int v = v0 + t;
    ring = a.ring_of[v];
    const int f = a.ring_first[ring];
    nvr = a.ring_nv[ring];
    lf = f - v0;
    k = t - lf;
    s_lf[t] = lf;
    s_nv[t] = nvr;
    s_ln[t] = lf + (k + 1 == nvr ? 0 : k + 1);
    s_lp[t] = lf + (k == 0 ? nvr - 1 : k - 1);
    s_pos[t] = a.pos[v];
  }
  __syncthreads();
  if (t < nvt) {
    const double2 x = s_pos[t];
    const double2 xn = s_pos[s_ln[t]];
    const double2 seg = pbc2(p, xn, x);
    s_seg[t] = seg;
    const double2 x0 = s_pos[lf];
    const double2 u = pbc2(p, x, x0);
    const double2 un = pbc2(p, xn, x0);
    s_r0[t] = u.x * un.y - un.x * u.y;
    s_r1[t] = dist_of(seg);
    s_r2[t] = u;
  }
  __syncthreads();
  if (t < nvt) {
    // calcAngle(nextSegment, previousSegment) (include/cudaKernel.cuh:423-427)
    const double2 ns = s_seg[t];
    const double2 ps = s_seg[s_lp[t]];
    s_theta[t] = atan2(ns.x * ps.y - ns.y * ps.x, ns.x * ps.x + ns.y * ps.y);
  }
  // deterministic per-ring tree over the ring's vertex range
  for (int stride = 1; stride < TV; stride <<= 1) {
    __syncthreads();
    if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) {
      s_r0[t] += s_r0[t + stride];
      s_r1[t] += s_r1[t + stride];
      s_r2[t].x += s_r2[t + stride].x;
      s_r2[t].y += s_r2[t + stride].y;
    }
  }
  __syncthreads();

  // ---- phase 2: shape force (kernelCalcShapeForceEnergy, include/cudaKernel.cuh:474-529)
  double2 fsh = make_double2(0.0, 0.0);
  double esh = 0.0;
  if (t < nvt) {
    const int v = v0 + t;
    const int lp = s_lp[t], ln = s_ln[t];
    const int vp = v0 + lp, vn = v0 + ln;
    const double area = fabs(s_r0[lf]) * 0.5;
    const double a0 = a.a0[ring];
    const double dA = (area / a0) - 1.0;
    const double gmA = p.ea * dA / a0;
    const double2 ns = s_seg[t];
    const double2 ps = s_seg[lp];
    // nRel - pRel = pos[next] - pos[prev]
    const double2 npd = make_double2(ns.x + ps.x, ns.y + ps.y);
    fsh.x += 0.5 * gmA * (-npd.y);
    fsh.y += 0.5 * gmA * (npd.x);
    esh += (0.5 * p.ea * dA * dA) / nvr;
    const double plen = dist_of(ps), nlen = dist_of(ns);
    const double tl0 = a.l0[v], pl0 = a.l0[vp];
    if (p.monomer == 0) {
      const double pd = (plen / pl0) - 1.0;
      const double nd = (nlen / tl0) - 1.0;
      fsh.x += p.el * ((nd * ns.x / (tl0 * nlen)) - (pd * ps.x / (pl0 * plen)));
      fsh.y += p.el * ((nd * ns.y / (tl0 * nlen)) - (pd * ps.y / (pl0 * plen)));
      esh += 0.5 * p.el * pd * pd;
    } else {
      const double c = 2.0 * p.el * p.stiff * p.ext_sq;
      const double an = nlen / (p.ext_sq * tl0 * tl0 - nlen * nlen);
      const double ap = plen / (p.ext_sq * pl0 * pl0 - plen * plen);
      fsh.x += c * (an * ns.x / nlen - ap * ps.x / plen);
      fsh.y += c * (an * ns.y / nlen - ap * ps.y / plen);
      esh += p.el * p.stiff * p.ext_sq * log(1.0 - plen * plen / (p.ext_sq * pl0 * pl0));
    }
    const double prevAD = s_theta[lp] - a.theta0[vp];
    const double thisAD = s_theta[t] - a.theta0[v];
    const double nextAD = s_theta[ln] - a.theta0[vn];
    const double pvar = (thisAD - prevAD) / (ps.x * ps.x + ps.y * ps.y);
    const double nvar = (thisAD - nextAD) / (ns.x * ns.x + ns.y * ns.y);
    fsh.x += p.eb * (pvar * ps.y + nvar * ns.y);
    fsh.y += p.eb * (pvar * (-ps.x) + nvar * (-ns.x));
    esh += 0.5 * p.eb * thisAD * thisAD;
  }

  // ---- phase 3: pair forces ------------------------------------------------
  {
    const int lv = t / L, lane = t % L;
    double2 fi = make_double2(0.0, 0.0), fq = make_double2(0.0, 0.0);
    double ei = 0.0;
    if (lv < nvt) {
      const int i = v0 + lv;
      const double2 xi = s_pos[lv];
      const double ri = a.rad[i];
      const int cnt = min(a.nbr_cnt[i], a.nbr_cap);  // a build that overflowed stores counts above capacity
      if constexpr (INTER == INT_VV) {
        for (int sl = lane; sl < cnt; sl += L) {
          const int j = __ldg(a.nbr + (size_t)sl * p.nv + i);
          const double2 xj = a.pos[j];
          pair_own<POT>(p, pbc2(p, xi, xj), ri + __ldg(a.rad + j), fi, ei);
        }
      } else {
        // local segment data of this vertex i as "o": q = prev(i), qq = prev(q)
        const int lq = s_lp[lv];
        const int lqq = s_lp[lq];
        const double2 xq = s_pos[lq], xqq = s_pos[lqq];
        const double2 seg_i = s_seg[lq];    // pbc(x_i - x_q)
        const double2 pseg_i = s_seg[lqq];  // pbc(x_q - x_qq)
        const double len2_i = fma(seg_i.y, seg_i.y, seg_i.x * seg_i.x);
        const double range = pot_range<POT>(p);
        double2 dummy = make_double2(0.0, 0.0);
        for (int sl = lane; sl < cnt; sl += L) {
          const int j = __ldg(a.nbr + (size_t)sl * p.nv + i);
          const double2 xj = a.pos[j];
          const double rsum = ri + __ldg(a.rad + j);
          const int2 pq = __ldg(a.pp_of + j);
          const double2 xjq = a.pos[pq.x];
          const double R = range * rsum;
          const double inv_rsum = 1.0 / rsum;
          const double2 w1 = pbc2(p, xi, xj);  // role 1: t = i, o = j
          const double w2 = fma(w1.y, w1.y, w1.x * w1.x);
          {
            // role 1: i against the segment prev(j) -> j of the other ring
            const double2 tq = pbc2(p, xi, xjq);
            const double tq2 = fma(tq.y, tq.y, tq.x * tq.x);
            const double2 seg = pbc2(p, xj, xjq);
            const double len2 = fma(seg.y, seg.y, seg.x * seg.x);
            if (!smooth_out_of_range(R, tq2, w2, len2)) {
              const double2 xjqq = a.pos[pq.y];
              smooth_core<POT, true>(p, xi, xjq, xjqq, seg, len2, pbc2(p, xjq, xjqq), tq, tq2, w1, rsum, inv_rsum,
                                     fi, dummy, dummy, ei);
            }
          }
          {
            // role 2: neighbour j against this vertex's segment prev(i) -> i
            const double2 tq = pbc2(p, xj, xq);
            const double tq2 = fma(tq.y, tq.y, tq.x * tq.x);
            if (!smooth_out_of_range(R, tq2, w2, len2_i)) {
              smooth_core<POT, false>(p, xj, xq, xqq, seg_i, len2_i, pseg_i, tq, tq2,
                                      make_double2(-w1.x, -w1.y), rsum, inv_rsum, dummy, fi, fq, ei);
            }
          }
        }
      }
    }
    // reduce over the L lanes of this vertex (lanes are contiguous in a warp)
#pragma unroll
    for (int o = L >> 1; o > 0; o >>= 1) {
      fi.x += __shfl_xor_sync(0xffffffffu, fi.x, o);
      fi.y += __shfl_xor_sync(0xffffffffu, fi.y, o);
      ei += __shfl_xor_sync(0xffffffffu, ei, o);
      if constexpr (INTER == INT_SMOOTH) {
        fq.x += __shfl_xor_sync(0xffffffffu, fq.x, o);
        fq.y += __shfl_xor_sync(0xffffffffu, fq.y, o);
      }
    }
    if (lane == 0 && lv < nvt) {
      s_fpair[lv] = fi;
      s_epair[lv] = ei;
      s_fprev[lv] = fq;
    }
  }
  __syncthreads();

  // ---- phase 4: totals and outputs ----------------------------------------
  double2 F = make_double2(0.0, 0.0);
  double evtx = 0.0;  // per-vertex energy as the reference stores it
  double epair = 0.0;
  if (t < nvt) {
    const double2 fp = s_fpair[t];
    F.x = fsh.x + fp.x;
    F.y = fsh.y + fp.y;
    if constexpr (INTER == INT_SMOOTH) {
      const double2 fn = s_fprev[s_ln[t]];
      F.x += fn.x;
      F.y += fn.y;
      evtx = esh;
    } else {
      evtx = esh + s_epair[t];
    }
    epair = s_epair[t];
  }

  if constexpr (MODE == MODE_FORCE) {
    if (t < nvt) {
      const int v = v0 + t;
      double2 Fo = F;
      if (s.active) {
        // DPM2D::addSelfPropulsion with the angle already advanced by the caller
        const double psi = s.p_angle[ring];
        double sn, cs;
        sincos(psi, &sn, &cs);
        Fo.x += s.driving * cs;
        Fo.y += s.driving * sn;
      }
      s.force[v] = Fo;
      s.energy[v] = evtx;
      s.theta_out[v] = s_theta[t];
      s.length_out[v] = dist_of(s_seg[t]);
      if (k == 0) {
        s.area_out[ring] = fabs(s_r0[t]) * 0.5;
        s.perim_out[ring] = s_r1[t];
        const double2 x0 = s_pos[t];
        s.ppos_out[ring] = make_double2(x0.x + s_r2[t].x / nvr, x0.y + s_r2[t].y / nvr);
      }
    }
    if constexpr (INTER == INT_SMOOTH) {
      // ring energy = sum of the unit energies gathered by its vertices
      __syncthreads();
      if (t < nvt) s_r1[t] = epair;
      for (int stride = 1; stride < TV; stride <<= 1) {
        __syncthreads();
        if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) s_r1[t] += s_r1[t + stride];
      }
      __syncthreads();
      if (t < nvt && k == 0) s.p_energy[ring] = s_r1[t];
    }
    return;
  } else {
    // ---- MODE_STEP: integrator tail (src/Simulator.cu, src/FIRE.cu) ----------
    double sums[NSUM] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const unsigned long long step = (unsigned long long)st->rng_step;
    if (s.active) {
      // addSelfPropulsion (src/DPM2D.cu:1995-2035): the ring's angle takes a
      // N(0, sqrt(2 dt / taup)) increment and is wrapped to [-pi, pi); the
      // ring's first vertex updates it once and shares it through its s_theta
      // slot, which the step tail no longer reads
      if (t < nvt && k == 0) {
        double psi = s.p_angle[ring];
        const double2 z = philox_normal2(s.seed, 2ull * step + 1ull, (unsigned long long)ring);
        psi += s.sp_amp * z.x;
        psi = psi + kPi;
        psi = psi - 2.0 * kPi * floor(psi / (2.0 * kPi));
        psi = psi - kPi;
        s.p_angle[ring] = psi;
        s_theta[t] = psi;
      }
      __syncthreads();
      if (t < nvt) {
        double sn, cs;
        sincos(s_theta[lf], &sn, &cs);
        F.x += s.driving * cs;
        F.y += s.driving * sn;
      }
    }
    if (t < nvt) {
      const int v = v0 + t;
      double2 vh = s.vel[v];
      const double2 x = s_pos[t];
      double2 vn;
      double hdt = s.hdt;
      if (s.kind == KIND_FIRE) hdt = 0.5 * s.fire_state[((st->fire_iters + 1) & 1) * 4];
      if (s.kind == KIND_LANGEVIN) {
        // langevinAddThermostatForces (src/Simulator.cu:68-73)
        const double2 z = philox_normal2(s.seed, 2ull * step, (unsigned long long)ring);
        F.x += s.noise * z.x - s.gamma * vh.x;
        F.y += s.noise * z.y - s.gamma * vh.y;
      }
      if (s.kind == KIND_BROWNIAN || s.kind == KIND_DRIVEN_BROWNIAN) {
        // updateBrownianVel / updateDrivenBrownianVel (src/Simulator.cu:168-200)
        if (s.kind == KIND_BROWNIAN) {
          const double2 z = philox_normal2(s.seed, 2ull * step, (unsigned long long)ring);
          vn = make_double2((F.x + s.noise * z.x) / s.gamma, (F.y + s.noise * z.y) / s.gamma);
        } else {
          vn = make_double2(F.x / s.gamma, F.y / s.gamma);
        }
        const double2 xn = make_double2(x.x + s.dt * vn.x, x.y + s.dt * vn.y);
        s.pos_out[v] = xn;
        s.vel[v] = vn;
        s.force[v] = F;
        if (s.write_out) s.energy[v] = evtx;
        const double2 lp = s.last_pos[v];
        if (3.0 * dist_of(pbc2(p, xn, lp)) > s.disp_cutoff) st->rebuild = 1;
      } else {
        // second half kick (kernelUpdateVertexVel, include/cudaKernel.cuh:1989-1996)
        vn = make_double2(vh.x + hdt * F.x, vh.y + hdt * F.y);
        if (s.advance) {
          double2 vh2, xn;
          if (s.kind == KIND_BAOAB) {
            // BAOAB::integrate (src/Simulator.cu:112-144) for the next step
            vh2 = make_double2(vn.x + s.hdt * F.x, vn.y + s.hdt * F.y);
            xn = make_double2(x.x + s.hdt * vh2.x, x.y + s.hdt * vh2.y);
            const double2 z = philox_normal2(s.seed, 2ull * (step + 1ull), (unsigned long long)ring);
            vh2 = make_double2(s.gamma_factor * vh2.x + s.noise * z.x, s.gamma_factor * vh2.y + s.noise * z.y);
            xn = make_double2(xn.x + s.hdt * vh2.x, xn.y + s.hdt * vh2.y);
          } else {
            vh2 = make_double2(vn.x + s.hdt * F.x, vn.y + s.hdt * F.y);
            xn = make_double2(x.x + s.dt * vh2.x, x.y + s.dt * vh2.y);
          }
          s.pos_out[v] = xn;
          s.vel[v] = vh2;
          const double2 lp = s.last_pos[v];
          if (3.0 * dist_of(pbc2(p, xn, lp)) > s.disp_cutoff) st->rebuild = 1;
        } else {
          s.vel[v] = vn;
          s.force[v] = F;
          if (s.write_out) s.energy[v] = evtx;
        }
      }
      if (s.accumulate) {
        sums[S_PE] = evtx + ((INTER == INT_SMOOTH) ? epair : 0.0);
        sums[S_VV] = vn.x * vn.x + vn.y * vn.y;
        sums[S_VF] = vn.x * F.x + vn.y * F.y;
        sums[S_FF] = F.x * F.x + F.y * F.y;
        sums[S_FMAX2] = fmax(F.x * F.x, F.y * F.y);
      }
      if (!(isfinite(F.x) && isfinite(F.y))) sums[S_NONFINITE] = 1.0;
    }
    if (s.write_out && INTER == INT_SMOOTH) {
      __syncthreads();
      if (t < nvt) s_r1[t] = epair;
      for (int stride = 1; stride < TV; stride <<= 1) {
        __syncthreads();
        if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) s_r1[t] += s_r1[t + stride];
      }
      __syncthreads();
      if (t < nvt && k == 0) s.p_energy[ring] = s_r1[t];
    }
    // per-CTA partials in a fixed order
    {
      const int warp = t / 32, wl = t % 32;
#pragma unroll
      for (int q = 0; q < NSUM; q++) {
        double x = sums[q];
        for (int o = 16; o > 0; o >>= 1) {
          double y = __shfl_xor_sync(0xffffffffu, x, o);
          x = (q == S_FMAX2) ? fmax(x, y) : x + y;
        }
        if (wl == 0) s_red[warp][q] = x;
      }
      __syncthreads();
      if (t < NSUM) {
        double x = (t == S_FMAX2) ? 0.0 : 0.0;
        for (int w = 0; w < BLOCK / 32; w++) x = (t == S_FMAX2) ? fmax(x, s_red[w][t]) : x + s_red[w][t];
        s.partials[(size_t)blockIdx.x * NSUM + t] = x;
      }
    }
    if (is_last_block(st)) {
      reduce_partials(s.partials, gridDim.x, st->sums);
      __syncthreads();
      if (t == 0) {
        __threadfence();
        if (st->sums[S_NONFINITE] != 0.0) { st->nonfinite = 1; st->abort = 1; }
        if (s.kind == KIND_FIRE) {
          st->fire_iters += 1;
          if (s.fire_tol >= 0.0 && st->sums[S_FMAX2] <= s.fire_tol * s.fire_tol) st->converged = 1;
        }
        st->ops_done += 1;
        if (s.kind != KIND_FIRE) st->rng_step += 1;
        st->done_ctr = 0;
        if (s.use_cond) cudaGraphSetConditional(s.cond, st->rebuild ? 1u : 0u);
      }
    }
  }
}

// ---------------------------------------------------------------- launchers

template <int POT, int INTER, int MODE>
static void launch_tile_t(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s) {
  if (c.lanes == 1) k_tile<POT, INTER, MODE, 128, 1><<<c.grid, 128, 0, c.stream>>>(p, a, s);
  else if (c.lanes == 4) k_tile<POT, INTER, MODE, 256, 4><<<c.grid, 256, 0, c.stream>>>(p, a, s);
  else if (c.lanes == 8) k_tile<POT, INTER, MODE, 256, 8><<<c.grid, 256, 0, c.stream>>>(p, a, s);
  else k_tile<POT, INTER, MODE, 128, 2><<<c.grid, 128, 0, c.stream>>>(p, a, s);
}

void launch_tile(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                 const StepArgs& s) {
#define CR_TILE_CASE(P)                                                                 \
  case P:                                                                               \
    if (inter == INT_VV) {                                                              \
      if (mode == MODE_FORCE) launch_tile_t<P, INT_VV, MODE_FORCE>(c, p, a, s);         \
      else launch_tile_t<P, INT_VV, MODE_STEP>(c, p, a, s);                             \
    } else {                                                                            \
      if (mode == MODE_FORCE) launch_tile_t<P, INT_SMOOTH, MODE_FORCE>(c, p, a, s);     \
      else launch_tile_t<P, INT_SMOOTH, MODE_STEP>(c, p, a, s);                         \
    }                                                                                   \
    break;
  switch (pot) {
    CR_TILE_CASE(POT_HARMONIC)
    CR_TILE_CASE(POT_LJ)
    CR_TILE_CASE(POT_ADHESIVE)
    CR_TILE_CASE(POT_WCA)
    default: break;
  }
#undef CR_TILE_CASE
}

// Tile capacity (vertices of whole rings per CTA) for a lane count:
// 1 -> 128 threads x 1, 2 -> 128 x 2, 4 -> 256 x 4, 8 -> 256 x 8.
int tile_vertices(int lanes) { return lanes >= 4 ? 256 / lanes : 128 / (lanes <= 0 ? 2 : lanes); }

}  // namespace cr
