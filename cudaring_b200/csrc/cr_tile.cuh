// Tiled force + integrator kernel for one system (sm_100a, FP64).
//
// One CTA owns a tile of whole rings (<= TV = BLOCK / L vertices).  Phases:
//   1. ring geometry in shared memory: segment vectors, turning angles,
//      shoelace area, perimeter and centroid by a deterministic per-ring tree;
//   2. shape force per vertex (area, segment length or FENE, bending);
//   3. pair forces with L lanes per vertex striding over the slot-major
//      neighbour list; the smooth vertex-segment interaction is evaluated in a
//      gather form (smooth_unit, roles 1 and 2) so no global atomics are needed
//      and the result does not depend on scheduling order;
//   4. integrator tail: the second half kick of this step and, when the op
//      advances, the first half kick + drift of the next step written to a
//      second position buffer (ping-pong), plus the displacement check that
//      arms a neighbour-list rebuild.
#pragma once
#include "cr_common.cuh"

namespace cr {

enum Mode : int { MODE_FORCE = 0, MODE_STEP = 1 };
enum Kind : int {
  KIND_NVE = 0, KIND_LANGEVIN = 1, KIND_BAOAB = 2, KIND_BROWNIAN = 3, KIND_DRIVEN_BROWNIAN = 4,
  KIND_FIRE = 5, KIND_NONE = 6
};

constexpr int NSUM = 6;  // per-CTA partial sums: PE, sum v^2, v.F, sum v^2 (again), sum F^2, max F_d^2
enum SumIdx : int { S_PE = 0, S_VV = 1, S_VF = 2, S_FF = 3, S_FMAX2 = 4, S_NONFINITE = 5 };

struct StepArgs {
  double2* pos_out;        // next positions (MODE_STEP with advance)
  double2* vel;
  double2* force;
  const double2* last_pos;
  double* energy;          // per vertex
  double* p_energy;        // per ring (smooth interaction energies)
  double* theta_out;
  double* length_out;
  double* area_out;
  double* perim_out;
  double2* ppos_out;
  double* p_angle;         // self-propulsion angle per ring (active rings)
  double* partials;        // [gridDim.x][NSUM]
  DevStatus* status;
  const double* fire_state;  // [2][4] FIRE scalars {dt, a, numStep, -}, double-buffered by iteration parity
  cudaGraphConditionalHandle cond;
  int use_cond;
  int kind;
  int advance;
  int write_out;           // write force/energy/per-ring outputs
  int accumulate;          // per-CTA partial sums + final reduction by the last CTA
  int active;
  double dt, hdt, gamma, noise, gamma_factor;
  double driving, sp_amp;
  double disp_cutoff;
  double fire_tol;
  unsigned long long seed;
};

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ double dist_of(double2 dl) {
  double sq = dl.x * dl.x;
  sq = fma(dl.y, dl.y, sq);
  return sqrt(sq);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) -> two standard normals
// by Box-Muller.  counter = (index, stream), key = seed.
__device__ __forceinline__ double2 philox_normal2(unsigned long long seed, unsigned long long stream,
                                                  unsigned long long index) {
  uint32_t c0 = (uint32_t)index, c1 = (uint32_t)(index >> 32), c2 = (uint32_t)stream, c3 = (uint32_t)(stream >> 32);
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  unsigned long long a = (unsigned long long)c0 | ((unsigned long long)c1 << 32);
  unsigned long long b = (unsigned long long)c2 | ((unsigned long long)c3 << 32);
  double u1 = ((double)(a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
  double rr = sqrt(-2.0 * log(u1));
  double s, c;
  sincos(2.0 * kPi * u2, &s, &c);
  return make_double2(rr * c, rr * s);
}

// Interaction range in units of radSum: the distance beyond which every pair
// term of the potential is exactly zero.
template <int POT>
__device__ __forceinline__ double pot_range(const SysParams& p) {
  if constexpr (POT == POT_HARMONIC) return 1.0;
  else if constexpr (POT == POT_LJ) return p.lj_cutoff;
  else if constexpr (POT == POT_ADHESIVE) return 1.0 + p.l2;
  else return kWCAcut;
}

// Pair term from the squared distance: returns whether the pair is in range
// (the reference's own test), gradMultiple gm (force on "this" = gm * delta / d),
// 1/d and the half-pair energy.  Same arithmetic as calcContactInteraction ..
// calcWCAInteraction / calcGradMultipleAndEnergy (include/cudaKernel.cuh:531-668,
// 806-858) with the divisions by d and radSum taken as products with one
// reciprocal square root and one reciprocal (rounding-level differences).
template <int POT>
__device__ __forceinline__ bool pair_eval(const SysParams& p, double d2, double rsum, double inv_rsum, double& gm,
                                          double& inv_d, double& ep) {
  inv_d = rsqrt(d2);
  const double d = d2 * inv_d;
  if constexpr (POT == POT_HARMONIC) {
    const double ov = 1.0 - d * inv_rsum;
    if (!(ov > 0.0)) return false;
    gm = p.ec * ov * inv_rsum;
    ep = (0.5 * p.ec * ov * ov) * 0.5;
    return true;
  } else if constexpr (POT == POT_LJ) {
    if (!(d <= p.lj_cutoff * rsum)) return false;
    const double ratio = rsum * inv_d;
    const double r2 = ratio * ratio;
    const double r6 = r2 * r2 * r2;
    const double r12 = r6 * r6;
    const double fshift = p.lj_fshift * inv_rsum;
    gm = 24.0 * p.ec * (2.0 * r12 - r6) * inv_d - fshift;
    ep = 0.5 * (4.0 * p.ec * (r12 - r6) - p.lj_ecut - fabs(fshift) * (d - p.lj_cutoff * rsum));
    return true;
  } else if constexpr (POT == POT_ADHESIVE) {
    if (!(d < (1.0 + p.l2) * rsum)) return false;
    const double ov = 1.0 - d * inv_rsum;
    if (d < (1.0 + p.l1) * rsum) {
      gm = p.ec * ov * inv_rsum;
      ep = 0.5 * p.ec * (ov * ov - p.l1 * p.l2) * 0.5;
    } else {
      const double k = p.ec * p.l1 / (p.l2 - p.l1);
      gm = -k * (ov + p.l2) * inv_rsum;
      ep = -(0.5 * k * (ov + p.l2) * (ov + p.l2)) * 0.5;
    }
    return true;
  } else {
    if (!(d <= kWCAcut * rsum)) return false;
    const double ratio = rsum * inv_d;
    const double r2 = ratio * ratio;
    const double r6 = r2 * r2 * r2;
    const double r12 = r6 * r6;
    gm = 24.0 * p.ec * (2.0 * r12 - r6) * inv_d;
    ep = 0.5 * p.ec * (4.0 * (r12 - r6) + 1.0);
    return true;
  }
}

// Own-side vertex-vertex term of kernelCalcVertexInteraction (:690-722).
template <int POT>
__device__ __forceinline__ void pair_own(const SysParams& p, double2 dl, double rsum, double2& f, double& e) {
  const double d2 = fma(dl.y, dl.y, dl.x * dl.x);
  const double R = pot_range<POT>(p) * rsum * (1.0 + 1e-12);
  if (d2 > R * R) return;  // exactly zero beyond the range
  double gm, inv_d, ep = 0.0;
  if (pair_eval<POT>(p, d2, rsum, 1.0 / rsum, gm, inv_d, ep)) {
    const double s = gm * inv_d;
    f.x += s * dl.x;
    f.y += s * dl.y;
    e += ep;
  }
}

// sign = cross / |cross| of calcVertexSegmentInteraction (:882-884), NaN for
// cross == 0 exactly as there.
__device__ __forceinline__ double sign_of(double c) {
  return c > 0.0 ? 1.0 : (c < 0.0 ? -1.0 : __longlong_as_double(0x7ff8000000000000LL));
}

// Smooth unit from precomputed geometry.  t: the vertex, o: segment end,
// q = prev(o), qq = prev(q); seg = pbc(o - q), pseg = pbc(q - qq),
// tq = pbc(t - q), w = pbc(t - o), tq2 = |tq|^2.  See smooth_unit.
template <int POT, bool ROLE1>
__device__ __forceinline__ void smooth_core(const SysParams& p, double2 t, double2 q, double2 qq, double2 seg,
                                            double len2, double2 pseg, double2 tq, double tq2, double2 w,
                                            double rsum, double inv_rsum, double2& ft, double2& fo, double2& fq,
                                            double& e) {
  const double inv_len = rsqrt(len2);
  const double inv_lsq = inv_len * inv_len;
  const double proj = (tq.x * seg.x + tq.y * seg.y) * inv_lsq;
  const double2 tqq = pbc2(p, t, qq);
  const double pinv = rsqrt(fma(pseg.y, pseg.y, pseg.x * pseg.x));
  const double pproj = (tqq.x * pseg.x + tqq.y * pseg.y) * (pinv * pinv);
  if (proj >= 0.0 && proj < 1.0) {
    const double2 pj = make_double2(q.x + proj * seg.x, q.y + proj * seg.y);
    const double2 dp = pbc2(p, t, pj);
    double gm, inv_d, ep = 0.0;
    if (pair_eval<POT>(p, fma(dp.y, dp.y, dp.x * dp.x), rsum, inv_rsum, gm, inv_d, ep) && gm != 0.0) {
      const double cross = seg.x * w.y - w.x * seg.y;
      const double sign = sign_of(cross);
      const double g = gm * inv_len;
      if constexpr (ROLE1) {
        ft.x += g * sign * (-seg.y);
        ft.y += g * sign * seg.x;
      } else {
        const double a = fabs(cross) * inv_lsq;
        fo.x += g * (sign * tq.y - a * seg.x);
        fo.y += g * (-sign * tq.x - a * seg.y);
        fq.x += g * (-sign * w.y + a * seg.x);
        fq.y += g * (sign * w.x + a * seg.y);
      }
      e += ep;
    }
    if (pproj >= 0.0 && pproj < 1.0) {
      // calcVertexVertexInteraction(previousPos, thisPos, ...): delta = pbc(q - t)
      double g2, id2, ep2 = 0.0;
      if (pair_eval<POT>(p, tq2, rsum, inv_rsum, g2, id2, ep2) && g2 != 0.0) {
        const double s2 = g2 * id2;
        if constexpr (ROLE1) {
          ft.x -= s2 * tq.x;
          ft.y -= s2 * tq.y;
        } else {
          fq.x += s2 * tq.x;
          fq.y += s2 * tq.y;
        }
        e -= ep2;
      }
    }
  } else if (proj < 0.0 && pproj >= 1.0) {
    // calcVertexVertexInteraction(thisPos, previousPos, ...): delta = pbc(t - q)
    double g2, id2, ep2 = 0.0;
    if (pair_eval<POT>(p, tq2, rsum, inv_rsum, g2, id2, ep2) && g2 != 0.0) {
      const double s2 = g2 * id2;
      if constexpr (ROLE1) {
        ft.x += s2 * tq.x;
        ft.y += s2 * tq.y;
      } else {
        fq.x -= s2 * tq.x;
        fq.y -= s2 * tq.y;
      }
      e += ep2;
    }
  }
}

// True when no term of a smooth unit can be in range: every point of the
// segment is at least max(|t-o|, |t-q|) - |o-q| from t, and both corrections
// use |t-q|.  The relative margin covers rounding, so a skipped unit is one
// that would have contributed exactly zero.
__device__ __forceinline__ bool smooth_out_of_range(double R, double tq2, double w2, double len2) {
  const double Rm = R * (1.0 + 1e-12);
  if (!(tq2 > Rm * Rm)) return false;
  const double lim = Rm + sqrt(len2);
  return fmax(tq2, w2) > lim * lim;
}

// One unit U(t; o) of kernelCalcSmoothInteraction (include/cudaKernel.cuh:922-975):
// vertex t against the segment q -> o (q = prev(o)) of another ring, with the
// concave correction (t also projects onto qq -> q: subtract the t-q
// vertex-vertex term) and the convex one (t before q on both segments: add
// it).  ROLE1 (t is this vertex) returns the force on t; ROLE2 (o is this
// vertex, t a neighbour) returns the forces on o and on q.  Both add the unit
// energy, which the reference books on the rings of t and of o.
//   seg = pbc(o - q), pseg = pbc(q - qq).
template <int POT, bool ROLE1>
__device__ __forceinline__ void smooth_unit(const SysParams& p, double2 t, double2 o, double2 q, double2 qq,
                                            double2 seg, double2 pseg, double rsum, double2& ft, double2& fo,
                                            double2& fq, double& e) {
  double len = dist_of(seg);
  double lsq = len * len;
  double2 tq = pbc2(p, t, q);
  double proj = (tq.x * seg.x + tq.y * seg.y) / lsq;
  double plen = dist_of(pseg);
  double2 tqq = pbc2(p, t, qq);
  double pproj = (tqq.x * pseg.x + tqq.y * pseg.y) / (plen * plen);
  if (proj >= 0.0 && proj < 1.0) {
    double2 pj = make_double2(q.x + proj * seg.x, q.y + proj * seg.y);
    double dp = dist_of(pbc2(p, t, pj));
    double ep = 0.0;
    double gm = pair_gm<POT>(p, dp, rsum, ep);
    if (gm != 0.0) {
      double2 w = pbc2(p, t, o);
      double cross = seg.x * w.y - w.x * seg.y;
      double ac = fabs(cross);
      double sign = cross / ac;
      if constexpr (ROLE1) {
        ft.x += gm * sign * (-seg.y) / len;
        ft.y += gm * sign * seg.x / len;
      } else {
        fo.x += gm * (sign * tq.y - ac * seg.x / lsq) / len;
        fo.y += gm * (-sign * tq.x - ac * seg.y / lsq) / len;
        fq.x += gm * (-sign * w.y + ac * seg.x / lsq) / len;
        fq.y += gm * (sign * w.x + ac * seg.y / lsq) / len;
      }
      e += ep;
    }
    if (pproj >= 0.0 && pproj < 1.0) {
      // calcVertexVertexInteraction(previousPos, thisPos, ...): delta = pbc(q - t)
      double d = dist_of(tq);
      double ep2 = 0.0;
      double g2 = pair_gm<POT>(p, d, rsum, ep2);
      if (g2 != 0.0) {
        if constexpr (ROLE1) {
          ft.x += g2 * (-tq.x) / d;
          ft.y += g2 * (-tq.y) / d;
        } else {
          fq.x += g2 * tq.x / d;
          fq.y += g2 * tq.y / d;
        }
        e -= ep2;
      }
    }
  } else if (proj < 0.0) {
    if (pproj >= 1.0) {
      // calcVertexVertexInteraction(thisPos, previousPos, ...): delta = pbc(t - q)
      double d = dist_of(tq);
      double ep2 = 0.0;
      double g2 = pair_gm<POT>(p, d, rsum, ep2);
      if (g2 != 0.0) {
        if constexpr (ROLE1) {
          ft.x += g2 * tq.x / d;
          ft.y += g2 * tq.y / d;
        } else {
          fq.x -= g2 * tq.x / d;
          fq.y -= g2 * tq.y / d;
        }
        e += ep2;
      }
    }
  }
}

// Last-CTA epilogue shared by all per-step kernels: sums the per-CTA partials
// in a fixed order, updates the status block and arms the rebuild
// conditional of the enclosing CUDA graph.  Must be called by every thread.
__device__ __forceinline__ bool is_last_block(DevStatus* st) {
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned int prev = atomicAdd(&st->done_ctr, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  return s_last;
}

__device__ __forceinline__ void reduce_partials(const double* partials, int nblocks, double* out) {
  // one warp, fixed order: lane l sums blocks l, l+32, ... then a fixed tree
  int lane = threadIdx.x;
  if (lane < 32) {
    double acc[NSUM];
#pragma unroll
    for (int k = 0; k < NSUM; k++) acc[k] = 0.0;
    for (int b = lane; b < nblocks; b += 32) {
#pragma unroll
      for (int k = 0; k < NSUM; k++) {
        double x = __ldcg(partials + (size_t)b * NSUM + k);
        acc[k] = (k == S_FMAX2) ? fmax(acc[k], x) : acc[k] + x;
      }
    }
#pragma unroll
    for (int k = 0; k < NSUM; k++) {
      for (int o = 16; o > 0; o >>= 1) {
        double y = __shfl_xor_sync(0xffffffffu, acc[k], o);
        acc[k] = (k == S_FMAX2) ? fmax(acc[k], y) : acc[k] + y;
      }
      if (lane == 0) out[k] = acc[k];
    }
  }
}

}  // namespace cr
