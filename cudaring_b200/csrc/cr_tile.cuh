// Tiled force + integrator kernel for one system (sm_100a, FP64).
//
// One CTA owns a tile of whole rings (<= TV = BLOCK / L vertices).  Phases:
//   1. ring geometry in shared memory: segment vectors, turning angles,
//      shoelace area, perimeter and centroid by a deterministic per-ring tree;
//   2. shape force per vertex (area, segment length or FENE, bending);
//   3. pair forces with L lanes per vertex striding over the slot-major
//      neighbour list; the smooth vertex-segment interaction is evaluated in a
//      gather form (smooth_core, roles 1 and 2) so no global atomics are needed
//      and the result does not depend on scheduling order;
//   4. integrator tail: the second half kick of this step and, when the op
//      advances, the first half kick + drift of the next step written to a
//      second position buffer (ping-pong), plus the displacement check that
//      arms a neighbour-list rebuild.
#pragma once
#include <type_traits>

#include "cr_common.cuh"

namespace cr {

enum Mode : int { MODE_FORCE = 0, MODE_STEP = 1 };
enum Kind : int {
  KIND_NVE = 0, KIND_LANGEVIN = 1, KIND_BAOAB = 2, KIND_BROWNIAN = 3, KIND_DRIVEN_BROWNIAN = 4,
  KIND_FIRE = 5, KIND_NONE = 6, KIND_NVE_RESCALE = 7
};

constexpr int NSUM = 6;  // per-CTA partial sums: PE, sum v^2, v.F, sum v^2 (again), sum F^2, max F_d^2
enum SumIdx : int { S_PE = 0, S_VV = 1, S_VF = 2, S_FF = 3, S_FMAX2 = 4, S_NONFINITE = 5 };

// One system of a batch: its box, rebuild/convergence flags, FIRE counters
// and the sums its last tile reduces from its tiles' partials.
struct BatchSys {
  Box box;
  double disp_cutoff;      // DPM2D::cutoff of this system
  double fire_tol;         // FIRE stops when max_i,d |F_i,d| <= fire_tol (< 0: never)
  double sums[NSUM];
  long long fire_iters;
  int tile_begin, tile_end;
  int rebuild;             // this system's displacement check fired
  int converged;           // FIRE reached fire_tol: the system is frozen
  int active;              // 0: the system takes no part in step ops
  unsigned int done_ctr;   // tiles of this system finished in the current op
  long long fire_cap;      // > 0: FIRE stops (marks the system converged) after this many iterations
};

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
  double rescale_T;        // > 0: scale velocities to this temperature before the kick (NVERescale)
  BatchSys* bsys;          // batch mode: per-system table (tile.x is the system)
  const double* bfire_state;  // batch mode: [S][2][4] FIRE scalars per system
  unsigned long long seed;
  int persist_max;          // multi-step kernel: most steps per launch
};

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ double dist_of(double2 dl) {
  double sq = dl.x * dl.x;
  sq = fma(dl.y, dl.y, sq);
  return sqrt(sq);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): four 32-bit words for
// counter = (index, stream), key = seed.
__device__ __forceinline__ uint4 philox4x32(unsigned long long seed, unsigned long long stream,
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
  return make_uint4(c0, c1, c2, c3);
}

// Two uniforms on [0, 1) with 53-bit resolution from one Philox block.
__device__ __forceinline__ double2 philox_uniform2(unsigned long long seed, unsigned long long stream,
                                                   unsigned long long index) {
  const uint4 w = philox4x32(seed, stream, index);
  const unsigned long long a = (unsigned long long)w.x | ((unsigned long long)w.y << 32);
  const unsigned long long b = (unsigned long long)w.z | ((unsigned long long)w.w << 32);
  return make_double2((double)(a >> 11) * (1.0 / 9007199254740992.0), (double)(b >> 11) * (1.0 / 9007199254740992.0));
}

// Two standard normals by Box-Muller from one Philox block.
__device__ __forceinline__ double2 philox_normal2(unsigned long long seed, unsigned long long stream,
                                                  unsigned long long index) {
  const uint4 w = philox4x32(seed, stream, index);
  const uint32_t c0 = w.x, c1 = w.y, c2 = w.z, c3 = w.w;
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

// ----------------------------------------------------------------------------
// FP32 pair arithmetic of the mixed-precision path.  Offsets arrive as the
// FP64 minimum-image differences rounded to float; every smooth unit is
// written in coordinates relative to its vertex t (tq = t - q, tqq = t - qq,
// w = t - o), so no absolute coordinate is ever held in float.
// ----------------------------------------------------------------------------

__device__ __forceinline__ float2 f2(double2 d) { return make_float2((float)d.x, (float)d.y); }

template <int POT>
__device__ __forceinline__ float pot_range_f(const SysParams& p) {
  if constexpr (POT == POT_HARMONIC) return 1.0f;
  else if constexpr (POT == POT_LJ) return p.f_lj_cutoff;
  else if constexpr (POT == POT_ADHESIVE) return 1.0f + p.f_l2;
  else return (float)kWCAcut;
}

template <int POT>
__device__ __forceinline__ bool pair_eval_f(const SysParams& p, float d2, float rsum, float inv_rsum, float& gm,
                                            float& inv_d, float& ep) {
  inv_d = rsqrtf(d2);
  const float d = d2 * inv_d;
  const float ec = p.f_ec;
  if constexpr (POT == POT_HARMONIC) {
    const float ov = 1.0f - d * inv_rsum;
    if (!(ov > 0.0f)) return false;
    gm = ec * ov * inv_rsum;
    ep = 0.25f * ec * ov * ov;
    return true;
  } else if constexpr (POT == POT_LJ) {
    const float rc = p.f_lj_cutoff;
    if (!(d <= rc * rsum)) return false;
    const float ratio = rsum * inv_d;
    const float r2 = ratio * ratio;
    const float r6 = r2 * r2 * r2;
    const float r12 = r6 * r6;
    const float fshift = p.f_lj_fshift * inv_rsum;
    gm = 24.0f * ec * (2.0f * r12 - r6) * inv_d - fshift;
    ep = 0.5f * (4.0f * ec * (r12 - r6) - p.f_lj_ecut - fabsf(fshift) * (d - rc * rsum));
    return true;
  } else if constexpr (POT == POT_ADHESIVE) {
    const float l1 = p.f_l1, l2 = p.f_l2;
    if (!(d < (1.0f + l2) * rsum)) return false;
    const float ov = 1.0f - d * inv_rsum;
    if (d < (1.0f + l1) * rsum) {
      gm = ec * ov * inv_rsum;
      ep = 0.25f * ec * (ov * ov - l1 * l2);
    } else {
      const float k = ec * l1 / (l2 - l1);
      gm = -k * (ov + l2) * inv_rsum;
      ep = -0.25f * k * (ov + l2) * (ov + l2);
    }
    return true;
  } else {
    if (!(d <= (float)kWCAcut * rsum)) return false;
    const float ratio = rsum * inv_d;
    const float r2 = ratio * ratio;
    const float r6 = r2 * r2 * r2;
    const float r12 = r6 * r6;
    gm = 24.0f * ec * (2.0f * r12 - r6) * inv_d;
    ep = 0.5f * ec * (4.0f * (r12 - r6) + 1.0f);
    return true;
  }
}

template <int POT>
__device__ __forceinline__ void pair_own_f(const SysParams& p, float2 dl, float rsum, float2& f, double& e) {
  const float d2 = fmaf(dl.y, dl.y, dl.x * dl.x);
  const float R = pot_range_f<POT>(p) * rsum * 1.00001f;
  if (d2 > R * R) return;
  float gm, inv_d, ep = 0.0f;
  if (pair_eval_f<POT>(p, d2, rsum, 1.0f / rsum, gm, inv_d, ep)) {
    const float s = gm * inv_d;
    f.x = fmaf(s, dl.x, f.x);
    f.y = fmaf(s, dl.y, f.y);
    e += (double)ep;
  }
}

__device__ __forceinline__ float sign_of_f(float c) {
  return c > 0.0f ? 1.0f : (c < 0.0f ? -1.0f : __int_as_float(0x7fc00000));
}

// ----------------------------------------------------------------------------
// Smooth vertex-segment unit, one form for FP64 (the plain path) and FP32
// (the mixed path's pair terms).
//
// One unit U(t; o) of kernelCalcSmoothInteraction (include/cudaKernel.cuh:922-975):
// vertex t against the segment q -> o (q = prev(o), qq = prev(q)) of another
// ring, with the concave correction (t also projects onto qq -> q: subtract
// the t-q vertex-vertex term) and the convex one (t before q on both
// segments: add it).  ROLE1 (t is this vertex) returns the force on t; ROLE2
// (o is this vertex, t a neighbour) returns the forces on o and on q.  Both
// add the unit energy, which the reference books on the rings of t and of o.
//
// Inputs are offsets from t: tq = t - q (minimum image), w = t - o, and the
// segment vectors seg = o - q, pseg = q - qq; tabs, qabs are t and q in box
// coordinates.  The reference forms t - qq and the projection point
// q + proj * seg explicitly.  Here
//   * FP64 forms the projection point as the reference does, in box
//     coordinates; FP32 takes the projection distance as |tq - proj * seg|
//     (the same point, relative to t, with no box-sized coordinate in FP32),
//   * pproj = (t - qq).pseg / |pseg|^2 = 1 + tq.pseg / |pseg|^2, so its tests
//     pproj in [0, 1) and pproj >= 1 read -|pseg|^2 <= tq.pseg < 0 and
//     tq.pseg >= 0, with neither t - qq nor a division (this moves the
//     decision only for pproj within rounding of 0 or 1).
// ----------------------------------------------------------------------------

// Arithmetic of the pair terms: FP64, or FP32 on FP64-formed offsets.
enum Prec : int { PREC_FP64 = 0, PREC_MIXED = 1 };

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double sgn_nan0(double c) { return sign_of(c); }
__device__ __forceinline__ float sgn_nan0(float c) { return sign_of_f(c); }
template <int POT>
__device__ __forceinline__ bool pair_eval_t(const SysParams& p, double d2, double rsum, double inv_rsum, double& gm,
                                            double& inv_d, double& ep) {
  return pair_eval<POT>(p, d2, rsum, inv_rsum, gm, inv_d, ep);
}
template <int POT>
__device__ __forceinline__ bool pair_eval_t(const SysParams& p, float d2, float rsum, float inv_rsum, float& gm,
                                            float& inv_d, float& ep) {
  return pair_eval_f<POT>(p, d2, rsum, inv_rsum, gm, inv_d, ep);
}

template <int POT, bool ROLE1, typename T, class B, typename T2 = typename Vec2<T>::type>
__device__ __forceinline__ void smooth_core(const SysParams& p, const B& bx, T2 tq, T tq2, T2 w, T2 seg, T len2,
                                            T2 pseg, T rsum, T inv_rsum, double2 tabs, double2 qabs, T2& ft,
                                            T2& fo, T2& fq, double& e) {
  const T inv_len = rsq(len2);
  const T inv_lsq = inv_len * inv_len;
  const T proj = (tq.x * seg.x + tq.y * seg.y) * inv_lsq;
  const T pc = tq.x * pseg.x + tq.y * pseg.y;
  const T pl2 = fma(pseg.y, pseg.y, pseg.x * pseg.x);
  // One evaluation of the pair term serves the segment term (the foot of the
  // perpendicular inside the segment) or, before the segment's start, the
  // corner term at |t - q|: a lane needs at most one of them, so a warp
  // whose lanes split between the two runs the pair term once.  The corner
  // term taken away inside the segment's span (concave corners) is the
  // second, rarer evaluation.
  const bool on_seg = proj >= T(0) && proj < T(1);
  const bool before = !on_seg && proj < T(0) && pc >= T(0);
  if (on_seg || before) {
    T d2 = tq2;
    if (on_seg) {
      T dpx, dpy;
      if constexpr (std::is_same<T, double>::value) {
        // FP64: the projection point in box coordinates, as the reference
        // forms it (pbcDistance(thisPos, previousPos + proj * segment)), so
        // that near-contact distances carry the same rounding as there
        const double2 pj = make_double2(qabs.x + proj * seg.x, qabs.y + proj * seg.y);
        const double2 dpv = pbc2(bx, tabs, pj);
        dpx = dpv.x;
        dpy = dpv.y;
      } else {
        dpx = fma(-proj, seg.x, tq.x);
        dpy = fma(-proj, seg.y, tq.y);
      }
      d2 = fma(dpy, dpy, dpx * dpx);
    }
    T gm, inv_d, ep = T(0);
    if (pair_eval_t<POT>(p, d2, rsum, inv_rsum, gm, inv_d, ep) && gm != T(0)) {
      if (on_seg) {
        const T cross = seg.x * w.y - w.x * seg.y;
        const T sign = sgn_nan0(cross);
        const T g = gm * inv_len;
        if constexpr (ROLE1) {
          ft.x += g * sign * (-seg.y);
          ft.y += g * sign * seg.x;
        } else {
          const T a = fabs(cross) * inv_lsq;
          fo.x += g * (sign * tq.y - a * seg.x);
          fo.y += g * (-sign * tq.x - a * seg.y);
          fq.x += g * (-sign * w.y + a * seg.x);
          fq.y += g * (sign * w.x + a * seg.y);
        }
      } else {
        // calcVertexVertexInteraction(thisPos, previousPos, ...): delta = t - q
        const T s2 = gm * inv_d;
        if constexpr (ROLE1) {
          ft.x += s2 * tq.x;
          ft.y += s2 * tq.y;
        } else {
          fq.x -= s2 * tq.x;
          fq.y -= s2 * tq.y;
        }
      }
      e += (double)ep;
    }
  }
  if (on_seg && pc >= -pl2 && pc < T(0)) {
    // calcVertexVertexInteraction(previousPos, thisPos, ...): delta = q - t,
    // the corner term taken away
    T g2, id2, ep2 = T(0);
    if (pair_eval_t<POT>(p, tq2, rsum, inv_rsum, g2, id2, ep2) && g2 != T(0)) {
      const T s2 = g2 * id2;
      if constexpr (ROLE1) {
        ft.x -= s2 * tq.x;
        ft.y -= s2 * tq.y;
      } else {
        fq.x += s2 * tq.x;
        fq.y += s2 * tq.y;
      }
      e -= (double)ep2;
    }
  }
}

// Exact skip test for a smooth unit: every term vanishes beyond R = range *
// radSum, the projection distance is at least max(|tq|, |w|) - |seg| and the
// corner terms use |tq|.  Evaluated in FP32 with a relative margin far above
// FP32 rounding, so a skipped unit is one that contributes exactly zero.
__device__ __forceinline__ bool smooth_out_of_range(float R, float tq2, float w2, float len) {
  const float Rm = R * 1.00001f;
  if (!(tq2 > Rm * Rm)) return false;
  const float lim = Rm + len * 1.00001f;
  return fmaxf(tq2, w2) > lim * lim;
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

// Compensated summation for the energy, kinetic-energy and power sums:
// TwoSum (Knuth, TAOCP vol. 2, 4.2.2) gives the exact rounding error of each
// addition, which is carried in c, so s + c holds the sum to about one
// rounding of the result whatever the number of terms and their
// cancellation (Neumaier 1974).
__device__ __forceinline__ void two_sum_add(double& s, double& c, double x) {
  const double t = s + x;
  const double bp = t - s;
  c += (s - (t - bp)) + (x - bp);
  s = t;
}

// Warp tree of a compensated pair; the total on lane 0.
__device__ __forceinline__ void warp_csum(double& s, double& c) {
  for (int o = 16; o > 0; o >>= 1) {
    const double ys = __shfl_xor_sync(0xffffffffu, s, o), yc = __shfl_xor_sync(0xffffffffu, c, o);
    two_sum_add(s, c, ys);
    c += yc;
  }
}

// Per-CTA partials of the NSUM quantities in a fixed order (every thread
// calls it with its own values): the additive ones summed with
// compensation, the largest force component and the non-finite flag by
// max.  s_red: shared [BLOCK / 32][NSUM]; out: this CTA's NSUM partials.
template <int BLOCK>
__device__ __forceinline__ void block_partials(const double (&v)[NSUM], double (*s_red)[NSUM], double* out) {
  const int warp = threadIdx.x / 32, wl = threadIdx.x % 32;
#pragma unroll
  for (int q = 0; q < NSUM; q++) {
    double s = v[q], c = 0.0;
    if (q == S_FMAX2 || q == S_NONFINITE) {
      for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    } else {
      warp_csum(s, c);
      s += c;
    }
    if (wl == 0) s_red[warp][q] = s;
  }
  __syncthreads();
  if (threadIdx.x < NSUM) {
    const int q = threadIdx.x;
    double s = 0.0, c = 0.0;
    for (int w = 0; w < BLOCK / 32; w++) {
      if (q == S_FMAX2 || q == S_NONFINITE) s = fmax(s, s_red[w][q]);
      else two_sum_add(s, c, s_red[w][q]);
    }
    out[q] = s + c;
  }
}

__device__ __forceinline__ void reduce_partials(const double* partials, int nblocks, double* out) {
  // one warp, fixed order: lane l sums blocks l, l+32, ... then a fixed tree,
  // the additive sums with compensation
  int lane = threadIdx.x;
  if (lane < 32) {
    double acc[NSUM], cmp[NSUM];
#pragma unroll
    for (int k = 0; k < NSUM; k++) acc[k] = cmp[k] = 0.0;
    for (int b = lane; b < nblocks; b += 32) {
#pragma unroll
      for (int k = 0; k < NSUM; k++) {
        const double x = __ldcg(partials + (size_t)b * NSUM + k);
        if (k == S_FMAX2 || k == S_NONFINITE) acc[k] = fmax(acc[k], x);
        else two_sum_add(acc[k], cmp[k], x);
      }
    }
#pragma unroll
    for (int k = 0; k < NSUM; k++) {
      if (k == S_FMAX2 || k == S_NONFINITE) {
        for (int o = 16; o > 0; o >>= 1) acc[k] = fmax(acc[k], __shfl_xor_sync(0xffffffffu, acc[k], o));
      } else {
        warp_csum(acc[k], cmp[k]);
        acc[k] += cmp[k];
      }
      if (lane == 0) out[k] = acc[k];
    }
  }
}

}  // namespace cr
