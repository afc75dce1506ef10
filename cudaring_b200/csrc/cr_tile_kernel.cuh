// Tiled force + integrator kernel body (see cr_tile.cuh for the phase
// structure), shared by the FP64 instantiations (cr_tile.cu) and the
// mixed-precision ones (cr_tile_mixed.cu).
//
// Latency layout.  A step of this workload is one wave of CTAs with a few
// warps per SM, so the time of a launch is the dependent-latency chain of one
// thread, not a throughput limit.  The kernel therefore keeps that chain
// short:
//   * every per-vertex input is fetched in the prologue, in parallel: the ring
//     topology from the packed vtopo word (no ring_of -> ring_first chain),
//     rest lengths / angles into shared memory (neighbours read them there),
//     and, for a step, velocity and last-build position by cp.async straight
//     into shared memory (no registers held across the pair phase);
//   * the neighbour gather reads each listed neighbour's ring predecessors
//     from the companion list (nbr_pq), so the neighbour's position and both
//     predecessor positions are loaded together, and the next slot's list
//     entries are fetched before the current slot is evaluated;
//   * per-CTA partial sums are formed only when an op needs them (FIRE); the
//     non-finite check otherwise is one __syncthreads_or.
#pragma once
#include <type_traits>

#include "cr_tile.cuh"

namespace cr {


// Occupancy target in threads per SM.  One lane per vertex: 512 leaves 128
// registers per thread, where the FP64 smooth-interaction body compiles
// without spills.  Two lanes per vertex (192-thread CTAs, tiles of up to 96
// vertices): 576 threads (three CTAs, 96 registers), so that the grid of a
// 39,424-vertex system (about 430 tiles) runs as one wave.  The mixed path
// takes the same budgets: it holds an FP64 unit body for its near-contact
// slots beside the FP32 one, and at 80 registers (four CTAs) its spills cost
// more than the fourth CTA gains (27.5 against 25.5 us per step measured at
// 39,424 vertices).
template <int PREC, int L = 1>
constexpr int tile_threads_per_sm() {
  return L >= 2 ? 576 : 512;
}

template <typename T2> __device__ __forceinline__ T2 cvt2(double2 d);
template <> __device__ __forceinline__ double2 cvt2<double2>(double2 d) { return d; }
template <> __device__ __forceinline__ float2 cvt2<float2>(double2 d) { return f2(d); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Box of the current tile: the system's parameters, or one system of a batch.
template <bool BATCH> struct BoxSel;
template <> struct BoxSel<false> {
  __device__ static const SysParams& get(const SysParams& p, const Box&) { return p; }
};
template <> struct BoxSel<true> {
  __device__ static const Box& get(const SysParams&, const Box& b) { return b; }
};

// Every CTA ends in the last-block protocol so that the op counter and the
// conditional rebuild node of a batch graph see each op exactly once.
__device__ __forceinline__ void tile_skip(const StepArgs& s, DevStatus* st) {
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      st->done_ctr = 0;
      if (s.use_cond) cudaGraphSetConditional(s.cond, st->rebuild ? 1u : 0u);
    }
  }
}

// BATCH: the grid covers the tiles of many independent systems; tile.x is
// the system, whose box, displacement cutoff, FIRE scalars and flags come
// from s.bsys, and whose last tile reduces the system's partial sums.
// Positions: the read-only path for a single-step launch; plain loads in the
// multi-step kernel, where other CTAs rewrite them between steps (the grid
// barrier's acquire makes their writes visible to plain loads, not to the
// non-coherent read-only path).
template <bool PERSIST>
__device__ __forceinline__ double2 ld_pos(const double2* p) {
  if constexpr (PERSIST) return *p;
  else return __ldg(p);
}

// ---------------------------------------------------------------------------
// Mixed-precision smooth units.
//
// Near contact the FP32 evaluation of a steep potential cannot meet a 1e-6
// force error: one rounding of the distance or of (radSum/d)^6 moves a unit
// force by ~1e-6 of the net force, which is a small residual of pair and
// shape forces several times larger.  So each list slot (vertex i against
// neighbour j: role 1, i against the segment prev(j) -> j; role 2, j against
// i's segment prev(i) -> i) first takes a near test in FP32: whether a live
// unit's vertex lies within f_near * radSum of its segment.  Far slots are
// evaluated in FP32 (every term of such a unit is at least that far away);
// near slots are evaluated afterwards exactly as the FP64 path evaluates
// them (same differences, same arithmetic, FP64 accumulators).  Each lane
// first walks its slots in FP32, deferring near ones to a bit mask, then
// runs the deferred ones in FP64: each loop carries one precision, and a
// vertex's force is the same whatever happened at earlier evaluations.
// ---------------------------------------------------------------------------

// Whether t lies within Rn of the segment q -> o (tq = t - q, w = t - o,
// seg = o - q, len2 = |seg|^2, squared lengths precomputed), without a
// division: an end point within Rn, or the foot of the perpendicular on the
// segment and |tq x seg|^2 < Rn^2 |seg|^2.
__device__ __forceinline__ bool seg_near(float2 tq, float tq2, float w2, float2 seg, float len2, float Rn2) {
  if (tq2 < Rn2 || w2 < Rn2) return true;
  const float dot = tq.x * seg.x + tq.y * seg.y;
  const float cr = tq.x * seg.y - tq.y * seg.x;
  return dot > 0.0f && dot < len2 && cr * cr < Rn2 * len2;
}

// FP32 body of one slot; returns true (and evaluates nothing) when the slot
// is near and belongs to the FP64 pass.  The slot's FP32 sums enter the FP64
// accumulators.  seg_i64 = x_i - x_q (q = prev(i)).
template <int POT, class B>
__device__ __forceinline__ bool mixed_slot_f32(const SysParams& p, const B& bx, double2 xi, double2 seg_i64,
                                               float2 seg_i, float2 pseg_i, float len2_i, float len_i, double ri,
                                               double rj, double2 xj, double2 xjq, double2 xjqq, double2& fi64,
                                               double2& fq64, double& ei) {
  const double rsum64 = ri + rj;
  const float rsum = (float)rsum64;
  const float R = pot_range_f<POT>(p) * rsum;
  const double2 w64 = pbc2(bx, xi, xj);    // x_i - x_j
  const double2 tq64 = pbc2(bx, xi, xjq);  // x_i - x_jq
  const float2 w1 = f2(w64), tq1 = f2(tq64);
  // x_j - x_jq as the difference of the two offsets from x_i: the same image
  // of ring j unless x_j and x_jq have their nearest images on different
  // sides (a box under about twice the interaction range); then directly
  double2 seg1_64 = make_double2(tq64.x - w64.x, tq64.y - w64.y);
  if (fabs(seg1_64.x) > 0.25 * bx.lx || fabs(seg1_64.y) > 0.25 * bx.ly) seg1_64 = pbc2(bx, xj, xjq);
  const float2 seg1 = f2(seg1_64);
  const float2 tq2 = f2(make_double2(seg_i64.x - w64.x, seg_i64.y - w64.y));  // x_j - x_q
  const float w2 = fmaf(w1.y, w1.y, w1.x * w1.x);
  const float tq1_2 = fmaf(tq1.y, tq1.y, tq1.x * tq1.x);
  const float len1 = fmaf(seg1.y, seg1.y, seg1.x * seg1.x);
  const float tq2_2 = fmaf(tq2.y, tq2.y, tq2.x * tq2.x);
  const bool in1 = !smooth_out_of_range(R, tq1_2, w2, sqrtf(len1));
  const bool in2 = !smooth_out_of_range(R, tq2_2, w2, len_i);
  if (!(in1 | in2)) return false;
  const float Rn = p.f_near * rsum, Rn2 = Rn * Rn;
  if ((in1 && seg_near(tq1, tq1_2, w2, seg1, len1, Rn2)) || (in2 && seg_near(tq2, tq2_2, w2, seg_i, len2_i, Rn2)))
    return true;
  const float inv_rsum = 1.0f / rsum;
  float2 fs{0.0f, 0.0f}, fqs{0.0f, 0.0f}, dummy{0.0f, 0.0f};
  if (in1) {
    const float2 pseg1 = f2(pbc2(bx, xjq, xjqq));  // x_jq - x_jqq
    smooth_core<POT, true, float>(p, bx, tq1, tq1_2, w1, seg1, len1, pseg1, rsum, inv_rsum, xi, xjq, fs, dummy, dummy,
                                  ei);
  }
  if (in2) {
    const float2 mw1{-w1.x, -w1.y};  // x_j - x_i
    smooth_core<POT, false, float>(p, bx, tq2, tq2_2, mw1, seg_i, len2_i, pseg_i, rsum, inv_rsum, xj, xj, dummy, fs,
                                   fqs, ei);  // (box coordinates are read by the FP64 body only)
  }
  fi64.x += (double)fs.x;
  fi64.y += (double)fs.y;
  fq64.x += (double)fqs.x;
  fq64.y += (double)fqs.y;
  return false;
}

// Single-precision test of one smooth unit (tq = t - q, seg = o - q, pseg =
// q - qq, Rm2 = (range * radSum)^2 with a margin): false only when the unit
// adds nothing.  A unit contributes only through its segment term (foot of
// the perpendicular inside the segment, a = tq . seg in [0, |seg|^2), its
// distance within range), its convex-corner term (a < 0 and tq . pseg >= 0,
// |tq| within range) or its concave-corner correction (inside the segment's
// span with |tq| within range, so within the first test).  The margins (1e-3
// of the scale of each dot product, 1e-4 |tq|^2 and 1% of the squared range)
// are far above the rounding of offsets formed in FP64 and rounded once.
__device__ __forceinline__ bool unit_may_contribute(float2 tq, float2 seg, float2 pseg, float Rm2) {
  const float t2 = fmaf(tq.y, tq.y, tq.x * tq.x);
  const float l2 = fmaf(seg.y, seg.y, seg.x * seg.x);
  const float a = fmaf(tq.y, seg.y, tq.x * seg.x);
  const float ma = 1e-3f * (t2 + l2);
  const float slack = fmaf(1e-4f, t2, Rm2);
  if (a >= -ma && a < l2 + ma && t2 * l2 - a * a < slack * l2) return true;
  if (a < ma && t2 < slack) {
    const float b = fmaf(tq.y, pseg.y, tq.x * pseg.x);
    const float pl2 = fmaf(pseg.y, pseg.y, pseg.x * pseg.x);
    if (b >= -1e-3f * (t2 + pl2)) return true;
  }
  return false;
}

// Whether either smooth unit of a slot (vertex i against neighbour j) may
// contribute: offsets formed in FP64 as the mixed path forms them, rounded
// once, then the single-precision unit test.  seg_i64 = x_i - x_q.
template <int POT, class B>
__device__ __forceinline__ bool slot_may_contribute(const SysParams& p, const B& bx, double2 xi, double2 seg_i64,
                                                    float2 seg_i, float2 pseg_i, double ri, double rj, double2 xj,
                                                    double2 xjq, double2 xjqq) {
  const float R = pot_range_f<POT>(p) * (float)(ri + rj);
  const float Rm2 = 1.01f * R * R;
  const double2 w64 = pbc2(bx, xi, xj);    // x_i - x_j
  const double2 tq64 = pbc2(bx, xi, xjq);  // x_i - x_jq
  double2 seg1_64 = make_double2(tq64.x - w64.x, tq64.y - w64.y);  // x_j - x_jq
  if (fabs(seg1_64.x) > 0.25 * bx.lx || fabs(seg1_64.y) > 0.25 * bx.ly) seg1_64 = pbc2(bx, xj, xjq);
  if (unit_may_contribute(f2(tq64), f2(seg1_64), f2(pbc2(bx, xjq, xjqq)), Rm2)) return true;
  const float2 tq2 = f2(make_double2(seg_i64.x - w64.x, seg_i64.y - w64.y));  // x_j - x_q
  return unit_may_contribute(tq2, seg_i, pseg_i, Rm2);
}

// FP64 body of one slot, shared by the FP64 path and the mixed path's
// near-contact slots: the reference's own differences of box coordinates
// (pbcDistance of each pair of vertices) and the FP64 skip tests.
// seg_i = x_i - x_q, pseg_i = x_q - x_qq: vertex i's segments (q = prev(i)).
template <int POT, class B>
__device__ __forceinline__ void smooth_slot_f64(const SysParams& p, const B& bx, double2 xi, double2 xq,
                                                double2 seg_i, double2 pseg_i, double len2_i, float len_i, double ri,
                                                double rj, double2 xj, double2 xjq, double2 xjqq, double2& fi,
                                                double2& fq, double& ei) {
  const double rsum = ri + rj;
  const double inv_rsum = 1.0 / rsum;
  const float R = pot_range_f<POT>(p) * (float)rsum;
  const double2 w1 = pbc2(bx, xi, xj);     // x_i - x_j
  const double2 tq1 = pbc2(bx, xi, xjq);   // x_i - x_jq
  const double2 seg1 = pbc2(bx, xj, xjq);  // x_j - x_jq
  const double2 tq2 = pbc2(bx, xj, xq);    // x_j - x_q
  const double w2 = fma(w1.y, w1.y, w1.x * w1.x);
  const double tq1_2 = fma(tq1.y, tq1.y, tq1.x * tq1.x);
  const double len1 = fma(seg1.y, seg1.y, seg1.x * seg1.x);
  const double tq2_2 = fma(tq2.y, tq2.y, tq2.x * tq2.x);
  double2 dummy{0.0, 0.0};
  if (!smooth_out_of_range(R, (float)tq1_2, (float)w2, sqrtf((float)len1))) {
    const double2 pseg1 = pbc2(bx, xjq, xjqq);  // x_jq - x_jqq
    smooth_core<POT, true, double>(p, bx, tq1, tq1_2, w1, seg1, len1, pseg1, rsum, inv_rsum, xi, xjq, fi, dummy,
                                   dummy, ei);
  }
  if (!smooth_out_of_range(R, (float)tq2_2, (float)w2, len_i)) {
    const double2 mw1{-w1.x, -w1.y};  // x_j - x_i
    smooth_core<POT, false, double>(p, bx, tq2, tq2_2, mw1, seg_i, len2_i, pseg_i, rsum, inv_rsum, xj, xq, dummy, fi,
                                    fq, ei);
  }
}

// One step (or force evaluation) of one tile.  pin / pout: positions read
// and written; step: the integrator step index (Philox stream of the noise).
// PERSIST: 0 for one op per launch; 1 the multi-step kernel: positions
// read with plain loads (other CTAs rewrite them between steps), a rebuild
// due or a non-finite force reported in *pflag instead of the status block,
// and the last-block protocol left to the caller; 2 the persistent batched
// FIRE kernel: plain position loads, everything else as for one op.
template <int POT, int INTER, int MODE, int BLOCK, int L, int PREC, bool BATCH, int PERSIST>
__device__ __forceinline__ void tile_body(const SysParams& p, const SysArrays& a, const StepArgs& s,
                                          const double2* __restrict__ pin, double2* __restrict__ pout,
                                          unsigned long long step, int* pflag, bool reuse = false) {
  constexpr int TV = BLOCK / L;
  // the multi-step kernel stores no energies and no sums (its ops run with
  // write_out = accumulate = 0), so its energy terms are left out at compile time
  constexpr bool kOut = PERSIST != 1;
  constexpr int TS = (MODE == MODE_STEP) ? TV : 1;
  __shared__ double2 s_pos[TV];
  __shared__ double2 s_seg[TV];     // pbc(pos[next] - pos[v])
  __shared__ double s_theta[TV];
  __shared__ double s_l0[TV];       // rest length of segment v -> next(v)
  __shared__ double s_il0[TV];      // its reciprocal
  __shared__ double s_th0[TV];      // rest angle at v
  __shared__ double s_r0[TV];       // shoelace terms -> ring area
  __shared__ double s_r1[TV];       // segment lengths -> perimeter
  __shared__ double2 s_r2[TV];      // offsets from the first vertex -> centroid
  __shared__ double2 s_fpair[TV];   // pair force on v
  __shared__ double2 s_fprev[TV];   // smooth: force on prev(v) gathered by v
  __shared__ double s_epair[TV];
  __shared__ double2 s_fsh[TV];     // shape force on v, parked across the pair phase
  __shared__ double s_esh[TV];      // shape energy booked on v
  __shared__ int s_lp[TV];
  __shared__ int2 s_tp[TV];         // topology word (ring, k | nv << 16)
  __shared__ double s_a0[TV];       // rest area of the vertex's ring
  __shared__ __align__(16) double2 s_vel[TS];
  __shared__ __align__(16) double2 s_last[TS];
  __shared__ double s_red[BLOCK / 32][NSUM];
  __shared__ Box s_box;
  __shared__ bool s_syslast;

  DevStatus* st = s.status;
  const int4 tile = a.tiles[blockIdx.x];
  const int v0 = tile.z, nvt = tile.w - tile.z;
  const int t = threadIdx.x;
  const int sysid = BATCH ? tile.x : 0;
  if constexpr (BATCH) {
    const BatchSys& bs = s.bsys[sysid];
    if (!bs.active || (MODE == MODE_STEP && bs.converged)) {
      if constexpr (MODE == MODE_STEP) tile_skip(s, st);
      return;
    }
    if (t == 0) s_box = bs.box;
  }
  const auto& bx = BoxSel<BATCH>::get(p, s_box);

  // ---- prologue: every per-vertex input, in parallel ------------------------
  int ring = -1, k = 0, lf = 0, lp = 0, ln = 0, nvr = 1;
  double a0r = 1.0;
  if (t < nvt) {
    const int v = v0 + t;
    int2 tp;
    if (PERSIST == 1 && reuse) {
      // a later step of the multi-step kernel: the CTA holds the same tile,
      // so its topology, rest lengths and angles, last-build positions and its
      // own positions and velocities (stored by the last step's tail) are
      // still in shared memory
      tp = s_tp[t];
      a0r = s_a0[t];
    } else {
      if constexpr (MODE == MODE_STEP) {
        cp_async16(&s_vel[t], s.vel + v);
        cp_async16(&s_last[t], s.last_pos + v);
        cp_async_commit();
      }
      tp = __ldg(a.vtopo + v);
      s_pos[t] = ld_pos<(PERSIST != 0)>(pin + v);
      const double l0v = __ldg(a.l0 + v);
      s_l0[t] = l0v;
      s_il0[t] = 1.0 / l0v;
      s_th0[t] = __ldg(a.theta0 + v);
      a0r = __ldg(a.a0 + tp.x);
      if constexpr (PERSIST == 1) {
        s_tp[t] = tp;
        s_a0[t] = a0r;
      }
    }
    ring = tp.x;
    k = tp.y & 0xffff;
    nvr = tp.y >> 16;
    lf = t - k;
    ln = lf + (k + 1 == nvr ? 0 : k + 1);
    lp = lf + (k == 0 ? nvr - 1 : k - 1);
    s_lp[t] = lp;
  }
  __syncthreads();

  // ---- phase 1: geometry --------------------------------------------------
  if (t < nvt) {
    const double2 x = s_pos[t];
    const double2 xn = s_pos[ln];
    const double2 seg = pbc2(bx, xn, x);
    s_seg[t] = seg;
    const double2 x0 = s_pos[lf];
    const double2 u = pbc2(bx, x, x0);
    const double2 un = pbc2(bx, xn, x0);
    s_r0[t] = u.x * un.y - un.x * u.y;
    s_r1[t] = dist_of(seg);
    s_r2[t] = u;
  }
  __syncthreads();
  if (t < nvt) {
    // calcAngle(nextSegment, previousSegment) (include/cudaKernel.cuh:423-427)
    const double2 ns = s_seg[t];
    const double2 ps = s_seg[lp];
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
    // The reference's divisions are taken as products with a few
    // reciprocals (1/A0, 1/l0 and the segments' 1/l from one rsqrt each),
    // a rounding-level difference
    const double area = fabs(s_r0[lf]) * 0.5;
    const double inv_a0 = 1.0 / a0r;
    const double dA = area * inv_a0 - 1.0;
    const double gmA = p.ea * dA * inv_a0;
    const double2 ns = s_seg[t];
    const double2 ps = s_seg[lp];
    // nRel - pRel = pos[next] - pos[prev]
    const double2 npd = make_double2(ns.x + ps.x, ns.y + ps.y);
    fsh.x += 0.5 * gmA * (-npd.y);
    fsh.y += 0.5 * gmA * (npd.x);
    esh += (0.5 * p.ea * dA * dA) / nvr;
    const double ps2 = fma(ps.y, ps.y, ps.x * ps.x), ns2 = fma(ns.y, ns.y, ns.x * ns.x);
    const double r_pl = rsqrt(ps2), r_nl = rsqrt(ns2);  // 1 / |segment|
    const double plen = ps2 * r_pl, nlen = ns2 * r_nl;
    const double tl0 = s_l0[t], pl0 = s_l0[lp];
    if (p.monomer == 0) {
      const double inv_tl0 = s_il0[t], inv_pl0 = s_il0[lp];
      const double pd = plen * inv_pl0 - 1.0;
      const double nd = nlen * inv_tl0 - 1.0;
      const double cn = nd * inv_tl0 * r_nl, cp = pd * inv_pl0 * r_pl;
      fsh.x += p.el * (cn * ns.x - cp * ps.x);
      fsh.y += p.el * (cn * ns.y - cp * ps.y);
      esh += 0.5 * p.el * pd * pd;
    } else {
      const double c = 2.0 * p.el * p.stiff * p.ext_sq;
      const double an = nlen / (p.ext_sq * tl0 * tl0 - nlen * nlen);
      const double ap = plen / (p.ext_sq * pl0 * pl0 - plen * plen);
      fsh.x += c * (an * ns.x / nlen - ap * ps.x / plen);
      fsh.y += c * (an * ns.y / nlen - ap * ps.y / plen);
      esh += p.el * p.stiff * p.ext_sq * log(1.0 - plen * plen / (p.ext_sq * pl0 * pl0));
    }
    const double prevAD = s_theta[lp] - s_th0[lp];
    const double thisAD = s_theta[t] - s_th0[t];
    const double nextAD = s_theta[ln] - s_th0[ln];
    const double pvar = (thisAD - prevAD) * (r_pl * r_pl);
    const double nvar = (thisAD - nextAD) * (r_nl * r_nl);
    fsh.x += p.eb * (pvar * ps.y + nvar * ns.y);
    fsh.y += p.eb * (pvar * (-ps.x) + nvar * (-ns.x));
    esh += 0.5 * p.eb * thisAD * thisAD;
    s_fsh[t] = fsh;
    s_esh[t] = esh;
  }

  // ---- phase 3: pair forces ------------------------------------------------
  // L lanes per vertex stride over its list slots; each slot's list entries
  // (neighbour id and packed predecessor offsets) are fetched two slots ahead
  // and the neighbour's three positions one slot ahead, all three together.
  {
    const int lv = t / L, lane = t % L;
    using T = typename std::conditional<PREC == PREC_MIXED, float, double>::type;
    typename Vec2<T>::type fi{0, 0}, fq{0, 0};
    double2 fi64{0.0, 0.0}, fq64{0.0, 0.0};  // mixed smooth path: FP64 accumulators
    double ei = 0.0;
    if (lv < nvt) {
      const int i = v0 + lv;
      const double2 xi = s_pos[lv];
      const double ri = __ldg(a.rad + i);
      const int cnt = min(__ldg(a.nbr_cnt + i), a.nbr_cap);  // an overflowed build stores counts above capacity
      const size_t stride = (size_t)p.nv;
      int sl = lane;
      int jn = 0, pkn = 0;
      if (sl < cnt) {
        jn = __ldg(a.nbr + (size_t)sl * stride + i);
        if constexpr (INTER == INT_SMOOTH) pkn = __ldg(a.nbr_pq + (size_t)sl * stride + i);
      }
      // two-stage pipeline: list entries two slots ahead, the neighbour's
      // positions one slot ahead of the slot being evaluated
      int j2 = 0, pk2 = 0;
      if (sl + L < cnt) {
        j2 = __ldg(a.nbr + (size_t)(sl + L) * stride + i);
        if constexpr (INTER == INT_SMOOTH) pk2 = __ldg(a.nbr_pq + (size_t)(sl + L) * stride + i);
      }
      if constexpr (INTER == INT_VV) {
        double2 nxj = make_double2(0.0, 0.0);
        double nr = 0.0;
        if (sl < cnt) {
          nxj = ld_pos<(PERSIST != 0)>(pin + jn);
          nr = __ldg(a.rad + jn);
        }
        while (sl < cnt) {
          const double2 xj = nxj;
          const double rj = nr;
          sl += L;
          if (sl < cnt) {
            nxj = ld_pos<(PERSIST != 0)>(pin + j2);
            nr = __ldg(a.rad + j2);
            if (sl + L < cnt) j2 = __ldg(a.nbr + (size_t)(sl + L) * stride + i);
          }
          if constexpr (PREC == PREC_MIXED) pair_own_f<POT>(p, f2(pbc2(bx, xi, xj)), (float)(ri + rj), fi, ei);
          else pair_own<POT>(p, pbc2(bx, xi, xj), ri + rj, fi, ei);
        }
      } else if constexpr (PREC == PREC_FP64) {
        // Smooth units of vertex i: role 1 (i against the segment prev(j) -> j)
        // and role 2 (j against i's own segment prev(i) -> i), in FP64.
        const int lq = s_lp[lv];
        const double2 xq = s_pos[lq];
        const double2 seg_i64 = s_seg[lq];         // x_i - x_q
        const double2 pseg_i64 = s_seg[s_lp[lq]];  // x_q - x_qq
        const double len2_i = fma(seg_i64.y, seg_i64.y, seg_i64.x * seg_i64.x);
        const float len_i = sqrtf((float)len2_i);
        const float2 seg_i = f2(seg_i64), pseg_i = f2(pseg_i64);
        // Most slots add nothing (the foot of the perpendicular past the
        // segment's end, where the next segment's unit takes over, or out of
        // range), and a warp issues every slot any of its lanes evaluates.  So
        // a single-precision pass marks the slots that may contribute (64 lane
        // slots at a time; a superset, see unit_may_contribute), and only the
        // marked ones are evaluated in FP64, in slot order: each vertex's sums
        // are those of evaluating every slot, as an unmarked slot adds nothing.
        for (int base = lane; base < cnt; base += 64 * L) {
          const int end = min(cnt, base + 64 * L);
          unsigned long long need = 0ull;
          int s0 = base;
          int j1 = 0, pk1 = 0;
          const int j0 = __ldg(a.nbr + (size_t)s0 * stride + i), pk0 = __ldg(a.nbr_pq + (size_t)s0 * stride + i);
          if (s0 + L < end) {
            j1 = __ldg(a.nbr + (size_t)(s0 + L) * stride + i);
            pk1 = __ldg(a.nbr_pq + (size_t)(s0 + L) * stride + i);
          }
          double2 xj = ld_pos<(PERSIST != 0)>(pin + j0), xjq = ld_pos<(PERSIST != 0)>(pin + j0 + pq_first(pk0)),
                  xjqq = ld_pos<(PERSIST != 0)>(pin + j0 + pq_second(pk0));
          double rj = __ldg(a.rad + j0);
          while (true) {
            const int s1 = s0 + L;
            int jn2 = 0, pkn2 = 0;
            double2 nxj = xj, nxjq = xjq, nxjqq = xjqq;
            double nr = rj;
            if (s1 < end) {
              if (s1 + L < end) {
                jn2 = __ldg(a.nbr + (size_t)(s1 + L) * stride + i);
                pkn2 = __ldg(a.nbr_pq + (size_t)(s1 + L) * stride + i);
              }
              nxj = ld_pos<(PERSIST != 0)>(pin + j1);
              nxjq = ld_pos<(PERSIST != 0)>(pin + j1 + pq_first(pk1));
              nxjqq = ld_pos<(PERSIST != 0)>(pin + j1 + pq_second(pk1));
              nr = __ldg(a.rad + j1);
            }
            if (slot_may_contribute<POT>(p, bx, xi, seg_i64, seg_i, pseg_i, ri, rj, xj, xjq, xjqq))
              need |= 1ull << ((s0 - base) / L);
            if (s1 >= end) break;
            s0 = s1;
            xj = nxj;
            xjq = nxjq;
            xjqq = nxjqq;
            rj = nr;
            j1 = jn2;
            pk1 = pkn2;
          }
          for (; need; need &= need - 1ull) {
            const int sm = base + (__ffsll((long long)need) - 1) * L;
            const int j = __ldg(a.nbr + (size_t)sm * stride + i), pk = __ldg(a.nbr_pq + (size_t)sm * stride + i);
            smooth_slot_f64<POT>(p, bx, xi, xq, seg_i64, pseg_i64, len2_i, len_i, ri, __ldg(a.rad + j),
                                 ld_pos<(PERSIST != 0)>(pin + j), ld_pos<(PERSIST != 0)>(pin + j + pq_first(pk)),
                                 ld_pos<(PERSIST != 0)>(pin + j + pq_second(pk)), fi, fq, ei);
          }
        }
      } else {
        // Smooth units, mixed precision: the lane's slots in FP32, near ones
        // deferred (64 lane slots at a time), then the deferred ones in FP64
        const int lq = s_lp[lv], lqq = s_lp[lq];
        const double2 seg_i64 = s_seg[lq];  // x_i - x_q
        const float2 seg_i = f2(seg_i64), pseg_i = f2(s_seg[lqq]);  // x_q - x_qq
        const float len2_i = fmaf(seg_i.y, seg_i.y, seg_i.x * seg_i.x);
        const float len_i = sqrtf(len2_i);
        for (int base = lane; base < cnt; base += 64 * L) {
          const int end = min(cnt, base + 64 * L);
          unsigned long long late = 0ull;
          int s0 = base;
          int j1 = 0, pk1 = 0;
          const int j0 = __ldg(a.nbr + (size_t)s0 * stride + i), pk0 = __ldg(a.nbr_pq + (size_t)s0 * stride + i);
          if (s0 + L < end) {
            j1 = __ldg(a.nbr + (size_t)(s0 + L) * stride + i);
            pk1 = __ldg(a.nbr_pq + (size_t)(s0 + L) * stride + i);
          }
          double2 xj = ld_pos<(PERSIST != 0)>(pin + j0), xjq = ld_pos<(PERSIST != 0)>(pin + j0 + pq_first(pk0)),
                  xjqq = ld_pos<(PERSIST != 0)>(pin + j0 + pq_second(pk0));
          double rj = __ldg(a.rad + j0);
          while (true) {
            const int s1 = s0 + L;
            int j2 = 0, pk2 = 0;
            double2 nxj = xj, nxjq = xjq, nxjqq = xjqq;
            double nr = rj;
            if (s1 < end) {
              if (s1 + L < end) {
                j2 = __ldg(a.nbr + (size_t)(s1 + L) * stride + i);
                pk2 = __ldg(a.nbr_pq + (size_t)(s1 + L) * stride + i);
              }
              nxj = ld_pos<(PERSIST != 0)>(pin + j1);
              nxjq = ld_pos<(PERSIST != 0)>(pin + j1 + pq_first(pk1));
              nxjqq = ld_pos<(PERSIST != 0)>(pin + j1 + pq_second(pk1));
              nr = __ldg(a.rad + j1);
            }
            if (mixed_slot_f32<POT>(p, bx, xi, seg_i64, seg_i, pseg_i, len2_i, len_i, ri, rj, xj, xjq, xjqq, fi64,
                                    fq64, ei))
              late |= 1ull << ((s0 - base) / L);
            if (s1 >= end) break;
            s0 = s1;
            xj = nxj;
            xjq = nxjq;
            xjqq = nxjqq;
            rj = nr;
            j1 = j2;
            pk1 = pk2;
          }
          if (late) {
            const double2 xq = s_pos[lq], pseg_i64 = s_seg[lqq];
            const double len2_i64 = fma(seg_i64.y, seg_i64.y, seg_i64.x * seg_i64.x);
            const float len_i64 = sqrtf((float)len2_i64);
            for (; late; late &= late - 1ull) {
              const int s = base + (__ffsll((long long)late) - 1) * L;
              const int j = __ldg(a.nbr + (size_t)s * stride + i), pk = __ldg(a.nbr_pq + (size_t)s * stride + i);
              smooth_slot_f64<POT>(p, bx, xi, xq, seg_i64, pseg_i64, len2_i64, len_i64, ri, __ldg(a.rad + j),
                                   ld_pos<(PERSIST != 0)>(pin + j), ld_pos<(PERSIST != 0)>(pin + j + pq_first(pk)),
                                   ld_pos<(PERSIST != 0)>(pin + j + pq_second(pk)), fi64, fq64, ei);
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
      if constexpr (INTER == INT_SMOOTH && PREC == PREC_MIXED) {
        fi64.x += __shfl_xor_sync(0xffffffffu, fi64.x, o);
        fi64.y += __shfl_xor_sync(0xffffffffu, fi64.y, o);
        fq64.x += __shfl_xor_sync(0xffffffffu, fq64.x, o);
        fq64.y += __shfl_xor_sync(0xffffffffu, fq64.y, o);
      }
    }
    if (lane == 0 && lv < nvt) {
      if constexpr (INTER == INT_SMOOTH && PREC == PREC_MIXED) {
        s_fpair[lv] = fi64;
        s_fprev[lv] = fq64;
      } else {
        s_fpair[lv] = make_double2(fi.x, fi.y);
        s_fprev[lv] = make_double2(fq.x, fq.y);
      }
      s_epair[lv] = ei;
    }
  }
  __syncthreads();

  // ---- phase 4: totals and outputs ----------------------------------------
  double2 F = make_double2(0.0, 0.0);
  double evtx = 0.0;  // per-vertex energy as the reference stores it
  double epair = 0.0;
  if (t < nvt) {
    // ring topology again (an L1 hit) rather than registers held across phase 3
    const int2 tp = __ldg(a.vtopo + v0 + t);
    ring = tp.x;
    k = tp.y & 0xffff;
    nvr = tp.y >> 16;
    lf = t - k;
    ln = lf + (k + 1 == nvr ? 0 : k + 1);
    const double2 fp = s_fpair[t];
    const double2 fsh = s_fsh[t];
    const double esh = s_esh[t];
    F.x = fsh.x + fp.x;
    F.y = fsh.y + fp.y;
    if constexpr (INTER == INT_SMOOTH) {
      const double2 fn = s_fprev[ln];
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
    int nonfinite = 0;
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
      cp_async_wait_all();  // this thread's own copies of vel and last_pos
      double2 vh = s_vel[t];
      const double2 xl = s_last[t];
      const double2 x = s_pos[t];
      double2 vn;
      double hdt = s.hdt;
      if (s.kind == KIND_FIRE) {
        if constexpr (BATCH) hdt = 0.5 * s.bfire_state[(sysid * 2 + ((s.bsys[sysid].fire_iters + 1) & 1)) * 4];
        else hdt = 0.5 * s.fire_state[((st->fire_iters + 1) & 1) * 4];
      }
      const double dcut = BATCH ? s.bsys[sysid].disp_cutoff : s.disp_cutoff;
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
        pout[v] = xn;
        s.vel[v] = vn;
        s.force[v] = F;
        if (kOut && s.write_out) s.energy[v] = evtx;
        if (3.0 * dist_of(pbc2(bx, xn, xl)) > dcut) {
          st->rebuild = 1;
          if constexpr (PERSIST == 1) atomicOr(pflag, 1);
          if constexpr (BATCH) s.bsys[sysid].rebuild = 1;
        }
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
          pout[v] = xn;
          s.vel[v] = vh2;
          if constexpr (PERSIST == 1) {
            // kept for the next step of the multi-step kernel (this thread
            // alone reads its slots until the barrier between steps)
            s_pos[t] = xn;
            s_vel[t] = vh2;
          }
          if (3.0 * dist_of(pbc2(bx, xn, xl)) > dcut) {
            st->rebuild = 1;
            if constexpr (PERSIST == 1) atomicOr(pflag, 1);
            if constexpr (BATCH) s.bsys[sysid].rebuild = 1;
          }
        } else {
          s.vel[v] = vn;
          s.force[v] = F;
          if (kOut && s.write_out) s.energy[v] = evtx;
        }
      }
      if (kOut && s.accumulate) {
        // products and sums rounded as written, so every kernel built on
        // this body (one op per launch, multi-step, persistent FIRE) sums alike
        sums[S_PE] = evtx + ((INTER == INT_SMOOTH) ? epair : 0.0);
        sums[S_VV] = __fma_rn(vn.y, vn.y, __dmul_rn(vn.x, vn.x));
        sums[S_VF] = __fma_rn(vn.y, F.y, __dmul_rn(vn.x, F.x));
        sums[S_FF] = __fma_rn(F.y, F.y, __dmul_rn(F.x, F.x));
        sums[S_FMAX2] = fmax(__dmul_rn(F.x, F.x), __dmul_rn(F.y, F.y));
      }
      if (!(isfinite(F.x) && isfinite(F.y))) {
        sums[S_NONFINITE] = 1.0;
        nonfinite = 1;
      }
    }
    if (kOut && s.write_out && INTER == INT_SMOOTH) {
      __syncthreads();
      if (t < nvt) s_r1[t] = epair;
      for (int stride = 1; stride < TV; stride <<= 1) {
        __syncthreads();
        if (t < nvt && (k % (2 * stride)) == 0 && k + stride < nvr) s_r1[t] += s_r1[t + stride];
      }
      __syncthreads();
      if (t < nvt && k == 0) s.p_energy[ring] = s_r1[t];
    }
    if (kOut && s.accumulate) {
      // per-CTA partials in a fixed order, compensated
      block_partials<BLOCK>(sums, s_red, s.partials + (size_t)blockIdx.x * NSUM);
    } else if (__syncthreads_or(nonfinite) && t == 0) {
      if constexpr (PERSIST == 1) {
        atomicOr(pflag, 2);
      } else {
        st->nonfinite = 1;
        st->abort = 1;
      }
    }
    if constexpr (PERSIST == 1) return;
    if constexpr (BATCH) {
      if (kOut && s.accumulate) {
        // the system's last tile reduces the system's partials
        BatchSys& bs = s.bsys[sysid];
        __syncthreads();
        if (t == 0) {
          __threadfence();
          const unsigned int prev = atomicAdd(&bs.done_ctr, 1u);
          s_syslast = (prev == (unsigned int)(bs.tile_end - bs.tile_begin - 1));
        }
        __syncthreads();
        if (s_syslast) {
          reduce_partials(s.partials + (size_t)bs.tile_begin * NSUM, bs.tile_end - bs.tile_begin, bs.sums);
          __syncthreads();
          if (t == 0) {
            __threadfence();
            if (bs.sums[S_NONFINITE] != 0.0) {
              st->nonfinite = 1;
              st->abort = 1;
            }
            if (s.kind == KIND_FIRE) {
              bs.fire_iters += 1;
              if (bs.fire_tol >= 0.0 && bs.sums[S_FMAX2] <= bs.fire_tol * bs.fire_tol) bs.converged = 1;
            }
            bs.done_ctr = 0;
          }
        }
      }
    }
    if (is_last_block(st)) {
      if (!BATCH && kOut && s.accumulate) reduce_partials(s.partials, gridDim.x, st->sums);
      __syncthreads();
      if (t == 0) {
        __threadfence();
        if (!BATCH && kOut && s.accumulate && st->sums[S_NONFINITE] != 0.0) {
          st->nonfinite = 1;
          st->abort = 1;
        }
        if (!BATCH && s.kind == KIND_FIRE) {
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

template <int POT, int INTER, int MODE, int BLOCK, int L, int PREC, bool BATCH = false>
__global__ void __launch_bounds__(BLOCK, tile_threads_per_sm<PREC, L>() / BLOCK) k_tile(const __grid_constant__ SysParams p,
                                                const __grid_constant__ SysArrays a,
                                                const __grid_constant__ StepArgs s) {
  // every input may come from the kernel before this one (positions, lists,
  // status); the next kernel (the rebuild check) may be scheduled at once and
  // waits for this one's completion itself
  pdl_wait();
  pdl_trigger();
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
  tile_body<POT, INTER, MODE, BLOCK, L, PREC, BATCH, 0>(p, a, s, a.pos, s.pos_out,
                                                           (unsigned long long)st->rng_step, nullptr);
}

// ---------------------------------------------------------------------------
// Multi-step kernel: up to s.persist_max middle steps of an NVE / Langevin /
// BAOAB sequence in one launch, with a grid barrier between steps in place
// of a kernel boundary.  Every tile is one resident CTA (the host launches it
// only when occupancy x SMs holds the grid).  Positions ping-pong between
// pos0 (read by step 0) and pos1; a launch that ends after an odd number of
// steps copies its tiles' positions back, so the result is always in pos0.
// The launch stops after the first step whose displacement check fired (the
// one-launch build that follows it rebuilds the list) or that met a
// non-finite force.
//
// Those stop decisions must be the same in every CTA, so they travel in three
// flag words used in rotation: step j writes slot (base + j) % 3, every CTA
// reads it after barrier j, and CTA 0 clears slot (base + j + 1) % 3 during
// step j (its last reader passed barrier j - 1, its next writer waits for
// barrier j).  base advances by the steps run, so every launch starts on a
// clean slot.  The step counters (rng_step, ops_done, steps_left, base) are
// read by every CTA before barrier 0 and updated by CTA 0 after the loop.
// Every barrier wait is bounded: a CTA that gives up sets stalled and abort
// and leaves; the others see stalled and leave too.

__device__ __forceinline__ unsigned long long pst_ld_acquire(const unsigned long long* a) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long pst_atom_add_release(unsigned long long* a, unsigned long long x) {
  unsigned long long old;
  asm volatile("atom.add.release.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(a), "l"(x) : "memory");
  return old;
}

// Barrier over the grid on status.pbar (a multiple of gridDim.x at launch; a
// 64-bit count, so a sequence of any length never wraps it).
__device__ __forceinline__ bool steps_barrier(DevStatus* st) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned long long g = gridDim.x;
    const unsigned long long prev = pst_atom_add_release(&st->pbar, 1ull);
    const unsigned long long target = (prev / g + 1ull) * g;
    const long long lim = barrier_poll_limit(st);
    long long it = 0;
    while (pst_ld_acquire(&st->pbar) < target) {
      if (++it > lim || *(volatile int*)&st->stalled) {
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    if (!ok) {
      atomicExch(&st->stalled, 1);
      atomicExch(&st->abort, 1);
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int POT, int INTER, int BLOCK, int L, int PREC>
__global__ void __launch_bounds__(BLOCK, tile_threads_per_sm<PREC, L>() / BLOCK)
    k_tile_steps(const __grid_constant__ SysParams p, const __grid_constant__ SysArrays a,
                 const __grid_constant__ StepArgs s) {
  pdl_wait();
  pdl_trigger();
  DevStatus* st = s.status;
  const volatile DevStatus* vs = st;
  __shared__ int s_flag;
  if (vs->abort | vs->converged) return;
  const long long left = vs->steps_left;
  const int n = (int)(left < (long long)s.persist_max ? left : (long long)s.persist_max);
  const unsigned long long step0 = (unsigned long long)vs->rng_step;
  const long long base = vs->pbase;
  double2* pos0 = const_cast<double2*>(a.pos);
  double2* pos1 = s.pos_out;
  int done = 0;
  bool stalled = false;
  for (int j = 0; j < n; j++) {
    int* slot = &st->pflag[(base + j) % 3];
    if (blockIdx.x == 0 && threadIdx.x == 0) st->pflag[(base + j + 1) % 3] = 0;
    const double2* pin = (j & 1) ? pos1 : pos0;
    double2* pout = (j & 1) ? pos0 : pos1;
    tile_body<POT, INTER, MODE_STEP, BLOCK, L, PREC, false, 1>(p, a, s, pin, pout, step0 + (unsigned long long)j,
                                                                 slot, j > 0);
    done = j + 1;
    if (!steps_barrier(st)) {
      stalled = true;
      break;
    }
    if (threadIdx.x == 0) s_flag = *(volatile int*)slot;
    __syncthreads();
    const int f = s_flag;
    __syncthreads();
    if (f) break;
  }
  if (stalled) return;
  if (done & 1) {
    // the last step wrote pos1: this tile's vertices back to pos0 (every read
    // of pos0 by the last step finished before the last barrier)
    const int4 tile = a.tiles[blockIdx.x];
    for (int v = tile.z + threadIdx.x; v < tile.w; v += BLOCK) pos0[v] = pos1[v];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && done > 0) {
    const int f = *(volatile int*)&st->pflag[(base + done - 1) % 3];
    if (f & 2) {
      st->nonfinite = 1;
      st->abort = 1;
    }
    st->rng_step += done;
    st->ops_done += done;
    st->steps_left -= done;
    st->pbase = base + done;
  }
}

}  // namespace cr
