// Forces and energies in hyper-dual arithmetic: the derivative kernel behind
// the Hessian-vector product, the virial pressure and the parameter
// derivatives (cr_hvp, cr_calc_pressure, cr_param_derivatives).
//
// One thread per vertex evaluates the same per-vertex force and energy as the
// fused kernel (shape terms of kernelCalcShapeForceEnergy,
// include/cudaKernel.cuh:474-529, with harmonic or FENE monomers, and the pair
// terms: vertex-vertex, kernelCalcVertexInteraction :690-722, or smooth
// vertex-segment, kernelCalcSmoothInteraction :922-975, in the gather form of
// the fused kernel) with every input a hyper-dual number: positions x + t1 e1 + t2 e2, box L (1 + s1 e1 + s2 e2),
// and the shape constants and rest lengths / radii along parameter tangents.
// The e1 part of the force is then D_t1 F = -H t1 (the Hessian-vector
// product), the e1 part of the energy along the affine dilation t1 = x,
// s1 = 1 is dU/dlambda = -2 A P, and the e1 e2 parts give the mixed
// derivatives that the adjoint gradients need.  The rings' areas are summed
// once per ring by a first kernel.  These kernels serve small systems and
// iterative solves, not the time-stepping hot path.
#include <algorithm>

#include "cr_hd.cuh"
#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {
namespace {

struct HBox {
  HD lx, ly;
};

__device__ __forceinline__ HD pbc_hd(HD d, const HD& L) {
  const double k = round(d.a / L.a);
  return d - k * L;
}

__device__ __forceinline__ HD2 pbc2_hd(const HD2& a, const HD2& b, const HBox& bx) {
  return HD2{pbc_hd(a.x - b.x, bx.lx), pbc_hd(a.y - b.y, bx.ly)};
}

__device__ __forceinline__ HD2 load_x(const DiffArgs& g, int i) {
  const double2 x = g.pos[i];
  double2 u1 = make_double2(0.0, 0.0), u2 = make_double2(0.0, 0.0);
  if (g.t1) u1 = g.t1[i];
  if (g.t2) u2 = g.t2[i];
  return HD2{HD{x.x, u1.x, u2.x, 0.0}, HD{x.y, u1.y, u2.y, 0.0}};
}

// l0 and rad scale as sqrt(calA0) (the reference's conventions: l0 from the
// preferred perimeter, rad = l0 / 2); along ln(calA0) a length w takes
// w (1 + c1/2 e1 + c2/2 e2 - c1 c2 / 4 e1 e2).
__device__ __forceinline__ HD scaled_length(const DiffArgs& g, double w) {
  return HD{w, 0.5 * g.c1 * w, 0.5 * g.c2 * w, -0.25 * g.c1 * g.c2 * w};
}

template <int POT>
__device__ __forceinline__ bool pair_hd(const DiffArgs& g, HD d, HD rsum, HD& gm, HD& ep) {
  const SysParams& p = g.p;
  const double ec = p.ec;
  if constexpr (POT == POT_HARMONIC) {
    const HD ov = 1.0 - d / rsum;
    if (!(ov.a > 0.0)) return false;
    gm = ec * ov / rsum;
    ep = (0.25 * ec) * ov * ov;
    return true;
  } else if constexpr (POT == POT_LJ) {
    if (!(d.a <= p.lj_cutoff * rsum.a)) return false;
    const HD ratio = rsum / d;
    const HD r2 = ratio * ratio;
    const HD r6 = r2 * r2 * r2;
    const HD r12 = r6 * r6;
    const HD fshift = p.lj_fshift / rsum;
    gm = (24.0 * ec) * (2.0 * r12 - r6) / d - fshift;
    ep = 0.5 * ((4.0 * ec) * (r12 - r6) - p.lj_ecut - habs(fshift) * (d - p.lj_cutoff * rsum));
    return true;
  } else if constexpr (POT == POT_ADHESIVE) {
    if (!(d.a < (1.0 + p.l2) * rsum.a)) return false;
    const HD ov = 1.0 - d / rsum;
    if (d.a < (1.0 + p.l1) * rsum.a) {
      gm = ec * ov / rsum;
      ep = (0.25 * ec) * (ov * ov - p.l1 * p.l2);
    } else {
      const double k = ec * p.l1 / (p.l2 - p.l1);
      gm = -k * (ov + p.l2) / rsum;
      ep = (-0.25 * k) * (ov + p.l2) * (ov + p.l2);
    }
    return true;
  } else {
    if (!(d.a <= kWCAcut * rsum.a)) return false;
    const HD ratio = rsum / d;
    const HD r2 = ratio * ratio;
    const HD r6 = r2 * r2 * r2;
    const HD r12 = r6 * r6;
    gm = (24.0 * ec) * (2.0 * r12 - r6) / d;
    ep = (0.5 * ec) * (4.0 * (r12 - r6) + 1.0);
    return true;
  }
}

__device__ __forceinline__ HD cross(const HD2& a, const HD2& b) { return a.x * b.y - b.x * a.y; }
__device__ __forceinline__ HD dot(const HD2& a, const HD2& b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ HD norm(const HD2& a) { return hsqrt(dot(a, a)); }
// calcAngle(nextSegment, previousSegment) (include/cudaKernel.cuh:423-427)
__device__ __forceinline__ HD angle(const HD2& ns, const HD2& ps) { return hatan2(cross(ns, ps), dot(ns, ps)); }

// One smooth unit (calcGradMultipleAndEnergy / calcVertexSegmentInteraction /
// calcVertexVertexInteraction, include/cudaKernel.cuh:806-912): vertex t
// against the segment q -> o, with tq = t - q, w = t - o, seg = o - q and
// pseg = q - qq.  WHO = 1 adds the force on t, 2 the force on o, 3 the force
// on q; the unit energy is booked for WHO 1 and 2 (each unit is evaluated
// once in each role, as the fused kernel gathers it).  The branches are taken
// on the real parts.
template <int POT, int WHO>
__device__ void smooth_hd(const DiffArgs& g, const HD2& tq, const HD2& w, const HD2& seg, const HD2& pseg,
                          const HD& rsum, HD2& f, HD& e) {
  const HD len2 = dot(seg, seg);
  const HD inv_len = 1.0 / hsqrt(len2);
  const HD inv_lsq = inv_len * inv_len;
  const HD proj = dot(tq, seg) * inv_lsq;
  const HD pc = dot(tq, pseg);
  const HD pl2 = dot(pseg, pseg);
  auto corner = [&](double sgn) {  // sgn +1: convex (added), -1: concave (removed)
    const HD d2 = norm(tq);
    HD g2, ep2;
    if (pair_hd<POT>(g, d2, rsum, g2, ep2) && g2.a != 0.0) {
      const HD s2 = g2 / d2;
      if (WHO == 1) {
        f.x += sgn * (s2 * tq.x);
        f.y += sgn * (s2 * tq.y);
      } else if (WHO == 3) {
        f.x -= sgn * (s2 * tq.x);
        f.y -= sgn * (s2 * tq.y);
      }
      if (WHO != 3) e += sgn * ep2;
    }
  };
  if (proj.a >= 0.0 && proj.a < 1.0) {
    const HD2 dp{tq.x - proj * seg.x, tq.y - proj * seg.y};
    const HD d = norm(dp);
    HD gm, ep;
    if (pair_hd<POT>(g, d, rsum, gm, ep) && gm.a != 0.0) {
      const HD cr = seg.x * w.y - w.x * seg.y;
      const double sign = cr.a > 0.0 ? 1.0 : (cr.a < 0.0 ? -1.0 : __longlong_as_double(0x7ff8000000000000LL));
      const HD gg = gm * inv_len;
      if (WHO == 1) {
        f.x += gg * (sign * (-1.0) * seg.y);
        f.y += gg * (sign * seg.x);
      } else {
        const HD a = habs(cr) * inv_lsq;
        if (WHO == 2) {
          f.x += gg * (sign * tq.y - a * seg.x);
          f.y += gg * ((-sign) * tq.x - a * seg.y);
        } else {
          f.x += gg * ((-sign) * w.y + a * seg.x);
          f.y += gg * (sign * w.x + a * seg.y);
        }
      }
      if (WHO != 3) e += ep;
    }
    if (pc.a >= -pl2.a && pc.a < 0.0) corner(-1.0);
  } else if (proj.a < 0.0 && pc.a >= 0.0) {
    corner(1.0);
  }
}

// ring predecessor of vertex j from its topology
__device__ __forceinline__ int prev_of(const DiffArgs& g, int j, int back) {
  const int2 tp = g.vtopo[j];
  const int k = tp.y & 0xffff, n = tp.y >> 16;
  return j - k + (k - back + 2 * n) % n;
}

// ring area by the shoelace sum of offsets from the ring's first vertex, one
// thread per ring
__global__ void __launch_bounds__(64) k_ring_area_hd(const __grid_constant__ DiffArgs g, const int* ring_first,
                                                     const int* ring_nv) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.p.np || (g.skip && *g.skip)) return;
  const SysParams& p = g.p;
  const HBox bx{HD{p.lx, p.lx * g.s1, p.lx * g.s2, 0.0}, HD{p.ly, p.ly * g.s1, p.ly * g.s2, 0.0}};
  const int f = ring_first[q], nvr = ring_nv[q];
  const HD2 x0 = load_x(g, f);
  HD sum = hd(0.0);
  HD2 u = HD2{hd(0.0), hd(0.0)};
  for (int k = 0; k < nvr; k++) {
    const HD2 un = pbc2_hd(load_x(g, f + (k + 1) % nvr), x0, bx);
    sum += cross(u, un);
    u = un;
  }
  const HD area = 0.5 * habs(sum);
  double* o = g.ring_area + (size_t)4 * q;
  o[0] = area.a;
  o[1] = g.diag ? (sum.a >= 0.0 ? 1.0 : -1.0) : area.b;  // diag mode: the ring's orientation
  o[2] = area.c;
  o[3] = area.d;
}

template <int POT, int INTER>
__global__ void __launch_bounds__(64) k_diff(const __grid_constant__ DiffArgs g) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= g.p.nv || (g.skip && *g.skip)) return;
  const SysParams& p = g.p;
  const HBox bx{HD{p.lx, p.lx * g.s1, p.lx * g.s2, 0.0}, HD{p.ly, p.ly * g.s1, p.ly * g.s2, 0.0}};
  const HD ea{p.ea, g.pe1[0], g.pe2[0], 0.0}, el{p.el, g.pe1[1], g.pe2[1], 0.0}, eb{p.eb, g.pe1[2], g.pe2[2], 0.0};
  const int2 tp = g.vtopo[v];
  const int ring = tp.x, k = tp.y & 0xffff, nvr = tp.y >> 16;
  const int f = v - k;
  auto at = [&](int kk) { return f + ((kk % nvr) + nvr) % nvr; };
  const int vp = at(k - 1), vn = at(k + 1), vpp = at(k - 2), vnn = at(k + 2);

  const double* ra = g.ring_area + (size_t)4 * ring;
  HD2 x = load_x(g, v);
  const HD2 xn = load_x(g, vn), xp = load_x(g, vp);
  if (g.diag) x = HD2{HD{x.x.a, 1.0, 0.0, 0.0}, HD{x.y.a, 0.0, 1.0, 0.0}};
  const HD2 ns = pbc2_hd(xn, x, bx), ps = pbc2_hd(x, xp, bx);
  // ring area; with the own-vertex seeding its tangents are the shoelace
  // derivatives dA/dx_v = s (y_next - y_prev) / 2, dA/dy_v = s (x_prev - x_next) / 2
  // (s the ring's orientation), second derivative zero
  const HD area = g.diag ? HD{ra[0], 0.5 * ra[1] * (ns.y.a + ps.y.a), -0.5 * ra[1] * (ns.x.a + ps.x.a), 0.0}
                         : HD{ra[0], ra[1], ra[2], ra[3]};
  const HD2 pps = pbc2_hd(xp, load_x(g, vpp), bx), nns = pbc2_hd(load_x(g, vnn), xn, bx);
  const HD th = angle(ns, ps), thp = angle(ps, pps), thn = angle(nns, ns);

  HD2 F{hd(0.0), hd(0.0)};
  HD E = hd(0.0);
  // area
  const double a0 = g.a0[ring];
  const HD dA = area / a0 - 1.0;
  const HD gmA = ea * dA / a0;
  const HD2 npd{ns.x + ps.x, ns.y + ps.y};
  F.x += 0.5 * gmA * (-npd.y);
  F.y += 0.5 * gmA * npd.x;
  E += (0.5 * ea * dA * dA) / (double)nvr;
  // segment lengths: harmonic or FENE monomers (include/cudaKernel.cuh:442-471)
  const HD plen = norm(ps), nlen = norm(ns);
  const HD tl0 = scaled_length(g, g.l0[v]), pl0 = scaled_length(g, g.l0[vp]);
  if (p.monomer == 0) {
    const HD pd = plen / pl0 - 1.0, nd = nlen / tl0 - 1.0;
    F.x += el * (nd * ns.x / (tl0 * nlen) - pd * ps.x / (pl0 * plen));
    F.y += el * (nd * ns.y / (tl0 * nlen) - pd * ps.y / (pl0 * plen));
    E += 0.5 * el * pd * pd;
  } else {
    const HD c = (2.0 * p.stiff * p.ext_sq) * el;
    const HD an = nlen / (p.ext_sq * tl0 * tl0 - nlen * nlen);
    const HD ap = plen / (p.ext_sq * pl0 * pl0 - plen * plen);
    F.x += c * (an * ns.x / nlen - ap * ps.x / plen);
    F.y += c * (an * ns.y / nlen - ap * ps.y / plen);
    E += (p.stiff * p.ext_sq) * el * hlog(1.0 - plen * plen / (p.ext_sq * pl0 * pl0));
  }
  // bending
  const HD prevAD = thp - g.theta0[vp], thisAD = th - g.theta0[v], nextAD = thn - g.theta0[vn];
  const HD pvar = (thisAD - prevAD) / dot(ps, ps);
  const HD nvar = (thisAD - nextAD) / dot(ns, ns);
  F.x += eb * (pvar * ps.y + nvar * ns.y);
  F.y += eb * (pvar * (-ps.x) + nvar * (-ns.x));
  E += 0.5 * eb * thisAD * thisAD;

  const HD ri = scaled_length(g, g.rad[v]);
  const int cnt = min(g.nbr_cnt[v], g.nbr_cap);
  if constexpr (INTER == INT_VV) {
    // vertex-vertex pairs
    for (int s = 0; s < cnt; s++) {
      const int j = g.nbr[(size_t)s * p.nv + v];
      const HD2 dl = pbc2_hd(x, load_x(g, j), bx);
      const HD d = norm(dl);
      const HD rsum = ri + scaled_length(g, g.rad[j]);
      HD gm, ep;
      if (pair_hd<POT>(g, d, rsum, gm, ep)) {
        const HD s2 = gm / d;
        F.x += s2 * dl.x;
        F.y += s2 * dl.y;
        E += ep;
      }
    }
  } else {
    // smooth units gathered as the fused kernel gathers them: this vertex
    // against each neighbour's segment prev(j) -> j (force on v), each
    // neighbour against this vertex's segment prev(v) -> v (force on v as its
    // end o), and each neighbour of next(v) against the segment v -> next(v)
    // (force on v as its start q)
    for (int s = 0; s < cnt; s++) {
      const int j = g.nbr[(size_t)s * p.nv + v];
      const HD2 xj = load_x(g, j), xjq = load_x(g, prev_of(g, j, 1)), xjqq = load_x(g, prev_of(g, j, 2));
      const HD rsum = ri + scaled_length(g, g.rad[j]);
      smooth_hd<POT, 1>(g, pbc2_hd(x, xjq, bx), pbc2_hd(x, xj, bx), pbc2_hd(xj, xjq, bx), pbc2_hd(xjq, xjqq, bx), rsum,
                        F, E);
      smooth_hd<POT, 2>(g, pbc2_hd(xj, xp, bx), pbc2_hd(xj, x, bx), ps, pps, rsum, F, E);
    }
    const HD rn = scaled_length(g, g.rad[vn]);
    const int cntn = min(g.nbr_cnt[vn], g.nbr_cap);
    HD none = hd(0.0);
    for (int s = 0; s < cntn; s++) {
      const int j = g.nbr[(size_t)s * p.nv + vn];
      const HD2 xj = load_x(g, j);
      smooth_hd<POT, 3>(g, pbc2_hd(xj, x, bx), pbc2_hd(xj, xn, bx), ns, ps, rn + scaled_length(g, g.rad[j]), F, none);
    }
  }
  double* fo = g.force_out + (size_t)v * 8;
  fo[0] = F.x.a; fo[1] = F.x.b; fo[2] = F.x.c; fo[3] = F.x.d;
  fo[4] = F.y.a; fo[5] = F.y.b; fo[6] = F.y.c; fo[7] = F.y.d;
  double* eo = g.energy_out + (size_t)v * 4;
  eo[0] = E.a; eo[1] = E.b; eo[2] = E.c; eo[3] = E.d;
}

}  // namespace

namespace {
// small CTAs: the systems these derivatives serve hold a few thousand
// vertices, so 32-thread CTAs spread them over every SM
template <int INTER>
void launch_diff_i(cudaStream_t st, int pot, const DiffArgs& g) {
  const int nb = (g.p.nv + 31) / 32;
  switch (pot) {
    case POT_HARMONIC: k_diff<POT_HARMONIC, INTER><<<nb, 32, 0, st>>>(g); break;
    case POT_LJ: k_diff<POT_LJ, INTER><<<nb, 32, 0, st>>>(g); break;
    case POT_ADHESIVE: k_diff<POT_ADHESIVE, INTER><<<nb, 32, 0, st>>>(g); break;
    default: k_diff<POT_WCA, INTER><<<nb, 32, 0, st>>>(g); break;
  }
}
}  // namespace

void launch_diff(cudaStream_t st, int pot, int inter, const DiffArgs& g, const int* ring_first, const int* ring_nv) {
  k_ring_area_hd<<<(g.p.np + 63) / 64, 64, 0, st>>>(g, ring_first, ring_nv);
  if (inter == INT_VV) launch_diff_i<INT_VV>(st, pot, g);
  else launch_diff_i<INT_SMOOTH>(st, pot, g);
}

// Fixed-order dot products for the Hessian solves: one partial per CTA, the
// host sums them in CTA order.
__global__ void __launch_bounds__(256) k_dot_partials(int n, const double* a, const double* b, double* out) {
  double acc = 0.0;
  for (int i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) acc += a[i] * b[i];
  __shared__ double s[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0;
    for (int w = 0; w < 8; w++) x += s[w];
    out[blockIdx.x] = x;
  }
}

// y = a x + b y
__global__ void k_axpby(int n, double a, const double* x, double b, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i] + b * y[i];
}

// the e1 part of the hyper-dual forces, negated: H t1
__global__ void k_extract_hv(int nv, const double* fhd, double* hv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    hv[2 * v] = -fhd[(size_t)v * 8 + 1];
    hv[2 * v + 1] = -fhd[(size_t)v * 8 + 5];
  }
}

// remove the mean of x and y components (the uniform translations, which
// span the Hessian's null space of a periodic system)
__global__ void k_sub_mean(int nv, double* x, double mx, double my) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    x[2 * v] -= mx;
    x[2 * v + 1] -= my;
  }
}

void launch_dot_partials(cudaStream_t st, int n, const double* a, const double* b, double* out, int nblocks) {
  k_dot_partials<<<nblocks, 256, 0, st>>>(n, a, b, out);
}
void launch_axpby(cudaStream_t st, int n, double a, const double* x, double b, double* y) {
  k_axpby<<<(n + 255) / 256, 256, 0, st>>>(n, a, x, b, y);
}
void launch_extract_hv(cudaStream_t st, int nv, const double* fhd, double* hv) {
  k_extract_hv<<<(nv + 255) / 256, 256, 0, st>>>(nv, fhd, hv);
}
void launch_sub_mean(cudaStream_t st, int nv, double* x, double mx, double my) {
  k_sub_mean<<<(nv + 255) / 256, 256, 0, st>>>(nv, x, mx, my);
}

// ----------------------------------------------- device-resident CG iteration
namespace {
constexpr int kCgBlock = 256;

__device__ __forceinline__ void cg_block_sums(double* v, int n, double* out) {
  // fixed-order CTA sums of n values per thread; results in out[0..n) on thread 0
  __shared__ double s[kCgBlock / 32][4];
  for (int q = 0; q < n; q++) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5][q] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < n; q++) {
      double t = 0.0;
      for (int w = 0; w < kCgBlock / 32; w++) t += s[w][q];
      out[q] = t;
    }
  }
}

// hp = H p (the negated e1 parts of the forces); partials: sum hp.x, sum hp.y, p.hp
__global__ void __launch_bounds__(kCgBlock) k_cg_hp(const __grid_constant__ CgArgs a) {
  if (((volatile CgState*)a.st)->done) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int v = blockIdx.x * kCgBlock + threadIdx.x; v < a.nv; v += a.nblk * kCgBlock) {
    const double hx = -a.fhd[(size_t)v * 8 + 1], hy = -a.fhd[(size_t)v * 8 + 5];
    a.hp[2 * v] = hx;
    a.hp[2 * v + 1] = hy;
    acc[0] += hx;
    acc[1] += hy;
    acc[2] += a.p[2 * v] * hx + a.p[2 * v + 1] * hy;
  }
  double out[3];
  cg_block_sums(acc, 3, out);
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) a.partials[(size_t)8 * blockIdx.x + q] = out[q];
}

// one thread: the mean of H p and the step alpha = r.z / p.Hp (p carries no
// translation, so p.Hp is the curvature along p of the projected Hessian)
__global__ void k_cg_alpha(const __grid_constant__ CgArgs a) {
  CgState& st = *a.st;
  if (st.done) return;
  double sx = 0.0, sy = 0.0, php = 0.0;
  for (int b = 0; b < a.nblk; b++) {
    sx += a.partials[8 * b];
    sy += a.partials[8 * b + 1];
    php += a.partials[8 * b + 2];
  }
  st.mx = sx / a.nv;
  st.my = sy / a.nv;
  if (!(php > 0.0)) {
    st.bad = 1;
    st.done = 1;
    return;
  }
  st.alpha = st.rz / php;
}

// z = M^-1 r at vertex v (2 x 2 block), or z = r without a preconditioner
__device__ __forceinline__ double2 cg_precondition(const double* minv, int v, double rx, double ry) {
  if (!minv) return make_double2(rx, ry);
  const double* m = minv + (size_t)3 * v;
  return make_double2(m[0] * rx + m[1] * ry, m[1] * rx + m[2] * ry);
}

// x += alpha p; r -= alpha (H p - mean); z = M^-1 r; partials: |r|^2, r.z,
// sum z.x, sum z.y (one vertex, both components, per thread)
__global__ void __launch_bounds__(kCgBlock) k_cg_update(const __grid_constant__ CgArgs a) {
  const CgState st = *(const CgState*)a.st;
  if (st.done) return;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int v = blockIdx.x * kCgBlock + threadIdx.x; v < a.nv; v += a.nblk * kCgBlock) {
    a.x[2 * v] += st.alpha * a.p[2 * v];
    a.x[2 * v + 1] += st.alpha * a.p[2 * v + 1];
    const double rx = a.r[2 * v] - st.alpha * (a.hp[2 * v] - st.mx);
    const double ry = a.r[2 * v + 1] - st.alpha * (a.hp[2 * v + 1] - st.my);
    a.r[2 * v] = rx;
    a.r[2 * v + 1] = ry;
    const double2 z = cg_precondition(a.minv, v, rx, ry);
    a.z[2 * v] = z.x;
    a.z[2 * v + 1] = z.y;
    acc[0] += rx * rx + ry * ry;
    acc[1] += rx * z.x + ry * z.y;
    acc[2] += z.x;
    acc[3] += z.y;
  }
  double out[4];
  cg_block_sums(acc, 4, out);
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; q++) a.partials[(size_t)8 * blockIdx.x + 3 + q] = out[q];
}

// one thread: the new |r|^2 and r.z, beta = r.z / previous r.z, the mean of
// z, the iteration count and the stop tests of the host loop (relative
// residual, iteration limit)
__global__ void k_cg_beta(const __grid_constant__ CgArgs a) {
  CgState& st = *a.st;
  if (st.done) return;
  double rr2 = 0.0, rz2 = 0.0, zx = 0.0, zy = 0.0;
  for (int b = 0; b < a.nblk; b++) {
    rr2 += a.partials[8 * b + 3];
    rz2 += a.partials[8 * b + 4];
    zx += a.partials[8 * b + 5];
    zy += a.partials[8 * b + 6];
  }
  st.beta = rz2 / st.rz;
  st.rz = rz2;
  st.rr = rr2;
  st.zx = zx / a.nv;
  st.zy = zy / a.nv;
  st.iters += 1;
  if (!(sqrt(st.rr / st.bb) > st.tol) || st.iters >= st.max_iters) st.done = 1;
}

// p = (z - mean z) + beta p: the preconditioned residual without its
// translation (r carries none, so r.z needs no correction)
__global__ void __launch_bounds__(kCgBlock) k_cg_direction(const __grid_constant__ CgArgs a) {
  const CgState st = *(const CgState*)a.st;
  if (st.done) return;
  for (int i = blockIdx.x * kCgBlock + threadIdx.x; i < 2 * a.nv; i += a.nblk * kCgBlock)
    a.p[i] = (a.z[i] - ((i & 1) ? st.zy : st.zx)) + st.beta * a.p[i];
}

// inverse diagonal blocks from a diag-mode launch: H_vv = -[[Fx.b, Fx.c],
// [Fy.b, Fy.c]] symmetrised; where it is not positive definite, the inverse
// of its diagonal's magnitudes (floored at 1e-3 of the larger), and the
// identity for a zero block
__global__ void k_cg_prec(int nv, const double* fhd, double* minv) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const double* f = fhd + (size_t)8 * v;
  const double h11 = -f[1], h22 = -f[6], h12 = -0.5 * (f[2] + f[5]);
  const double det = h11 * h22 - h12 * h12;
  double* m = minv + (size_t)3 * v;
  if (h11 > 0.0 && h22 > 0.0 && det > 1e-12 * h11 * h22) {
    m[0] = h22 / det;
    m[1] = -h12 / det;
    m[2] = h11 / det;
  } else {
    const double s = fmax(fabs(h11), fabs(h22));
    m[0] = s > 0.0 ? 1.0 / fmax(fabs(h11), 1e-3 * s) : 1.0;
    m[1] = 0.0;
    m[2] = s > 0.0 ? 1.0 / fmax(fabs(h22), 1e-3 * s) : 1.0;
  }
}

__global__ void k_cg_apply(int nv, const double* minv, const double* r, double* z) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const double2 q = cg_precondition(minv, v, r[2 * v], r[2 * v + 1]);
  z[2 * v] = q.x;
  z[2 * v + 1] = q.y;
}
}  // namespace

int cg_blocks(int nv) { return std::max(1, std::min(148, (nv + kCgBlock - 1) / kCgBlock)); }

void launch_cg_prec(cudaStream_t st, int nv, const double* fhd, double* minv) {
  k_cg_prec<<<(nv + 127) / 128, 128, 0, st>>>(nv, fhd, minv);
}

void launch_cg_apply(cudaStream_t st, int nv, const double* minv, const double* r, double* z) {
  k_cg_apply<<<(nv + 127) / 128, 128, 0, st>>>(nv, minv, r, z);
}

void launch_cg_iteration(cudaStream_t st, const CgArgs& a) {
  k_cg_hp<<<a.nblk, kCgBlock, 0, st>>>(a);
  k_cg_alpha<<<1, 1, 0, st>>>(a);
  k_cg_update<<<a.nblk, kCgBlock, 0, st>>>(a);
  k_cg_beta<<<1, 1, 0, st>>>(a);
  k_cg_direction<<<a.nblk, kCgBlock, 0, st>>>(a);
}

}  // namespace cr
