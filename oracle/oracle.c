/* CPU oracle: plain-C restatement of the cudaRing hot path.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg.  Each function restates the reference
 * function cited beside it (paths are within the farceri/cudaRing project).
 * The arithmetic follows the reference's order of operations so that results
 * agree with the reference kernels to rounding; parity is pinned against the
 * reference compiled as host code (oracle/_ref) via tests/golden/.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double OC_PI = 3.141592653589793238462643383279502884197;
static const double OC_WCACUT = 1.122462048; /* include/defs.h:17 */

/* pbcDistance (include/cudaKernel.cuh:70-74) */
static inline double pbc(const oc_sys* s, double x1, double x2, int dim) {
  double delta = x1 - x2;
  double size = dim == 0 ? s->lx : s->ly;
  return delta - size * round(delta / size);
}

/* getNextId / getPreviousId (include/cudaKernel.cuh:220-243) */
static inline long next_id(const oc_sys* s, long v, long p) {
  if (v == s->nv - 1) return v - s->nv_list[p] + 1;
  long n = v + 1;
  return s->pid[n] == p ? n : n - s->nv_list[p];
}
static inline long prev_id(const oc_sys* s, long v, long p) {
  if (v == 0) return s->nv_list[p] - 1;
  long q = v - 1;
  return s->pid[q] == p ? q : q + s->nv_list[p];
}

/* calcDeltaAndDistance for periodic geometry (include/cudaKernel.cuh:163-203) */
static inline double delta_dist(const oc_sys* s, const double* a, const double* b, double* d) {
  d[0] = pbc(s, a[0], b[0], 0);
  d[1] = pbc(s, a[1], b[1], 1);
  double sq = d[0] * d[0];
  sq += d[1] * d[1];
  return sqrt(sq);
}
static inline double dist(const oc_sys* s, const double* a, const double* b) {
  double d[2];
  return delta_dist(s, a, b, d);
}

/* kernelCalcParticleShape (include/cudaKernel.cuh:1571-1606): serial walk of
 * each ring in PBC-unwrapped coordinates; theta by calcAngle (:423-427). */
void oc_particle_shape(const oc_sys* s, const double* pos, double* length, double* theta,
                       double* area, double* perimeter) {
#pragma omp parallel for schedule(static)
  for (long p = 0; p < s->np; p++) {
    double temp_area = 0.0, per = 0.0;
    long first = s->first[p];
    double cur[2] = {pos[2 * first], pos[2 * first + 1]};
    for (long c = first; c < first + s->nv_list[p]; c++) {
      long n = next_id(s, c, p), q = prev_id(s, c, p);
      double nextp[2], prevp[2], seglen = 0.0;
      for (int d = 0; d < 2; d++) {
        double dl = pbc(s, pos[2 * n + d], cur[d], d);
        nextp[d] = cur[d] + dl;
        seglen += dl * dl;
        dl = pbc(s, pos[2 * q + d], cur[d], d);
        prevp[d] = cur[d] + dl;
      }
      double ns[2] = {nextp[0] - cur[0], nextp[1] - cur[1]};
      double ps[2] = {cur[0] - prevp[0], cur[1] - prevp[1]};
      double sine = ns[0] * ps[1] - ns[1] * ps[0];
      double cosine = ns[0] * ps[0] + ns[1] * ps[1];
      theta[c] = atan2(sine, cosine);
      length[c] = sqrt(seglen);
      per += length[c];
      temp_area += cur[0] * nextp[1] - nextp[0] * cur[1];
      cur[0] = nextp[0];
      cur[1] = nextp[1];
    }
    perimeter[p] = per;
    area[p] = fabs(temp_area) * 0.5;
  }
}

/* calcParticlePos (include/cudaKernel.cuh:365-388) */
void oc_particle_positions(const oc_sys* s, const double* pos, double* ppos) {
#pragma omp parallel for schedule(static)
  for (long p = 0; p < s->np; p++) {
    long first = s->first[p];
    double cur[2] = {pos[2 * first], pos[2 * first + 1]};
    double sum[2] = {cur[0], cur[1]};
    for (long c = first; c < first + s->nv_list[p] - 1; c++) {
      long n = next_id(s, c, p);
      for (int d = 0; d < 2; d++) {
        double dl = pbc(s, pos[2 * n + d], cur[d], d);
        cur[d] += dl;
        sum[d] += cur[d];
      }
    }
    ppos[2 * p] = sum[0] / s->nv_list[p];
    ppos[2 * p + 1] = sum[1] / s->nv_list[p];
  }
}

/* kernelCalcShapeForceEnergy (include/cudaKernel.cuh:474-529) with
 * calcAreaForceEnergy (:429-435), calcPerimeterForceEnergy (:437-447),
 * calcFENEPerimeterForceEnergy (:449-455), calcBendingForceEnergy (:457-471). */
void oc_shape_force_energy(const oc_sys* s, const double* a0, const double* area, const double* ppos,
                           const double* l0, const double* theta0, const double* theta,
                           const double* pos, double* force, double* energy) {
#pragma omp parallel for schedule(static)
  for (long v = 0; v < s->nv; v++) {
    long p = s->pid[v];
    long n = next_id(s, v, p), q = prev_id(s, v, p);
    double pc[2] = {ppos[2 * p], ppos[2 * p + 1]};
    double vp[2], np_[2], pp[2];
    for (int d = 0; d < 2; d++) {
      vp[d] = pbc(s, pos[2 * v + d], pc[d], d);
      np_[d] = pbc(s, pos[2 * n + d], pc[d], d);
      pp[d] = pbc(s, pos[2 * q + d], pc[d], d);
    }
    double f[2] = {0.0, 0.0};
    double e = 0.0;
    /* area */
    double dA = (area[p] / a0[p]) - 1.;
    double gm = s->ea * dA / a0[p];
    f[0] += 0.5 * gm * (pp[1] - np_[1]);
    f[1] += 0.5 * gm * (np_[0] - pp[0]);
    e += (0.5 * s->ea * dA * dA) / s->nv_list[p];
    /* segments */
    double nseg[2] = {np_[0] - vp[0], np_[1] - vp[1]};
    double pseg[2] = {vp[0] - pp[0], vp[1] - pp[1]};
    double plen = sqrt(pseg[0] * pseg[0] + pseg[1] * pseg[1]);
    double nlen = sqrt(nseg[0] * nseg[0] + nseg[1] * nseg[1]);
    double tl0 = l0[v], pl0 = l0[q];
    if (s->monomer == OC_MONO_HARMONIC) {
      double pd = (plen / pl0) - 1.;
      double nd = (nlen / tl0) - 1.;
      for (int d = 0; d < 2; d++)
        f[d] += s->el * ((nd * (np_[d] - vp[d]) / (tl0 * nlen)) - (pd * (vp[d] - pp[d]) / (pl0 * plen)));
      e += 0.5 * s->el * pd * pd;
    } else {
      for (int d = 0; d < 2; d++)
        f[d] += 2 * s->el * s->stiff * s->ext_sq *
                ((nlen / (s->ext_sq * tl0 * tl0 - nlen * nlen)) * (np_[d] - vp[d]) / nlen -
                 (plen / (s->ext_sq * pl0 * pl0 - plen * plen)) * (vp[d] - pp[d]) / plen);
      e += s->el * s->stiff * s->ext_sq * log(1 - plen * plen / (s->ext_sq * pl0 * pl0));
    }
    /* bending */
    double prevAD = theta[q] - theta0[q];
    double thisAD = theta[v] - theta0[v];
    double nextAD = theta[n] - theta0[n];
    double pnorm[2] = {pseg[1], -pseg[0]};
    double nnorm[2] = {nseg[1], -nseg[0]};
    double pvar = (thisAD - prevAD) / (pseg[0] * pseg[0] + pseg[1] * pseg[1]);
    double nvar = (thisAD - nextAD) / (nseg[0] * nseg[0] + nseg[1] * nseg[1]);
    for (int d = 0; d < 2; d++) f[d] += s->eb * (pvar * pnorm[d] + nvar * nnorm[d]);
    e += 0.5 * s->eb * thisAD * thisAD;
    force[2 * v] = f[0];
    force[2 * v + 1] = f[1];
    energy[v] = e;
  }
}

/* Own-side pair force of kernelCalcVertexInteraction: calcContactInteraction
 * (:531-544), calcLJInteraction (:567-583), calcAdhesiveInteraction (:604-626),
 * calcWCAInteraction (:653-668).  Adds to f, returns the half-pair energy. */
static double pair_own(const oc_sys* s, const double* a, const double* b, double rsum, double* f) {
  double dl[2];
  double d = delta_dist(s, a, b, dl);
  if (s->potential == OC_HARMONIC) {
    double ov = 1 - d / rsum;
    if (ov > 0) {
      double gm = s->ec * ov / rsum;
      for (int k = 0; k < 2; k++) f[k] += gm * dl[k] / d;
      return (0.5 * s->ec * ov * ov) * 0.5;
    }
    return 0.0;
  } else if (s->potential == OC_LJ) {
    double ratio = rsum / d;
    double r6 = pow(ratio, 6);
    double r12 = r6 * r6;
    if (d <= (s->lj_cutoff * rsum)) {
      double fshift = s->lj_fshift / rsum;
      double gm = 24 * s->ec * (2 * r12 - r6) / d - fshift;
      for (int k = 0; k < 2; k++) f[k] += gm * dl[k] / d;
      return 0.5 * (4 * s->ec * (r12 - r6) - s->lj_ecut - fabs(fshift) * (d - s->lj_cutoff * rsum));
    }
    return 0.0;
  } else if (s->potential == OC_ADHESIVE) {
    double ov = 1 - d / rsum, gm, ep;
    if (d < (1 + s->l2) * rsum) {
      if (d < (1 + s->l1) * rsum) {
        gm = s->ec * ov / rsum;
        ep = 0.5 * s->ec * (ov * ov - s->l1 * s->l2) * 0.5;
      } else {
        gm = -(s->ec * s->l1 / (s->l2 - s->l1)) * (ov + s->l2) / rsum;
        ep = -(0.5 * (s->ec * s->l1 / (s->l2 - s->l1)) * (ov + s->l2) * (ov + s->l2)) * 0.5;
      }
      for (int k = 0; k < 2; k++) f[k] += gm * dl[k] / d;
      return ep;
    }
    return 0.0;
  } else { /* WCA */
    double ratio = rsum / d;
    double r6 = pow(ratio, 6);
    double r12 = r6 * r6;
    if (d <= (OC_WCACUT * rsum)) {
      double gm = 24 * s->ec * (2 * r12 - r6) / d;
      for (int k = 0; k < 2; k++) f[k] += gm * dl[k] / d;
      return 0.5 * s->ec * (4 * (r12 - r6) + 1);
    }
    return 0.0;
  }
}

/* kernelCalcVertexInteraction (include/cudaKernel.cuh:690-722): accumulates
 * into force/energy (the shape pass zeroed them). */
void oc_vertex_interaction(const oc_sys* s, const double* rad, const double* pos, const long* nbr,
                           const long* cnt, long list_size, double* force, double* energy) {
#pragma omp parallel for schedule(static)
  for (long v = 0; v < s->nv; v++) {
    const double* a = pos + 2 * v;
    for (long k = 0; k < cnt[v]; k++) {
      long o = nbr[v * list_size + k];
      if (o != v && o != -1) {
        energy[v] += pair_own(s, a, pos + 2 * o, rad[v] + rad[o], force + 2 * v);
      }
    }
  }
}

/* kernelCalcAllToAllVertexInteraction (include/cudaKernel.cuh:725-757) */
void oc_all_to_all_interaction(const oc_sys* s, const double* rad, const double* pos, double* force,
                               double* energy) {
#pragma omp parallel for schedule(static)
  for (long v = 0; v < s->nv; v++) {
    for (long o = 0; o < s->nv; o++) {
      if (s->pid[v] != s->pid[o]) {
        energy[v] += pair_own(s, pos + 2 * v, pos + 2 * o, rad[v] + rad[o], force + 2 * v);
      }
    }
  }
}

/* calcGradMultipleAndEnergy (include/cudaKernel.cuh:806-858) */
static double grad_multiple(const oc_sys* s, const double* a, const double* b, double rsum, double* ep) {
  double d = dist(s, a, b);
  double ov, ratio, r6, r12;
  switch (s->potential) {
    case OC_HARMONIC:
      ov = 1 - d / rsum;
      if (ov > 0) {
        *ep = 0.5 * s->ec * ov * ov * 0.5;
        return s->ec * ov / rsum;
      }
      return 0;
    case OC_LJ:
      ratio = rsum / d;
      r12 = pow(ratio, 12);
      r6 = pow(ratio, 6);
      if (d <= (s->lj_cutoff * rsum)) {
        double fshift = s->lj_fshift / rsum;
        *ep = 0.5 * (4 * s->ec * (r12 - r6) - s->lj_ecut - fabs(fshift) * (d - s->lj_cutoff * rsum));
        return 24 * s->ec * (2 * r12 - r6) / d - fshift;
      }
      return 0;
    case OC_ADHESIVE:
      ov = 1 - d / rsum;
      if (d < (1 + s->l1) * rsum) {
        *ep = 0.5 * s->ec * (ov * ov - s->l1 * s->l2) * 0.5;
        return s->ec * ov / rsum;
      } else if ((d >= (1 + s->l1) * rsum) && (d < (1 + s->l2) * rsum)) {
        *ep = -(0.5 * (s->ec * s->l1 / (s->l2 - s->l1)) * (ov + s->l2) * (ov + s->l2)) * 0.5;
        return -(s->ec * s->l1 / (s->l2 - s->l1)) * (ov + s->l2) / rsum;
      }
      return 0;
    default: /* WCA */
      ratio = rsum / d;
      r6 = pow(ratio, 6);
      r12 = r6 * r6;
      if (d <= (OC_WCACUT * rsum)) {
        *ep = 0.5 * s->ec * (4 * (r12 - r6) + 1);
        return 4 * s->ec * (12 * r12 - 6 * r6) / d;
      }
      return 0;
  }
}

static inline void atomic_add(double* a, double v) {
#pragma omp atomic
  *a += v;
}

/* calcVertexSegmentInteraction (include/cudaKernel.cuh:877-897) */
static double vertex_segment(const oc_sys* s, const double* t, const double* proj, const double* o,
                             const double* q, double len, double rsum, double* ft, double* fo,
                             double* fq) {
  double ep = 0.0;
  double gm = grad_multiple(s, t, proj, rsum, &ep);
  if (gm != 0) {
    double cross = pbc(s, q[0], o[0], 0) * pbc(s, o[1], t[1], 1) - pbc(s, o[0], t[0], 0) * pbc(s, q[1], o[1], 1);
    double ac = fabs(cross);
    double sign = cross / ac;
    atomic_add(&ft[0], gm * sign * pbc(s, q[1], o[1], 1) / len);
    atomic_add(&ft[1], gm * sign * pbc(s, o[0], q[0], 0) / len);
    atomic_add(&fo[0], gm * (sign * pbc(s, t[1], q[1], 1) + ac * pbc(s, q[0], o[0], 0) / (len * len)) / len);
    atomic_add(&fo[1], gm * (sign * pbc(s, q[0], t[0], 0) + ac * pbc(s, q[1], o[1], 1) / (len * len)) / len);
    atomic_add(&fq[0], gm * (sign * pbc(s, o[1], t[1], 1) - ac * pbc(s, q[0], o[0], 0) / (len * len)) / len);
    atomic_add(&fq[1], gm * (sign * pbc(s, t[0], o[0], 0) - ac * pbc(s, q[1], o[1], 1) / (len * len)) / len);
    return ep;
  }
  return 0.;
}

/* calcVertexVertexInteraction (include/cudaKernel.cuh:899-912) */
static double vertex_vertex(const oc_sys* s, const double* a, const double* b, double rsum, double* fa,
                            double* fb) {
  double ep = 0.0;
  double gm = grad_multiple(s, a, b, rsum, &ep);
  if (gm != 0) {
    double dl[2];
    double d = delta_dist(s, a, b, dl);
    for (int k = 0; k < 2; k++) {
      atomic_add(&fa[k], gm * dl[k] / d);
      atomic_add(&fb[k], -gm * dl[k] / d);
    }
    return ep;
  }
  return 0.;
}

/* getProjection (include/cudaKernel.cuh:861-864) */
static inline double projection(const oc_sys* s, const double* t, const double* o, const double* q, double len) {
  return (pbc(s, t[0], q[0], 0) * pbc(s, o[0], q[0], 0) + pbc(s, t[1], q[1], 1) * pbc(s, o[1], q[1], 1)) /
         (len * len);
}

/* kernelCalcSmoothInteraction (include/cudaKernel.cuh:922-975) */
void oc_smooth_interaction(const oc_sys* s, const double* rad, const double* pos, const long* nbr,
                           const long* cnt, long list_size, double* force, double* p_energy) {
#pragma omp parallel for schedule(dynamic, 64)
  for (long v = 0; v < s->nv; v++) {
    const double* t = pos + 2 * v;
    long p = s->pid[v];
    for (long k = 0; k < cnt[v]; k++) {
      long o = nbr[v * list_size + k];
      if (o == v || o == -1) continue;
      double rsum = rad[v] + rad[o];
      long op = s->pid[o];
      long q = prev_id(s, o, op);
      const double* ot = pos + 2 * o;
      const double* qt = pos + 2 * q;
      double seg[2] = {pbc(s, ot[0], qt[0], 0), pbc(s, ot[1], qt[1], 1)};
      double len = sqrt(seg[0] * seg[0] + seg[1] * seg[1]);
      double proj = projection(s, t, ot, qt, len);
      long qq = prev_id(s, q, op);
      const double* qqt = pos + 2 * qq;
      double pseg[2] = {pbc(s, qqt[0], qt[0], 0), pbc(s, qqt[1], qt[1], 1)};
      double plen = sqrt(pseg[0] * pseg[0] + pseg[1] * pseg[1]);
      double pproj = projection(s, t, qt, qqt, plen);
      if (proj >= 0 && proj < 1) {
        double rp = proj < 0 ? 0.0 : (proj > 1 ? 1.0 : proj);
        double pj[2] = {qt[0] + rp * seg[0], qt[1] + rp * seg[1]};
        double e = vertex_segment(s, t, pj, ot, qt, len, rsum, force + 2 * v, force + 2 * o, force + 2 * q);
        atomic_add(&p_energy[p], e);
        atomic_add(&p_energy[op], e);
        if (pproj >= 0 && pproj < 1) {
          e = vertex_vertex(s, qt, t, rsum, force + 2 * v, force + 2 * q);
          atomic_add(&p_energy[p], -e);
          atomic_add(&p_energy[op], -e);
        }
      } else if (proj < 0) {
        if (pproj >= 1) {
          double e = vertex_vertex(s, t, qt, rsum, force + 2 * v, force + 2 * q);
          atomic_add(&p_energy[p], e);
          atomic_add(&p_energy[op], e);
        }
      }
    }
  }
}

/* kernelCalcNeighborList (include/cudaKernel.cuh:1735-1763): neighbours are
 * vertices of other rings with -(1 - d/radSum) < cutDistance, ascending. */
long oc_neighbor_list(const oc_sys* s, const double* pos, const double* rad, double cut_distance,
                      long list_size, long* nbr, long* cnt) {
  long maxc = -1;
#pragma omp parallel for schedule(dynamic, 64) reduction(max : maxc)
  for (long v = 0; v < s->nv; v++) {
    long added = 0;
    for (long o = 0; o < s->nv; o++) {
      if (s->pid[o] == s->pid[v]) continue;
      double rsum = rad[v] + rad[o];
      int is_nb = (-(1 - dist(s, pos + 2 * v, pos + 2 * o) / rsum) < cut_distance);
      if (added < list_size) nbr[v * list_size + added] = is_nb ? o : -1;
      added += is_nb;
    }
    cnt[v] = added;
    if (added > maxc) maxc = added;
  }
  return maxc;
}

int oc_check_displacement(const oc_sys* s, const double* pos, const double* last_pos, double cutoff) {
  int flag = 0;
  for (long v = 0; v < s->nv; v++) {
    if (3 * dist(s, pos + 2 * v, last_pos + 2 * v) > cutoff) flag = 1;
  }
  return flag;
}

void oc_calc_force_energy(const oc_sys* s, const double* pos, const double* rad, const double* a0,
                          const double* l0, const double* theta0, const long* nbr, const long* cnt,
                          long list_size, double* force, double* energy, double* p_energy,
                          double* length, double* theta, double* area, double* perimeter, double* ppos) {
  oc_particle_shape(s, pos, length, theta, area, perimeter);
  oc_particle_positions(s, pos, ppos);
  oc_shape_force_energy(s, a0, area, ppos, l0, theta0, theta, pos, force, energy);
  memset(p_energy, 0, sizeof(double) * s->np);
  if (s->interaction == OC_VERTEX_VERTEX) {
    oc_vertex_interaction(s, rad, pos, nbr, cnt, list_size, force, energy);
  } else if (s->interaction == OC_ALL) {
    oc_all_to_all_interaction(s, rad, pos, force, energy);
  } else {
    oc_smooth_interaction(s, rad, pos, nbr, cnt, list_size, force, p_energy);
  }
}

/* Rigid path: kernelCalcVertexForceTorque (:1412-1450),
 * kernelCalcTorqueAndMomentOfInertia (:1452-1470),
 * kernelCalcParticleRigidForceEnergy (:1472-1492), after
 * kernelCalcParticlePositions (DPM2D::calcRigidForceEnergy, src/DPM2D.cu:2128-2142). */
void oc_rigid_force_energy(const oc_sys* s, const double* pos, const double* rad, const long* nbr,
                           const long* cnt, long list_size, double* ppos, double* force,
                           double* torque, double* energy, double* moi, double* p_force,
                           double* p_torque, double* p_energy) {
  oc_particle_positions(s, pos, ppos);
#pragma omp parallel for schedule(static)
  for (long v = 0; v < s->nv; v++) {
    double f[2] = {0.0, 0.0};
    double e = 0.0;
    for (long k = 0; k < cnt[v]; k++) {
      long o = nbr[v * list_size + k];
      if (o != v && o != -1) e += pair_own(s, pos + 2 * v, pos + 2 * o, rad[v] + rad[o], f);
    }
    force[2 * v] = f[0];
    force[2 * v + 1] = f[1];
    energy[v] = e;
  }
#pragma omp parallel for schedule(static)
  for (long p = 0; p < s->np; p++) {
    double m = 0.0;
    for (long v = s->first[p]; v < s->first[p] + s->nv_list[p]; v++) {
      double r[2] = {pbc(s, pos[2 * v], ppos[2 * p], 0), pbc(s, pos[2 * v + 1], ppos[2 * p + 1], 1)};
      torque[v] = r[0] * force[2 * v + 1] - r[1] * force[2 * v];
      m += r[0] * r[0] + r[1] * r[1];
    }
    moi[p] = m;
    double pf[2] = {0.0, 0.0}, pt = 0.0, pe = 0.0;
    for (long v = s->first[p]; v < s->first[p] + s->nv_list[p]; v++) {
      pf[0] += force[2 * v];
      pf[1] += force[2 * v + 1];
      pt += torque[v];
      pe += energy[v];
    }
    p_force[2 * p] = pf[0];
    p_force[2 * p + 1] = pf[1];
    p_torque[p] = pt / m;
    p_energy[p] = pe;
  }
}

/* kernelTranslateVertices then kernelRotateVertices (:1678-1713) */
void oc_translate_rotate(const oc_sys* s, const double* ppos, const double* plast_pos,
                         const double* pangle, const double* plast_angle, double* pos) {
#pragma omp parallel for schedule(static)
  for (long p = 0; p < s->np; p++) {
    double dl[2] = {pbc(s, ppos[2 * p], plast_pos[2 * p], 0), pbc(s, ppos[2 * p + 1], plast_pos[2 * p + 1], 1)};
    double da = pangle[p] - plast_angle[p];
    double c = cos(da), sn = sin(da);
    for (long v = s->first[p]; v < s->first[p] + s->nv_list[p]; v++) {
      pos[2 * v] += dl[0];
      pos[2 * v + 1] += dl[1];
    }
    for (long v = s->first[p]; v < s->first[p] + s->nv_list[p]; v++) {
      double r[2] = {pbc(s, pos[2 * v], ppos[2 * p], 0), pbc(s, pos[2 * v + 1], ppos[2 * p + 1], 1)};
      double nx = r[0] * c - r[1] * sn;
      double ny = r[0] * sn + r[1] * c;
      pos[2 * v] += nx - r[0];
      pos[2 * v + 1] += ny - r[1];
    }
  }
}

/* Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11.  Multipliers and Weyl increments from the paper. */
void oc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Two standard normals from one Philox block: counter = (index, stream),
 * key = seed; Box-Muller on two 53-bit uniforms. */
void oc_normal2(uint64_t seed, uint64_t stream, uint64_t index, double out[2]) {
  uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t r[4];
  oc_philox4x32(ctr, key, r);
  uint64_t a = (uint64_t)r[0] | ((uint64_t)r[1] << 32);
  uint64_t b = (uint64_t)r[2] | ((uint64_t)r[3] << 32);
  double u1 = ((double)(a >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
  double rad = sqrt(-2.0 * log(u1));
  double ang = 2.0 * OC_PI * u2;
  out[0] = rad * cos(ang);
  out[1] = rad * sin(ang);
}
