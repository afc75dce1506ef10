// FIRE pre-kick of batched systems: the part of a FIRE iteration up to the
// position update, per vertex, with each system's own scalars, sums and
// convergence (the single-system k_fire_pre: FIRE::minimizerVertexLoop,
// src/FIRE.cu:338-406).  Used by the one-op-per-launch kernel k_bfire_pre
// (cr_batch.cu) and by the persistent batched FIRE kernel k_bfire_steps
// (cr_tile_bsteps.cu).
#pragma once
#include "cr_launch.h"
#include "cr_tile.cuh"

namespace cr {

struct BFire {
  double2* pos;
  double2* vel;
  const double2* force;
  const double2* last_pos;
  const int* vsys;
  const int* sys_v0;
  BatchSys* bsys;
  double* bfire;
  FireParams fp;
  DevStatus* st;
  int nv;
  int use_cond;
  cudaGraphConditionalHandle cond;
};

// Vertex v: the system's FIRE scalars from its sums of the last force op
// (P = v.F, |v|^2, |F|^2), the velocity mixing, the first half kick and the
// position update, and the displacement check (a rebuild flags the system
// and the status block).  The system's first vertex stores the next scalars.
// A system at its iteration limit stops as if converged.
__device__ __forceinline__ void bfire_prekick(const BFire& f, int v) {
  DevStatus* st = f.st;
  const int s = f.vsys[v];
  BatchSys& bs = f.bsys[s];
  if (bs.active && !bs.converged && bs.fire_cap > 0 && bs.fire_iters >= bs.fire_cap) {
    // the tiles of the system skip the force op that follows
    if (v == f.sys_v0[s]) bs.converged = 1;
    return;
  }
  if (!bs.active || bs.converged) return;
  const long long it = bs.fire_iters;
  const double* cur = f.bfire + ((size_t)s * 2 + (it & 1)) * 4;
  double dt = cur[0], alpha = cur[1];
  long long nstep = (long long)cur[2];
  const double dt_max = cur[3];  // the system's own bound (10 x its starting dt in the reference drivers)
  const double P = bs.sums[S_VF], vv = bs.sums[S_VV], ff = bs.sums[S_FF];
  bool rollback = false;
  if (P > 0) {
    nstep++;
    if (nstep > f.fp.min_step) {
      dt = fmin(dt * f.fp.f_inc, dt_max);
      alpha *= f.fp.f_a;
    }
  } else {
    nstep = 0;
    dt = fmax(dt * f.fp.f_dec, dt_max / 10);
    alpha = f.fp.a_start;
    rollback = true;
  }
  if (v == f.sys_v0[s]) {
    double* nxt = f.bfire + ((size_t)s * 2 + ((it + 1) & 1)) * 4;
    nxt[0] = dt;
    nxt[1] = alpha;
    nxt[2] = (double)nstep;
    nxt[3] = dt_max;
  }
  // every product and sum rounded as written (no contraction left to the
  // compiler), so each kernel that calls this computes the same iterate
  const double h = 0.5 * dt;
  const double hh = __dmul_rn(h, h);
  const double vpost2 = rollback ? __dmul_rn(hh, ff) : __fma_rn(hh, ff, __fma_rn(dt, P, vv));
  double2 x = f.pos[v];
  double2 vel = f.vel[v];
  const double2 fv = f.force[v];
  if (rollback) {
    x = make_double2(__fma_rn(-h, vel.x, x.x), __fma_rn(-h, vel.y, x.y));
    vel = make_double2(0.0, 0.0);
  }
  vel = make_double2(__fma_rn(h, fv.x, vel.x), __fma_rn(h, fv.y, vel.y));
  if (ff > 0) {
    const double ratio = sqrt(__ddiv_rn(vpost2, ff));
    const double am = 1.0 - alpha;
    vel = make_double2(__fma_rn(am, vel.x, __dmul_rn(__dmul_rn(alpha, fv.x), ratio)),
                       __fma_rn(am, vel.y, __dmul_rn(__dmul_rn(alpha, fv.y), ratio)));
  }
  x = make_double2(__fma_rn(dt, vel.x, x.x), __fma_rn(dt, vel.y, x.y));
  f.pos[v] = x;
  f.vel[v] = vel;
  if (3.0 * dist_of(pbc2(bs.box, x, f.last_pos[v])) > bs.disp_cutoff) {
    bs.rebuild = 1;
    st->rebuild = 1;
  }
}

// Persistent batched FIRE kernel (cr_tile_bsteps.cu): nullptr when the
// configuration has none (FP64 only; tile shapes (1, 128) and (2, 192)).
// nmax = 0 only completes a force op left pending by the last launch.
using BFireStepsFn = void (*)(SysParams, SysArrays, StepArgs, BFire, int);
BFireStepsFn bfire_steps_fn(int pot, int inter, int lanes, int block);
int bfire_steps_max_blocks(BFireStepsFn fn, int block);
void launch_bfire_steps(BFireStepsFn fn, const LaunchCfg& c, int block, const SysParams& p, const SysArrays& a,
                        const StepArgs& s, const BFire& f, int nmax);

}  // namespace cr
