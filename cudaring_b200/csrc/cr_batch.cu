// Batches of independent systems of deformable rings, advanced together.
//
// A batch concatenates S systems (each with its own periodic box, ring count
// and packing fraction) into one set of vertex and ring arrays; per-system
// offset tables locate each system's vertices, rings, tiles and cells.  Every
// op is one launch over all systems: the tiled force / FIRE kernel in batch
// mode (tile.x = system, cr_tile_kernel.cuh), the FIRE pre-kick, and the
// cell-list build, which rebuilds only the systems whose displacement check
// fired.  Each system keeps its own FIRE scalars, convergence flag and
// rebuild flag; a converged system's tiles exit at once, so an iteration
// costs what the unconverged systems cost.  Iterations run as captured CUDA
// graphs with one conditional rebuild node per iteration.
//
// On top runs the quasi-static compression protocol of the reference's
// compressFIRE driver (compressFIRE.cpp:101-205), per system: FIRE to the
// force tolerance, the jammed / under-jammed / over-jammed decision, the
// saved under-jammed state, and the halving of the compression step when a
// system overshoots.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "cr_bfire.cuh"
#include "cr_launch.h"
#include "cr_tile.cuh"

using namespace cr;

// Compression protocol state of one system (cr_batch_compress on the device).
struct CompSys {
  double phi, prev, dphi;
  long long steps, fire_total;
  int state;  // 0 compressing, 1 jammed, 2 step limit, 3 step halved below min_dphi
  int pad;
};

struct cr_batch {
  int device = 0;
  cudaStream_t stream = nullptr, side = nullptr;
  int S = 0, nv = 0, np = 0;
  std::vector<int> sys_np, sys_nv, sys_v0, sys_r0;  // per system: rings, vertices, first vertex, first ring
  std::vector<int> ring_nv_h, ring_first_h, ring_sys_h, vsys_h;
  std::vector<int4> tiles_h;
  std::vector<BatchSys> bsys_h;
  std::vector<Box> box_h;
  std::vector<double> rmax_h, rmean_h;
  SysParams p{};
  int potential = CR_POTENTIAL_HARMONIC;
  int interaction = CR_INTERACTION_VERTEX_VERTEX;
  int lanes = 1;
  int block = 0;  // threads per tile CTA (0: the lane count's default)
  int precision = CR_PRECISION_FP64;
  double cutoff_ = 0.5;
  double cut_distance = 1.5;
  // device state
  double2 *pos = nullptr, *vel = nullptr, *force = nullptr, *last_pos = nullptr, *ppos = nullptr;
  double *rad = nullptr, *l0 = nullptr, *theta0 = nullptr, *a0 = nullptr, *energy = nullptr, *p_energy = nullptr,
         *theta = nullptr, *length = nullptr, *area = nullptr, *perimeter = nullptr;
  int2* vtopo = nullptr;
  int *pq_pack = nullptr, *ring_of = nullptr, *vsys = nullptr, *ring_sys = nullptr, *sys_v0_d = nullptr;
  int4* tiles = nullptr;
  int *nbr = nullptr, *nbr_pq = nullptr, *nbr_cnt = nullptr;
  int cap = 0;
  bool nbr_built = false;
  int *cell_of = nullptr, *slot = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_vid = nullptr,
      *cell_ring = nullptr, *cell_pq = nullptr;
  double2* cell_pos = nullptr;
  double* cell_rad = nullptr;
  int ncells = 0, ncells_alloc = 0;
  int4* sgrid = nullptr;  // per system: cells in x, cells in y, first cell, 0
  std::vector<int4> sgrid_h;
  BatchSys* bsys = nullptr;
  double* bfire = nullptr;  // [S][2][4]
  double* partials = nullptr;
  int partials_n = 0;
  double* sys_scalar = nullptr;  // [S] scratch for per-system scale factors
  int* sys_flag = nullptr;       // [S] save / restore requests
  DevStatus* status = nullptr;
  DevStatus* status_h = nullptr;
  // snapshot for recovering from a list overflow inside a FIRE chunk
  double2 *snap_pos = nullptr, *snap_vel = nullptr;
  BatchSys* snap_bsys = nullptr;
  double* snap_bfire = nullptr;
  // saved under-jammed configuration (compression)
  double2* save_pos = nullptr;
  double *save_rad = nullptr, *save_l0 = nullptr, *save_a0 = nullptr;
  FireParams fp{};
  bool fire_ready = false;
  // compression on the device (compress_device)
  CompSys* comp = nullptr;             // [S] per-system protocol state
  int *sys_nv_d = nullptr, *sys_r0_d = nullptr, *sys_np_d = nullptr, *cells0_d = nullptr;
  cudaStream_t cap_s2 = nullptr, cap_s3 = nullptr;  // capture streams of the nested loop bodies
  cudaGraphExec_t comp_exec = nullptr;
  // persistent batched FIRE (k_bfire_steps): off by request or after a
  // grid-barrier wait gave up; the chunk graph of the current list capacity
  bool no_persist = false;
  std::map<BFireStepsFn, int> persist_max;  // CTAs each kernel holds resident at once
  cudaGraphExec_t pchunk = nullptr;
  std::map<std::pair<long, int>, cudaGraphExec_t> graphs;  // (iterations, cap) -> FIRE chunk
  long long launches = 0;
  std::string err;
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
};

#define BT_TRY(expr)                                                                                    \
  do {                                                                                                  \
    cudaError_t e_ = (expr);                                                                            \
    if (e_ != cudaSuccess) return b->fail(CR_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

// ------------------------------------------------------------------ kernels

struct BNbr {
  const double2* pos;
  const double* rad;
  const int* ring_of;
  const int* vsys;
  const int* pq_pack;
  int* nbr;
  int* nbr_pq;
  int* nbr_cnt;
  int cap;
  int nv;
  double cut_distance;
  double2* last_pos;
  int* cell_of;
  int* slot;
  int* cell_cnt;
  int* cell_start;
  int* cell_vid;
  double2* cell_pos;
  double* cell_rad;
  int* cell_ring;
  int* cell_pq;
  const int4* sgrid;
  BatchSys* bsys;
  DevStatus* status;
  int S;
  int all;  // 1: every active system; 0: the systems whose rebuild flag is set
};

__device__ __forceinline__ bool b_selected(const BNbr& n, int s) {
  const BatchSys& b = n.bsys[s];
  return b.active && (n.all || b.rebuild);
}

__device__ __forceinline__ int b_cell_coord(double x, double L, double invL, int nc) {
  const double w = x - L * floor(x * invL);  // wrap into [0, L]
  const int c = (int)(w * (nc * invL));
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void k_bguard(DevStatus* st) {
  if (threadIdx.x == 0) {
    st->overflow = 0;
    st->max_count = 0;
  }
}

__global__ void __launch_bounds__(256) k_bcell_count(const __grid_constant__ BNbr n) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n.nv) return;
  const int s = n.vsys[v];
  if (!b_selected(n, s)) return;
  const int4 g = n.sgrid[s];
  const Box bx = n.bsys[s].box;
  const double2 x = n.pos[v];
  const int cx = b_cell_coord(x.x, bx.lx, bx.inv_lx, g.x);
  const int cy = b_cell_coord(x.y, bx.ly, bx.inv_ly, g.y);
  const int c = g.z + cy * g.x + cx;
  n.cell_of[v] = c;
  n.slot[v] = atomicAdd(n.cell_cnt + c, 1);
}

__global__ void __launch_bounds__(256) k_bcell_fill(const __grid_constant__ BNbr n) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= n.nv) return;
  if (!b_selected(n, n.vsys[v])) return;
  n.cell_vid[n.cell_start[n.cell_of[v]] + n.slot[v]] = v;
}

// The list rule of kernelCalcNeighborList (include/cudaKernel.cuh:1735-1763)
// over the 3x3 stencil of the vertex's own system (one cell when the system
// has fewer than three cells per side); the last CTA publishes the build.
__global__ void __launch_bounds__(256) k_bnbr(const __grid_constant__ BNbr n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int cnt = 0;
  if (i < n.nv && b_selected(n, n.vsys[i])) {
    const int s = n.vsys[i];
    const int4 g = n.sgrid[s];
    const Box bx = n.bsys[s].box;
    const double2 xi = n.pos[i];
    const double ri = n.rad[i];
    const int ring = n.ring_of[i];
    const int local = n.cell_of[i] - g.z;
    const int cx = local % g.x, cy = local / g.x;
    const int span = (g.x >= 3 && g.y >= 3) ? 1 : 0;
    for (int dy = -span; dy <= span; dy++) {
      int yy = cy + dy;
      yy += (yy < 0) ? g.y : 0;
      yy -= (yy >= g.y) ? g.y : 0;
      for (int dx = -span; dx <= span; dx++) {
        int xx = cx + dx;
        xx += (xx < 0) ? g.x : 0;
        xx -= (xx >= g.x) ? g.x : 0;
        const int cc = g.z + yy * g.x + xx;
        const int kb = n.cell_start[cc], ke = n.cell_start[cc + 1];
        for (int k = kb; k < ke; k++) {
          if (n.cell_ring[k] == ring) continue;
          const double d = dist_of(pbc2(bx, xi, n.cell_pos[k]));
          if (-(1.0 - d / (ri + n.cell_rad[k])) < n.cut_distance) {
            if (cnt < n.cap) {
              n.nbr[(size_t)cnt * n.nv + i] = n.cell_vid[k];
              n.nbr_pq[(size_t)cnt * n.nv + i] = n.cell_pq[k];
            }
            cnt++;
          }
        }
      }
    }
    n.nbr_cnt[i] = cnt;
    n.last_pos[i] = xi;
  }
  int m = cnt;
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ int s_max[8];
  __shared__ int s_ovf;
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    int bm = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) bm = max(bm, s_max[w]);
    if (bm > 0) atomicMax(&n.status->max_count, bm);
    if (bm > n.cap) atomicOr(&n.status->overflow, 1);
  }
  DevStatus* st = n.status;
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      __threadfence();
      s_ovf = st->overflow;
      if (st->max_count > st->max_ever) st->max_ever = st->max_count;
    }
    __syncthreads();
    if (!s_ovf)
      for (int s = threadIdx.x; s < n.S; s += blockDim.x)
        if (b_selected(n, s)) n.bsys[s].rebuild = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_ovf) st->abort = 1;
      else st->rebuild = 0;
      st->done_ctr = 0;
    }
  }
}

// FIRE iteration up to the position update, per system (the single-system
// k_fire_pre: FIRE::minimizerVertexLoop, src/FIRE.cu:338-406) with each
// system's own scalars, sums and convergence (bfire_prekick, cr_bfire.cuh).
__global__ void __launch_bounds__(256) k_bfire_pre(const __grid_constant__ BFire f) {
  DevStatus* st = f.st;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (!st->abort && v < f.nv) bfire_prekick(f, v);
  if (is_last_block(st)) {
    if (threadIdx.x == 0) {
      st->done_ctr = 0;
      if (f.use_cond) cudaGraphSetConditional(f.cond, (!st->abort && st->rebuild) ? 1u : 0u);
    }
  }
}

// Per-system sums of the stored velocities, forces and energies, one tile
// per CTA in a fixed order; the system's last tile reduces them and, with
// set_converged, sets the system's FIRE convergence flag.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_btile_reduce(const int4* tiles, const double2* vel, const double2* force,
                                                        const double* energy, const double* p_energy,
                                                        const int2* vtopo, int use_pe, BatchSys* bsys,
                                                        double* partials, int set_converged) {
  const int4 tile = tiles[blockIdx.x];
  double acc[NSUM] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int v = tile.z + threadIdx.x; v < tile.w; v += BLOCK) {
    const double2 u = vel[v], fv = force[v];
    acc[S_PE] += energy[v];
    if (use_pe) {
      const int2 tp = vtopo[v];
      if ((tp.y & 0xffff) == 0) acc[S_PE] += p_energy[tp.x];
    }
    acc[S_VV] += u.x * u.x + u.y * u.y;
    acc[S_VF] += u.x * fv.x + u.y * fv.y;
    acc[S_FF] += fv.x * fv.x + fv.y * fv.y;
    acc[S_FMAX2] = fmax(acc[S_FMAX2], fmax(fv.x * fv.x, fv.y * fv.y));
    if (!(isfinite(fv.x) && isfinite(fv.y))) acc[S_NONFINITE] = 1.0;
  }
  __shared__ double s_red[BLOCK / 32][NSUM];
  __shared__ bool s_last;
  block_partials<BLOCK>(acc, s_red, partials + (size_t)blockIdx.x * NSUM);
  BatchSys& bs = bsys[tile.x];
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int prev = atomicAdd(&bs.done_ctr, 1u);
    s_last = (prev == (unsigned int)(bs.tile_end - bs.tile_begin - 1));
  }
  __syncthreads();
  if (s_last) {
    reduce_partials(partials + (size_t)bs.tile_begin * NSUM, bs.tile_end - bs.tile_begin, bs.sums);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      if (set_converged) bs.converged = (bs.fire_tol >= 0.0 && bs.sums[S_FMAX2] <= bs.fire_tol * bs.fire_tol);
      bs.done_ctr = 0;
    }
  }
}

// Per-tile sum of the packing-fraction numerator of the tile's rings:
// area (or rest area) + pi r_first^2 (nv / 2 - 1) (src/DPM2D.cu:1202-1220).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_btile_phi(const int4* tiles, const int2* vtopo, const double* ring_area,
                                                     const double* rad, double* out) {
  const int4 tile = tiles[blockIdx.x];
  double acc = 0.0;
  for (int v = tile.z + threadIdx.x; v < tile.w; v += BLOCK) {
    const int2 tp = vtopo[v];
    if ((tp.y & 0xffff) == 0) {
      const double r = rad[v];
      acc += ring_area[tp.x] + kPi * r * r * (0.5 * (tp.y >> 16) - 1);
    }
  }
  __shared__ double s_red[BLOCK / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0;
    for (int w = 0; w < BLOCK / 32; w++) x += s_red[w];
    out[blockIdx.x] = x;
  }
}

// Scale each system's rings about their centroids by its own factor
// (DPM2D::scaleVertices, src/DPM2D.cu:1802-1811, per system).
__global__ void k_bscale(int nv, int np, const int* vsys, const int* ring_sys, const int* ring_of,
                         const double2* ppos, const double* scale, double2* pos, double* l0, double* rad, double* a0,
                         double* area) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    const double f = scale[vsys[v]];
    if (f != 1.0) {
      const double2 c = ppos[ring_of[v]];
      double2 x = pos[v];
      x.x += (f - 1) * (x.x - c.x);
      x.y += (f - 1) * (x.y - c.y);
      pos[v] = x;
      l0[v] *= f;
      rad[v] *= f;
    }
  }
  if (v < np) {
    const double f = scale[ring_sys[v]];
    if (f != 1.0) {
      a0[v] *= f * f;
      area[v] *= f * f;
    }
  }
}

// flag[s] = 1: save system s's positions, radii, rest lengths and areas;
// 2: restore them.
__global__ void k_bsave(int nv, int np, const int* vsys, const int* ring_sys, const int* flag, double2* pos,
                        double* rad, double* l0, double* a0, double2* spos, double* srad, double* sl0, double* sa0) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < nv) {
    const int fl = flag[vsys[v]];
    if (fl == 1) {
      spos[v] = pos[v];
      srad[v] = rad[v];
      sl0[v] = l0[v];
    } else if (fl == 2) {
      pos[v] = spos[v];
      rad[v] = srad[v];
      l0[v] = sl0[v];
    }
  }
  if (v < np) {
    const int fl = flag[ring_sys[v]];
    if (fl == 1) sa0[v] = a0[v];
    else if (fl == 2) a0[v] = sa0[v];
  }
}

// ------------------------------------------------------------------ compression on the device
//
// The compressFIRE protocol of cr_batch_compress as one CUDA graph: an outer
// WHILE node over compression steps and, inside it, a WHILE node over chunks
// of FIRE iterations (the chunk of the host loop, with its conditional
// rebuild nodes).  Every decision the host loop makes between launches is
// made here by a kernel, with the host loop's arithmetic in the host loop's
// order (per-system sums run sequentially on one thread), so both loops
// produce the same states.

struct CompArgs {
  CompSys* comp;
  BatchSys* bsys;
  double* bfire;
  int4* sgrid;
  const int* cells0;   // cells of each system's grid when the run started (its share of the cell arrays)
  const double* rad;
  const double* a0;
  const int* sys_v0;
  const int* sys_nv;
  const int* sys_r0;
  const int* sys_np;
  const double* partials;  // per-tile packing-fraction numerators (k_btile_phi)
  double* scale;           // [S] scale factor of the step
  int* flag;               // [S] save / restore request
  DevStatus* st;
  int S;
  double cutoff_, cut_distance;
  double dphi0, min_dphi, fire_dt, tol0, energy_tol;
  long long max_fire_iters, max_steps;
  int criterion;
  cudaGraphConditionalHandle outer, inner;
};

// Start of a compression step, one thread per system: the FIRE setup of the
// host loop (cr_batch_init_fire with dt = fire_dt sigma, the tolerance
// tol0 / sigma, the active set), the radius statistics behind the
// displacement cutoff, and the cell grid for the current largest radius.
__global__ void k_cstep_begin(const __grid_constant__ CompArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.S || a.st->abort) return;
  BatchSys& bs = a.bsys[s];
  double sa = 0.0;
  for (int q = a.sys_r0[s]; q < a.sys_r0[s] + a.sys_np[s]; q++) sa += a.a0[q];
  const double sigma = 2 * sqrt(sa / (kPi * a.sys_np[s]));  // DPM2D::getMeanParticleSize
  const double dt = a.fire_dt * sigma, dmax = (10 * a.fire_dt) * (dt / a.fire_dt);
  for (int par = 0; par < 2; par++) {
    double* f = a.bfire + ((size_t)s * 2 + par) * 4;
    f[0] = dt;
    f[1] = 0.2;
    f[2] = 0.0;
    f[3] = dmax;
  }
  double m = 0.0, sr = 0.0;
  for (int v = a.sys_v0[s]; v < a.sys_v0[s] + a.sys_nv[s]; v++) {
    m = fmax(m, a.rad[v]);
    sr += a.rad[v];
  }
  bs.fire_iters = 0;
  bs.converged = 0;
  bs.fire_tol = a.tol0 / sigma;
  bs.rebuild = 0;
  bs.done_ctr = 0;
  bs.active = a.comp[s].state == 0 ? 1 : 0;
  bs.fire_cap = a.max_fire_iters;
  bs.disp_cutoff = a.cutoff_ * 2.0 * (sr / a.sys_nv[s]);
  const double cmin = (1.0 + a.cut_distance) * 2.0 * m * (1.0 + 1e-9);
  int ncx = cmin > 0 ? (int)floor(bs.box.lx / cmin) : 1;
  int ncy = cmin > 0 ? (int)floor(bs.box.ly / cmin) : 1;
  ncx = min(ncx, 4096);
  ncy = min(ncy, 4096);
  if (ncx < 3 || ncy < 3) ncx = ncy = 1;
  // radii never fall below the run's starting radii, so the grid never
  // outgrows the system's share of the cell arrays
  if ((long long)ncx * ncy <= a.cells0[s]) {
    a.sgrid[s].x = ncx;
    a.sgrid[s].y = ncy;
  }
}

// Status flags of a fresh FIRE run (clear_flags without the abort flag).
__global__ void k_cclear(DevStatus* st) {
  st->overflow = 0;
  st->rebuild = 0;
  st->nonfinite = 0;
  st->converged = 0;
  st->done_ctr = 0;
  st->pbar = 0;
  st->bpending = 0;
}

// Loop condition of the FIRE chunks: a system still running and no abort.
__global__ void k_cfire_more(const __grid_constant__ CompArgs a) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < a.S; s += blockDim.x)
    if (a.bsys[s].active && !a.bsys[s].converged) s_any = 1;
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(a.inner, (s_any && !a.st->abort) ? 1u : 0u);
}

// The jammed / under-jammed / over-jammed decision (compressFIRE.cpp:141-172)
// of every compressing system, on the sums of the relaxed state.
__global__ void k_cdecide(const __grid_constant__ CompArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.S) return;
  if (a.st->abort) {
    // the step is run again: nothing saved, restored or scaled
    a.flag[s] = 0;
    a.scale[s] = 1.0;
    return;
  }
  CompSys& c = a.comp[s];
  const BatchSys& bs = a.bsys[s];
  int flag = 0;
  double scale = 1.0;
  if (c.state == 0) {
    c.fire_total += bs.fire_iters;
    c.steps += 1;
    const double fmax = sqrt(bs.sums[S_FMAX2]), tol = bs.fire_tol;
    bool jam, over, under;
    if (a.criterion == 1) {
      const double u = bs.sums[S_PE] / a.sys_np[s];
      jam = u > a.energy_tol && u < 2 * a.energy_tol;
      over = u >= 2 * a.energy_tol;
      under = u <= a.energy_tol;
    } else {
      jam = fmax > tol && fmax < 2 * tol;
      over = fmax >= 2 * tol;
      under = fmax <= tol;
    }
    if (jam) {
      c.state = 1;
    } else {
      if (under) {
        scale = sqrt((c.phi + c.dphi) / c.phi);
        c.prev = c.phi;
        flag = 1;
      } else if (over) {
        c.dphi *= 0.5;
        scale = sqrt((c.prev + c.dphi) / c.prev);
        flag = 2;
      }
      if (c.dphi < a.min_dphi) c.state = 3;
    }
  }
  a.flag[s] = flag;
  a.scale[s] = c.state != 0 ? 1.0 : scale;
}

// Packing fraction of every system after the step (the host loop's order:
// tile numerators summed one after the other), the step limit, and the
// outer loop's condition.
__global__ void k_cstep_end(const __grid_constant__ CompArgs a, int count_step) {
  __shared__ int s_any;
  if (threadIdx.x == 0) s_any = 0;
  __syncthreads();
  if (!a.st->abort) {
    for (int s = threadIdx.x; s < a.S; s += blockDim.x) {
      CompSys& c = a.comp[s];
      if (count_step) {
        const BatchSys& bs = a.bsys[s];
        double x = 0.0;
        for (int t = bs.tile_begin; t < bs.tile_end; t++) x += a.partials[t];
        c.phi = x / (bs.box.lx * bs.box.ly);
        if (c.state == 0 && c.steps >= a.max_steps) c.state = 2;
      }
      if (c.state == 0) s_any = 1;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0)
    cudaGraphSetConditional(a.outer, (s_any && a.max_steps > 0 && !a.st->abort) ? 1u : 0u);
}

__global__ void k_copy2(int n, const double2* src, double2* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

// ------------------------------------------------------------------ host helpers

template <typename T>
int dalloc(cr_batch* b, T** p, size_t n) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return b->fail(CR_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(*p, 0, n * sizeof(T));
  if (e != cudaSuccess) return b->fail(CR_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  return CR_OK;
}

int upload(cr_batch* b, void* dst, const void* src, size_t bytes) {
  BT_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->stream));
  BT_TRY(cudaStreamSynchronize(b->stream));
  return CR_OK;
}

int download(cr_batch* b, void* dst, const void* src, size_t bytes) {
  BT_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, b->stream));
  BT_TRY(cudaStreamSynchronize(b->stream));
  return CR_OK;
}

void drop_graphs(cr_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  if (b->comp_exec) cudaGraphExecDestroy(b->comp_exec);
  b->comp_exec = nullptr;
  if (b->pchunk) cudaGraphExecDestroy(b->pchunk);
  b->pchunk = nullptr;
}

int read_status(cr_batch* b) { return download(b, b->status_h, b->status, sizeof(DevStatus)); }

int write_status(cr_batch* b) { return upload(b, b->status, b->status_h, sizeof(DevStatus)); }

int pull_sys(cr_batch* b) { return download(b, b->bsys_h.data(), b->bsys, b->S * sizeof(BatchSys)); }

int push_sys(cr_batch* b) { return upload(b, b->bsys, b->bsys_h.data(), b->S * sizeof(BatchSys)); }

int inter_kind(const cr_batch* b) {
  return (b->interaction == CR_INTERACTION_VERTEX_VERTEX || b->interaction == CR_INTERACTION_ALL) ? INT_VV
                                                                                                  : INT_SMOOTH;
}

// vertices a batch tile of this shape holds (0: unsupported shape)
int tile_capacity(int lanes, int block = 0) {
  const int bl = batch_tile_block(lanes, block);
  return bl ? bl / lanes : 0;
}

// Tiles of whole rings that never cross a system.
void make_tiles(cr_batch* b) {
  const int tv = tile_capacity(b->lanes, b->block);
  b->tiles_h.clear();
  for (int s = 0; s < b->S; s++) {
    b->bsys_h[s].tile_begin = (int)b->tiles_h.size();
    int r = b->sys_r0[s];
    const int r_end = b->sys_r0[s] + b->sys_np[s];
    while (r < r_end) {
      int r1 = r, cnt = 0;
      while (r1 < r_end && cnt + b->ring_nv_h[r1] <= tv) cnt += b->ring_nv_h[r1++];
      b->tiles_h.push_back(make_int4(s, r, b->ring_first_h[r], b->ring_first_h[r] + cnt));
      r = r1;
    }
    b->bsys_h[s].tile_end = (int)b->tiles_h.size();
  }
}

int upload_tiles(cr_batch* b) {
  int rc;
  if ((rc = dalloc(b, &b->tiles, b->tiles_h.size()))) return rc;
  if ((rc = upload(b, b->tiles, b->tiles_h.data(), b->tiles_h.size() * sizeof(int4)))) return rc;
  const int need = (int)b->tiles_h.size() * NSUM;
  if (need > b->partials_n) {
    if ((rc = dalloc(b, &b->partials, need))) return rc;
    b->partials_n = need;
  }
  return CR_OK;
}

void refresh_params(cr_batch* b) {
  b->p.nv = b->nv;
  b->p.np = b->np;
  b->p.lx = b->p.ly = 1.0;
  b->p.inv_lx = b->p.inv_ly = 1.0;
  b->p.monomer = 0;
  b->p.potential = b->potential;
}

// DPM2D::setDisplacementCutoff (src/DPM2D.cu:1300-1329) for the potential.
double cut_distance_of(const cr_batch* b, double cutoff_) {
  switch (b->potential) {
    case CR_POTENTIAL_LENNARD_JONES: return b->p.lj_cutoff + cutoff_;
    case CR_POTENTIAL_WCA: return kWCAcut + cutoff_;
    case CR_POTENTIAL_ADHESIVE: return 1.0 + b->p.l2 + cutoff_;
    default: return 1.0 + cutoff_;
  }
}

// Cell grid of every system for the current boxes, radii and cutDistance.
int setup_grids(cr_batch* b) {
  b->sgrid_h.assign(b->S, make_int4(1, 1, 0, 0));
  int total = 0;
  for (int s = 0; s < b->S; s++) {
    const double cmin = (1.0 + b->cut_distance) * 2.0 * b->rmax_h[s] * (1.0 + 1e-9);
    int ncx = cmin > 0 ? (int)std::floor(b->box_h[s].lx / cmin) : 1;
    int ncy = cmin > 0 ? (int)std::floor(b->box_h[s].ly / cmin) : 1;
    ncx = std::min(ncx, 4096);
    ncy = std::min(ncy, 4096);
    if (ncx < 3 || ncy < 3) ncx = ncy = 1;
    b->sgrid_h[s] = make_int4(ncx, ncy, total, 0);
    total += ncx * ncy;
  }
  b->ncells = total;
  int rc;
  if (total > b->ncells_alloc) {
    drop_graphs(b);
    if ((rc = dalloc(b, &b->cell_cnt, total))) return rc;
    if ((rc = dalloc(b, &b->cell_start, total + 1))) return rc;
    b->ncells_alloc = total;
  }
  return upload(b, b->sgrid, b->sgrid_h.data(), b->S * sizeof(int4));
}

BNbr nbr_args(cr_batch* b, int all) {
  BNbr n;
  n.pos = b->pos;
  n.rad = b->rad;
  n.ring_of = b->ring_of;
  n.vsys = b->vsys;
  n.pq_pack = b->pq_pack;
  n.nbr = b->nbr;
  n.nbr_pq = b->nbr_pq;
  n.nbr_cnt = b->nbr_cnt;
  n.cap = b->cap;
  n.nv = b->nv;
  n.cut_distance = b->cut_distance;
  n.last_pos = b->last_pos;
  n.cell_of = b->cell_of;
  n.slot = b->slot;
  n.cell_cnt = b->cell_cnt;
  n.cell_start = b->cell_start;
  n.cell_vid = b->cell_vid;
  n.cell_pos = b->cell_pos;
  n.cell_rad = b->cell_rad;
  n.cell_ring = b->cell_ring;
  n.cell_pq = b->cell_pq;
  n.sgrid = b->sgrid;
  n.bsys = b->bsys;
  n.status = b->status;
  n.S = b->S;
  n.all = all;
  return n;
}

// The batched build as stream-ordered launches (capturable).
void enqueue_build(cr_batch* b, cudaStream_t st, int all) {
  const BNbr n = nbr_args(b, all);
  const int nb = (b->nv + 255) / 256;
  k_bguard<<<1, 32, 0, st>>>(b->status);
  k_bcell_count<<<nb, 256, 0, st>>>(n);
  launch_cell_scan(st, b->ncells, b->cell_cnt, b->cell_start);
  k_bcell_fill<<<nb, 256, 0, st>>>(n);
  NbrArgs na{};
  na.pos = b->pos;
  na.rad = b->rad;
  na.ring_of = b->ring_of;
  na.cell_start = b->cell_start;
  na.cell_vid = b->cell_vid;
  na.cell_pos = b->cell_pos;
  na.cell_rad = b->cell_rad;
  na.cell_ring = b->cell_ring;
  na.pq_pack = b->pq_pack;
  na.nbr_pq = b->nbr_pq;
  na.cell_pq = b->cell_pq;
  launch_cell_sort(st, b->ncells, b->nv, na);
  k_bnbr<<<nb, 256, 0, st>>>(n);
  b->launches += 7;
}

int alloc_lists(cr_batch* b, int cap) {
  int rc;
  if ((rc = dalloc(b, &b->nbr, (size_t)cap * b->nv))) return rc;
  if ((rc = dalloc(b, &b->nbr_pq, (size_t)cap * b->nv))) return rc;
  b->cap = cap;
  drop_graphs(b);
  return CR_OK;
}

long long pow2ceil(long long x) {
  long long r = 1;
  while (r < x) r <<= 1;
  return r;
}

int clear_flags(cr_batch* b) {
  int rc;
  if ((rc = read_status(b))) return rc;
  b->status_h->abort = 0;
  b->status_h->overflow = 0;
  b->status_h->rebuild = 0;
  b->status_h->nonfinite = 0;
  b->status_h->converged = 0;
  b->status_h->done_ctr = 0;
  b->status_h->pbar = 0;
  b->status_h->bpending = 0;
  b->status_h->stalled = 0;
  return write_status(b);
}

// Builds the lists of every active system, growing the capacity (with
// headroom for rebuilds inside FIRE chunks) until they fit.
int build_all(cr_batch* b) {
  int rc;
  if ((rc = setup_grids(b))) return rc;
  for (int pass = 0; pass < 4; pass++) {
    if ((rc = clear_flags(b))) return rc;
    enqueue_build(b, b->stream, 1);
    BT_TRY(cudaGetLastError());
    if ((rc = read_status(b))) return rc;
    const int mc = b->status_h->max_count;
    if (!b->status_h->overflow && 2LL * mc <= b->cap) {
      b->nbr_built = true;
      return clear_flags(b);
    }
    if ((rc = alloc_lists(b, (int)std::max<long long>(16, pow2ceil(2LL * mc))))) return rc;
  }
  return b->fail(CR_ENBR_OVERFLOW, "batched neighbour lists did not fit after growing");
}

SysArrays arrays(cr_batch* b) {
  SysArrays a{};
  a.pos = b->pos;
  a.rad = b->rad;
  a.l0 = b->l0;
  a.theta0 = b->theta0;
  a.a0 = b->a0;
  a.ring_of = b->ring_of;
  a.nbr = b->nbr;
  a.nbr_cnt = b->nbr_cnt;
  a.tiles = b->tiles;
  a.nbr_cap = b->cap;
  a.vtopo = b->vtopo;
  a.nbr_pq = b->nbr_pq;
  return a;
}

StepArgs step_args(cr_batch* b) {
  StepArgs s;
  std::memset(&s, 0, sizeof(s));
  s.pos_out = b->pos;
  s.vel = b->vel;
  s.force = b->force;
  s.last_pos = b->last_pos;
  s.energy = b->energy;
  s.p_energy = b->p_energy;
  s.theta_out = b->theta;
  s.length_out = b->length;
  s.area_out = b->area;
  s.perim_out = b->perimeter;
  s.ppos_out = b->ppos;
  s.partials = b->partials;
  s.status = b->status;
  s.bsys = b->bsys;
  s.bfire_state = b->bfire;
  s.fire_tol = -1.0;
  return s;
}

LaunchCfg tile_cfg(cr_batch* b, cudaStream_t st) {
  LaunchCfg c{st, (int)b->tiles_h.size(), b->lanes, b->precision};
  c.block = b->block;
  return c;
}

int force_all(cr_batch* b, cudaStream_t st = nullptr) {
  StepArgs s = step_args(b);
  s.kind = KIND_NONE;
  s.write_out = 1;
  launch_tile_batch(tile_cfg(b, st ? st : b->stream), b->potential, inter_kind(b), MODE_FORCE, b->p, arrays(b), s);
  b->launches++;
  BT_TRY(cudaGetLastError());
  return CR_OK;
}

int reduce_sys(cr_batch* b, int set_converged, cudaStream_t st = nullptr) {
  k_btile_reduce<128><<<(int)b->tiles_h.size(), 128, 0, st ? st : b->stream>>>(
      b->tiles, b->vel, b->force, b->energy, b->p_energy, b->vtopo, inter_kind(b) == INT_SMOOTH, b->bsys,
      b->partials, set_converged);
  b->launches++;
  BT_TRY(cudaGetLastError());
  return CR_OK;
}

// One FIRE iteration over every unconverged system: pre-kick (with the
// displacement check), conditional rebuild of the flagged systems, force +
// second kick with per-system sums and convergence.
BFire bfire_args(cr_batch* b, bool use_cond, cudaGraphConditionalHandle h) {
  BFire f;
  f.pos = b->pos;
  f.vel = b->vel;
  f.force = b->force;
  f.last_pos = b->last_pos;
  f.vsys = b->vsys;
  f.sys_v0 = b->sys_v0_d;
  f.bsys = b->bsys;
  f.bfire = b->bfire;
  f.fp = b->fp;
  f.st = b->status;
  f.nv = b->nv;
  f.use_cond = use_cond ? 1 : 0;
  f.cond = h;
  return f;
}

void enqueue_fire_iteration(cr_batch* b, cudaStream_t st, bool use_cond, cudaGraphConditionalHandle h) {
  BFire f;
  f.pos = b->pos;
  f.vel = b->vel;
  f.force = b->force;
  f.last_pos = b->last_pos;
  f.vsys = b->vsys;
  f.sys_v0 = b->sys_v0_d;
  f.bsys = b->bsys;
  f.bfire = b->bfire;
  f.fp = b->fp;
  f.st = b->status;
  f.nv = b->nv;
  f.use_cond = use_cond ? 1 : 0;
  f.cond = h;
  k_bfire_pre<<<(b->nv + 255) / 256, 256, 0, st>>>(f);
  b->launches++;
}

void enqueue_fire_tile(cr_batch* b, cudaStream_t st) {
  StepArgs s = step_args(b);
  s.kind = KIND_FIRE;
  s.advance = 0;
  s.accumulate = 1;
  s.write_out = 1;
  launch_tile_batch(tile_cfg(b, st), b->potential, inter_kind(b), MODE_STEP, b->p, arrays(b), s);
  b->launches++;
}

// n FIRE iterations onto stream st, which is capturing into graph g: each
// iteration's rebuild is a conditional node whose body is captured on side.
int add_fire_iterations(cr_batch* b, cudaStream_t st, cudaStream_t side, cudaGraph_t g, long n) {
  for (long i = 0; i < n; i++) {
    cudaGraphConditionalHandle h = 0;
    BT_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    enqueue_fire_iteration(b, st, true, h);
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    BT_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    BT_TRY(cudaGraphAddNode(&node, cg, deps, ndeps, &cp));
    BT_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BT_TRY(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_build(b, side, 0);
    cudaGraph_t body_out;
    BT_TRY(cudaStreamEndCapture(side, &body_out));
    enqueue_fire_tile(b, st);
  }
  return CR_OK;
}

// The persistent FIRE kernel of the batch's configuration, when it has one
// and the GPU holds all of its CTAs at once; *block its CTA size.
BFireStepsFn persist_fn(cr_batch* b, int* block) {
  if (b->no_persist || b->precision != CR_PRECISION_FP64) return nullptr;
  const int bl = batch_tile_block(b->lanes, b->block);
  BFireStepsFn fn = bfire_steps_fn(b->potential, inter_kind(b), b->lanes, bl);
  if (!fn) return nullptr;
  auto it = b->persist_max.find(fn);
  if (it == b->persist_max.end()) it = b->persist_max.emplace(fn, bfire_steps_max_blocks(fn, bl)).first;
  if ((int)b->tiles_h.size() > it->second) return nullptr;
  *block = bl;
  return fn;
}

// FIRE iterations with the persistent kernel onto stream st (capturing into
// graph g): `launches` launches of up to 64 iterations, each followed by a
// conditional rebuild (body captured on side) that runs when the launch
// left with a system's displacement check fired, then one launch that only
// completes a force op left pending, so the chunk ends on a whole iteration.
int add_fire_persistent(cr_batch* b, cudaStream_t st, cudaStream_t side, cudaGraph_t g, int launches,
                        BFireStepsFn fn, int block) {
  StepArgs s = step_args(b);
  s.kind = KIND_FIRE;
  s.advance = 0;
  s.accumulate = 1;
  s.write_out = 1;
  s.use_cond = 0;
  const SysParams p = with_f32_constants(b->p);
  for (int i = 0; i < launches; i++) {
    cudaGraphConditionalHandle h = 0;
    BT_TRY(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    launch_bfire_steps(fn, tile_cfg(b, st), block, p, arrays(b), s, bfire_args(b, true, h), 64);
    b->launches++;
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    BT_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    BT_TRY(cudaGraphAddNode(&node, cg, deps, ndeps, &cp));
    BT_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    BT_TRY(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_build(b, side, 0);
    cudaGraph_t body_out;
    BT_TRY(cudaStreamEndCapture(side, &body_out));
  }
  launch_bfire_steps(fn, tile_cfg(b, st), block, p, arrays(b), s, bfire_args(b, false, 0), 0);
  b->launches++;
  BT_TRY(cudaGetLastError());
  return CR_OK;
}

int capture_fire_persistent(cr_batch* b, BFireStepsFn fn, int block, cudaGraphExec_t* out) {
  cudaGraph_t graph;
  BT_TRY(cudaGraphCreate(&graph, 0));
  BT_TRY(cudaStreamBeginCaptureToGraph(b->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const int rc = add_fire_persistent(b, b->stream, b->side, graph, 4, fn, block);
  cudaGraph_t g;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    cudaGraphDestroy(graph);
    return rc;
  }
  BT_TRY(e);
  BT_TRY(cudaGraphInstantiate(out, g, 0));
  cudaGraphDestroy(g);
  return CR_OK;
}

int capture_fire_chunk(cr_batch* b, long n, cudaGraphExec_t* out) {
  cudaGraph_t graph;
  BT_TRY(cudaGraphCreate(&graph, 0));
  BT_TRY(cudaStreamBeginCaptureToGraph(b->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const int rc = add_fire_iterations(b, b->stream, b->side, graph, n);
  cudaGraph_t g;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    cudaGraphDestroy(graph);
    return rc;
  }
  BT_TRY(e);
  BT_TRY(cudaGraphInstantiate(out, g, 0));
  cudaGraphDestroy(g);
  return CR_OK;
}

int snapshot(cr_batch* b, bool restore) {
  const size_t v2 = (size_t)b->nv * sizeof(double2);
  const size_t sb = (size_t)b->S * sizeof(BatchSys), fb = (size_t)b->S * 8 * sizeof(double);
  if (!restore) {
    BT_TRY(cudaMemcpyAsync(b->snap_pos, b->pos, v2, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->snap_vel, b->vel, v2, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->snap_bsys, b->bsys, sb, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->snap_bfire, b->bfire, fb, cudaMemcpyDeviceToDevice, b->stream));
  } else {
    BT_TRY(cudaMemcpyAsync(b->pos, b->snap_pos, v2, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->vel, b->snap_vel, v2, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->bsys, b->snap_bsys, sb, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->bfire, b->snap_bfire, fb, cudaMemcpyDeviceToDevice, b->stream));
  }
  return CR_OK;
}

// Forces, per-system sums and convergence of the current state (the start
// of a FIRE run): lists rebuilt for every active system first.
int fire_prologue(cr_batch* b) {
  int rc;
  if ((rc = build_all(b))) return rc;
  if ((rc = force_all(b))) return rc;
  if ((rc = reduce_sys(b, 1))) return rc;
  BT_TRY(cudaStreamSynchronize(b->stream));
  return CR_OK;
}

// FIRE iterations in chunks of graphs until every active system converged
// or maxIter iterations ran.  A list overflow inside a chunk restores the
// chunk's starting state, grows the lists and runs the chunk again.
int fire_loop(cr_batch* b, long maxIter, long* done_out) {
  int rc;
  long done = 0;
  const long chunk = 64;
  if (maxIter <= 0) {
    if (done_out) *done_out = 0;
    return CR_OK;
  }
  // persistent FIRE: chunks of up to 4 x 64 iterations; every system stops at
  // its iteration limit (fire_cap, set by the caller), so the loop ends when
  // every system has converged or reached it
  int block = 0;
  while (BFireStepsFn fn = persist_fn(b, &block)) {
    if ((rc = pull_sys(b))) return rc;
    bool any = false;
    for (const BatchSys& s : b->bsys_h) any = any || (s.active && !s.converged);
    if (!any) {
      if (done_out) *done_out = maxIter;
      return CR_OK;
    }
    if ((rc = snapshot(b, false))) return rc;
    if (!b->pchunk && (rc = capture_fire_persistent(b, fn, block, &b->pchunk))) return rc;
    BT_TRY(cudaGraphLaunch(b->pchunk, b->stream));
    if ((rc = read_status(b))) return rc;
    if (b->status_h->abort) {
      if (b->status_h->nonfinite) return b->fail(CR_ENONFINITE, "non-finite force in a batched FIRE run");
      if ((rc = snapshot(b, true))) return rc;
      if (b->status_h->stalled) {
        // a grid-barrier wait gave up: one launch per op from here on
        b->no_persist = true;
        drop_graphs(b);
      } else if (b->status_h->overflow) {
        if ((rc = alloc_lists(b, (int)pow2ceil(2LL * b->status_h->max_count)))) return rc;
      } else {
        return b->fail(CR_ECUDA, "batched FIRE chunk aborted");
      }
      if ((rc = fire_prologue(b))) return rc;  // same state, fresh lists, sums and flags
    }
  }
  while (done < maxIter) {
    if ((rc = pull_sys(b))) return rc;
    bool any = false;
    for (const BatchSys& s : b->bsys_h) any = any || (s.active && !s.converged);
    if (!any) break;
    const long n = std::min(chunk, maxIter - done);
    if ((rc = snapshot(b, false))) return rc;
    auto key = std::make_pair(n, b->cap);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraphExec_t ge;
      if ((rc = capture_fire_chunk(b, n, &ge))) return rc;
      it = b->graphs.emplace(key, ge).first;
    }
    BT_TRY(cudaGraphLaunch(it->second, b->stream));
    b->launches += 2 * n;
    if ((rc = read_status(b))) return rc;
    if (b->status_h->abort) {
      if (b->status_h->nonfinite) return b->fail(CR_ENONFINITE, "non-finite force in a batched FIRE run");
      if (!b->status_h->overflow) return b->fail(CR_ECUDA, "batched FIRE chunk aborted");
      if ((rc = snapshot(b, true))) return rc;
      if ((rc = alloc_lists(b, (int)pow2ceil(2LL * b->status_h->max_count)))) return rc;
      if ((rc = fire_prologue(b))) return rc;  // same state, fresh lists and sums
      continue;
    }
    done += n;
  }
  if (done_out) *done_out = done;
  return CR_OK;
}

int set_vertex_array(cr_batch* b, double* dst, const double* src, size_t n) {
  if (!b || !src) return CR_EINVAL;
  return upload(b, dst, src, n * sizeof(double));
}

void compute_radius_stats(cr_batch* b, const double* rad_h) {
  for (int s = 0; s < b->S; s++) {
    double m = 0.0, sum = 0.0;
    for (int v = b->sys_v0[s]; v < b->sys_v0[s] + b->sys_nv[s]; v++) {
      m = std::max(m, rad_h[v]);
      sum += rad_h[v];
    }
    b->rmax_h[s] = m;
    b->rmean_h[s] = sum / b->sys_nv[s];
  }
}

int refresh_radius_stats(cr_batch* b) {
  std::vector<double> r(b->nv);
  int rc = download(b, r.data(), b->rad, (size_t)b->nv * sizeof(double));
  if (rc) return rc;
  compute_radius_stats(b, r.data());
  return CR_OK;
}

// Per-system displacement cutoff cutoff_ * size_ with size_ = 2 <r> of the
// system (the reference drivers' choice, runNVE.cpp:129-130).
int apply_cutoffs(cr_batch* b) {
  int rc;
  if ((rc = pull_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) b->bsys_h[s].disp_cutoff = b->cutoff_ * 2.0 * b->rmean_h[s];
  b->cut_distance = cut_distance_of(b, b->cutoff_);
  return push_sys(b);
}

int phis(cr_batch* b, const double* ring_area, double* out) {
  k_btile_phi<128><<<(int)b->tiles_h.size(), 128, 0, b->stream>>>(b->tiles, b->vtopo, ring_area, b->rad,
                                                                     b->partials);
  b->launches++;
  BT_TRY(cudaGetLastError());
  std::vector<double> part(b->tiles_h.size());
  int rc = download(b, part.data(), b->partials, part.size() * sizeof(double));
  if (rc) return rc;
  for (int s = 0; s < b->S; s++) {
    double x = 0.0;
    for (int t = b->bsys_h[s].tile_begin; t < b->bsys_h[s].tile_end; t++) x += part[t];
    out[s] = x / (b->box_h[s].lx * b->box_h[s].ly);
  }
  return CR_OK;
}

int mean_particle_sizes(cr_batch* b, double* out) {
  std::vector<double> a(b->np);
  int rc = download(b, a.data(), b->a0, (size_t)b->np * sizeof(double));
  if (rc) return rc;
  for (int s = 0; s < b->S; s++) {
    double sum = 0.0;
    for (int q = b->sys_r0[s]; q < b->sys_r0[s] + b->sys_np[s]; q++) sum += a[q];
    out[s] = 2 * std::sqrt(sum / (kPi * b->sys_np[s]));  // DPM2D::getMeanParticleSize, src/DPM2D.cu:781-783
  }
  return CR_OK;
}


// The device compression loop as one graph (see k_cstep_begin): an outer
// WHILE node over compression steps, and inside it a WHILE node over chunks
// of 64 FIRE iterations.  The loop bodies are captured on their own streams
// while the enclosing capture is open.
int add_while(cr_batch* b, cudaStream_t st, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  BT_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &ndeps));
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  BT_TRY(cudaGraphAddNode(&node, cg, deps, ndeps, &cp));
  BT_TRY(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  *body = cp.conditional.phGraph_out[0];
  return CR_OK;
}

int compress_body(cr_batch* b, CompArgs a, cudaGraph_t outer_body) {
  cudaStream_t s2 = b->cap_s2, s3 = b->cap_s3;
  BT_TRY(cudaGraphConditionalHandleCreate(&a.inner, outer_body, 0, cudaGraphCondAssignDefault));
  const int nb = (b->nv + 255) / 256, sb = (b->S + 127) / 128;
  // the step's starting positions and velocities, for a rerun after a list overflow
  k_copy2<<<nb, 256, 0, s2>>>(b->nv, b->pos, b->snap_pos);
  k_copy2<<<nb, 256, 0, s2>>>(b->nv, b->vel, b->snap_vel);
  k_cstep_begin<<<sb, 128, 0, s2>>>(a);
  k_cclear<<<1, 1, 0, s2>>>(b->status);
  enqueue_build(b, s2, 1);
  int rc;
  if ((rc = force_all(b, s2)) || (rc = reduce_sys(b, 1, s2))) return rc;
  k_cfire_more<<<1, 256, 0, s2>>>(a);
  cudaGraph_t inner_body;
  if ((rc = add_while(b, s2, a.inner, &inner_body))) return rc;
  BT_TRY(cudaStreamBeginCaptureToGraph(s3, inner_body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int block = 0;
  if (BFireStepsFn fn = persist_fn(b, &block)) rc = add_fire_persistent(b, s3, b->side, inner_body, 4, fn, block);
  else rc = add_fire_iterations(b, s3, b->side, inner_body, 64);
  if (!rc) k_cfire_more<<<1, 256, 0, s3>>>(a);
  cudaGraph_t ib_out;
  const cudaError_t e = cudaStreamEndCapture(s3, &ib_out);
  if (rc) return rc;
  BT_TRY(e);
  if ((rc = reduce_sys(b, 0, s2))) return rc;
  k_cdecide<<<sb, 128, 0, s2>>>(a);
  const int n = std::max(b->nv, b->np);
  k_bsave<<<(n + 255) / 256, 256, 0, s2>>>(b->nv, b->np, b->vsys, b->ring_sys, b->sys_flag, b->pos, b->rad, b->l0,
                                           b->a0, b->save_pos, b->save_rad, b->save_l0, b->save_a0);
  if ((rc = force_all(b, s2))) return rc;  // ring centroids of the (restored) positions
  k_bscale<<<(n + 255) / 256, 256, 0, s2>>>(b->nv, b->np, b->vsys, b->ring_sys, b->ring_of, b->ppos, b->sys_scalar,
                                            b->pos, b->l0, b->rad, b->a0, b->area);
  if ((rc = force_all(b, s2))) return rc;  // ring areas of the scaled rings
  k_btile_phi<128><<<(int)b->tiles_h.size(), 128, 0, s2>>>(b->tiles, b->vtopo, b->area, b->rad, b->partials);
  k_cstep_end<<<1, 256, 0, s2>>>(a, 1);
  BT_TRY(cudaGetLastError());
  return CR_OK;
}

int capture_compress(cr_batch* b, CompArgs a, cudaGraphExec_t* out) {
  if (!b->cap_s2) BT_TRY(cudaStreamCreateWithFlags(&b->cap_s2, cudaStreamNonBlocking));
  if (!b->cap_s3) BT_TRY(cudaStreamCreateWithFlags(&b->cap_s3, cudaStreamNonBlocking));
  cudaGraph_t graph;
  BT_TRY(cudaGraphCreate(&graph, 0));
  BT_TRY(cudaGraphConditionalHandleCreate(&a.outer, graph, 0, cudaGraphCondAssignDefault));
  BT_TRY(cudaStreamBeginCaptureToGraph(b->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  k_cstep_end<<<1, 256, 0, b->stream>>>(a, 0);
  cudaGraph_t outer_body;
  int rc = add_while(b, b->stream, a.outer, &outer_body);
  if (!rc) {
    const cudaError_t e2 = cudaStreamBeginCaptureToGraph(b->cap_s2, outer_body, nullptr, nullptr, 0,
                                                         cudaStreamCaptureModeThreadLocal);
    if (e2 != cudaSuccess) {
      rc = b->fail(CR_ECUDA, std::string("capture of the compression step: ") + cudaGetErrorString(e2));
    } else {
      rc = compress_body(b, a, outer_body);
      cudaGraph_t ob_out;
      const cudaError_t e3 = cudaStreamEndCapture(b->cap_s2, &ob_out);
      if (!rc && e3 != cudaSuccess) rc = b->fail(CR_ECUDA, std::string("capture: ") + cudaGetErrorString(e3));
    }
  }
  cudaGraph_t g;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    cudaGraphDestroy(graph);
    return rc;
  }
  BT_TRY(e);
  BT_TRY(cudaGraphInstantiate(out, g, 0));
  cudaGraphDestroy(g);
  return CR_OK;
}

// cr_batch_compress: the protocol of compress_host with every step on the
// device, one graph launch for the whole run.  A list overflow stops the
// graph; the host restores the step's starting positions and velocities,
// grows the lists and launches the loop again from that step.  A system's
// FIRE run stops after max_fire_iters iterations exactly, as in the host loop.
int compress_device(cr_batch* b, const cr_compress_params* prm, double* phiOut, long* stepsOut, int* stateOut,
                    long* fireItersOut) {
  const int S = b->S;
  int rc;
  if (!b->nbr_built && (rc = cr_batch_calc_neighbor_lists(b))) return rc;
  if (!b->comp) {
    if ((rc = dalloc(b, &b->comp, S)) || (rc = dalloc(b, &b->sys_nv_d, S)) || (rc = dalloc(b, &b->sys_r0_d, S)) ||
        (rc = dalloc(b, &b->sys_np_d, S)) || (rc = dalloc(b, &b->cells0_d, S)))
      return rc;
    if ((rc = upload(b, b->sys_nv_d, b->sys_nv.data(), S * sizeof(int))) ||
        (rc = upload(b, b->sys_r0_d, b->sys_r0.data(), S * sizeof(int))) ||
        (rc = upload(b, b->sys_np_d, b->sys_np.data(), S * sizeof(int))))
      return rc;
  }
  // every system's share of the cell arrays: its grid for the starting radii
  if ((rc = refresh_radius_stats(b)) || (rc = apply_cutoffs(b)) || (rc = setup_grids(b))) return rc;
  std::vector<int> cells0(S);
  for (int s = 0; s < S; s++) cells0[s] = b->sgrid_h[s].x * b->sgrid_h[s].y;
  if ((rc = upload(b, b->cells0_d, cells0.data(), S * sizeof(int)))) return rc;
  // starting packing fractions; the starting configuration is the first saved state
  std::vector<double> phi(S);
  if ((rc = force_all(b)) || (rc = pull_sys(b)) || (rc = phis(b, b->area, phi.data()))) return rc;
  std::vector<int> flag(S, 1);
  if ((rc = upload(b, b->sys_flag, flag.data(), S * sizeof(int)))) return rc;
  const int n = std::max(b->nv, b->np);
  k_bsave<<<(n + 255) / 256, 256, 0, b->stream>>>(b->nv, b->np, b->vsys, b->ring_sys, b->sys_flag, b->pos, b->rad,
                                                  b->l0, b->a0, b->save_pos, b->save_rad, b->save_l0, b->save_a0);
  b->launches++;
  BT_TRY(cudaGetLastError());
  std::vector<CompSys> comp(S);
  for (int s = 0; s < S; s++) comp[s] = CompSys{phi[s], phi[s], prm->dphi, 0, 0, 0, 0};
  if ((rc = upload(b, b->comp, comp.data(), S * sizeof(CompSys)))) return rc;
  // FIRE parameters of compressFIRE.cpp:106 ({a_start, f_dec, f_inc, f_a, dt,
  // 10 dt, a}, minStep 20); each step's per-system dt comes from k_cstep_begin
  b->fp.a_start = 0.2;
  b->fp.f_dec = 0.5;
  b->fp.f_inc = 1.1;
  b->fp.f_a = 0.99;
  b->fp.dt_max = 10 * prm->fire_dt;
  b->fp.min_step = 20;
  b->fp.tol = -1.0;
  b->fire_ready = true;
  CompArgs a{};
  a.comp = b->comp;
  a.bsys = b->bsys;
  a.bfire = b->bfire;
  a.sgrid = b->sgrid;
  a.cells0 = b->cells0_d;
  a.rad = b->rad;
  a.a0 = b->a0;
  a.sys_v0 = b->sys_v0_d;
  a.sys_nv = b->sys_nv_d;
  a.sys_r0 = b->sys_r0_d;
  a.sys_np = b->sys_np_d;
  a.partials = b->partials;
  a.scale = b->sys_scalar;
  a.flag = b->sys_flag;
  a.st = b->status;
  a.S = S;
  a.cutoff_ = b->cutoff_;
  a.cut_distance = b->cut_distance;
  a.dphi0 = prm->dphi;
  a.min_dphi = prm->min_dphi;
  a.fire_dt = prm->fire_dt;
  a.tol0 = prm->tol0;
  a.energy_tol = prm->energy_tol;
  a.max_fire_iters = prm->max_fire_iters;
  a.max_steps = prm->max_steps;
  a.criterion = prm->criterion;
  if ((rc = clear_flags(b))) return rc;
  for (int attempt = 0;; attempt++) {
    drop_graphs(b);
    if ((rc = capture_compress(b, a, &b->comp_exec))) return rc;
    BT_TRY(cudaGraphLaunch(b->comp_exec, b->stream));
    if ((rc = read_status(b))) return rc;
    if (!b->status_h->abort) break;
    if (b->status_h->nonfinite) return b->fail(CR_ENONFINITE, "non-finite force in a batched compression");
    if ((!b->status_h->overflow && !b->status_h->stalled) || attempt >= 8)
      return b->fail(CR_ECUDA, "batched compression aborted");
    const size_t v2 = (size_t)b->nv * sizeof(double2);
    BT_TRY(cudaMemcpyAsync(b->pos, b->snap_pos, v2, cudaMemcpyDeviceToDevice, b->stream));
    BT_TRY(cudaMemcpyAsync(b->vel, b->snap_vel, v2, cudaMemcpyDeviceToDevice, b->stream));
    if (b->status_h->stalled) b->no_persist = true;  // a grid-barrier wait gave up: one launch per op
    else if ((rc = alloc_lists(b, (int)pow2ceil(2LL * b->status_h->max_count)))) return rc;
    if ((rc = clear_flags(b))) return rc;
  }
  drop_graphs(b);
  if ((rc = download(b, comp.data(), b->comp, S * sizeof(CompSys)))) return rc;
  long long iters = 0, steps = 0;
  for (int s = 0; s < S; s++) {
    if (phiOut) phiOut[s] = comp[s].phi;
    if (stepsOut) stepsOut[s] = (long)comp[s].steps;
    if (stateOut) stateOut[s] = comp[s].state;
    if (fireItersOut) fireItersOut[s] = (long)comp[s].fire_total;
    iters = std::max(iters, comp[s].fire_total);
    steps = std::max(steps, comp[s].steps);
  }
  b->launches += 2 * iters + 24 * steps;  // FIRE iterations, and the kernels of each step
  // the other entry points see every system active, no iteration limit, and
  // the host-side radius statistics and grids of the final radii
  if ((rc = pull_sys(b))) return rc;
  for (BatchSys& bs : b->bsys_h) {
    bs.active = 1;
    bs.fire_cap = 0;
  }
  if ((rc = push_sys(b))) return rc;
  if ((rc = refresh_radius_stats(b)) || (rc = setup_grids(b))) return rc;
  return CR_OK;
}
}  // namespace

extern "C" {

int cr_batch_create(long numSystems, const long* numParticles, const long* nvList, cr_batch** out) {
  if (!out || numSystems <= 0 || !numParticles || !nvList) return CR_EINVAL;
  *out = nullptr;
  cr_batch* b = new cr_batch();
  cudaGetDevice(&b->device);
  b->S = (int)numSystems;
  long rings = 0, total = 0;
  for (long s = 0; s < numSystems; s++) {
    if (numParticles[s] <= 0) {
      delete b;
      return CR_EINVAL;
    }
    b->sys_r0.push_back((int)rings);
    b->sys_v0.push_back((int)total);
    b->sys_np.push_back((int)numParticles[s]);
    long nvs = 0;
    for (long q = 0; q < numParticles[s]; q++) {
      const long n = nvList[rings + q];
      if (n < 3 || n > 192) {
        delete b;
        return n < 3 ? CR_EINVAL : CR_ENOTSUP;
      }
      b->ring_first_h.push_back((int)(total + nvs));
      b->ring_nv_h.push_back((int)n);
      b->ring_sys_h.push_back((int)s);
      nvs += n;
    }
    b->sys_nv.push_back((int)nvs);
    rings += numParticles[s];
    total += nvs;
  }
  if (total >= (1L << 30)) {
    delete b;
    return CR_EINVAL;
  }
  b->nv = (int)total;
  b->np = (int)rings;
  b->bsys_h.assign(b->S, BatchSys{});
  b->box_h.assign(b->S, Box{1.0, 1.0, 1.0, 1.0});
  b->rmax_h.assign(b->S, 0.0);
  b->rmean_h.assign(b->S, 0.0);
  std::vector<int2> vtopo(total);
  std::vector<int> pqp(total), ring_of(total), vsys(total);
  for (int q = 0; q < b->np; q++) {
    const int f = b->ring_first_h[q], n = b->ring_nv_h[q];
    for (int k = 0; k < n; k++) {
      const int prev = f + (k == 0 ? n - 1 : k - 1);
      const int k2 = (k - 2 + 2 * n) % n;
      vtopo[f + k] = make_int2(q, k | (n << 16));
      pqp[f + k] = pq_pack_of(prev - (f + k), (f + k2) - (f + k));
      ring_of[f + k] = q;
      vsys[f + k] = b->ring_sys_h[q];
    }
  }
  b->vsys_h = vsys;
  for (int s = 0; s < b->S; s++) {
    BatchSys& bs = b->bsys_h[s];
    bs.box = b->box_h[s];
    bs.fire_tol = -1.0;
    bs.active = 1;
  }
  // rings longer than the default tile's 128 vertices take the 192-vertex tile
  for (int n : b->ring_nv_h)
    if (n > 128) b->block = 192;
  make_tiles(b);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return CR_ECUDA;
  }
  const size_t nv = total, np = rings, S = numSystems;
  int rc;
  if ((rc = dalloc(b, &b->pos, nv)) || (rc = dalloc(b, &b->vel, nv)) || (rc = dalloc(b, &b->force, nv)) ||
      (rc = dalloc(b, &b->last_pos, nv)) || (rc = dalloc(b, &b->ppos, np)) || (rc = dalloc(b, &b->rad, nv)) ||
      (rc = dalloc(b, &b->l0, nv)) || (rc = dalloc(b, &b->theta0, nv)) || (rc = dalloc(b, &b->a0, np)) ||
      (rc = dalloc(b, &b->energy, nv)) || (rc = dalloc(b, &b->p_energy, np)) || (rc = dalloc(b, &b->theta, nv)) ||
      (rc = dalloc(b, &b->length, nv)) || (rc = dalloc(b, &b->area, np)) || (rc = dalloc(b, &b->perimeter, np)) ||
      (rc = dalloc(b, &b->vtopo, nv)) || (rc = dalloc(b, &b->pq_pack, nv)) || (rc = dalloc(b, &b->ring_of, nv)) ||
      (rc = dalloc(b, &b->vsys, nv)) || (rc = dalloc(b, &b->ring_sys, np)) || (rc = dalloc(b, &b->sys_v0_d, S)) ||
      (rc = dalloc(b, &b->nbr_cnt, nv)) || (rc = dalloc(b, &b->cell_of, nv)) || (rc = dalloc(b, &b->slot, nv)) ||
      (rc = dalloc(b, &b->cell_vid, nv)) || (rc = dalloc(b, &b->cell_ring, nv)) ||
      (rc = dalloc(b, &b->cell_pq, nv)) || (rc = dalloc(b, &b->cell_pos, nv)) || (rc = dalloc(b, &b->cell_rad, nv)) ||
      (rc = dalloc(b, &b->sgrid, S)) || (rc = dalloc(b, &b->bsys, S)) || (rc = dalloc(b, &b->bfire, 8 * S)) ||
      (rc = dalloc(b, &b->sys_scalar, S)) || (rc = dalloc(b, &b->sys_flag, S)) || (rc = dalloc(b, &b->status, 1)) ||
      (rc = dalloc(b, &b->snap_pos, nv)) || (rc = dalloc(b, &b->snap_vel, nv)) ||
      (rc = dalloc(b, &b->snap_bsys, S)) || (rc = dalloc(b, &b->snap_bfire, 8 * S)) ||
      (rc = dalloc(b, &b->save_pos, nv)) || (rc = dalloc(b, &b->save_rad, nv)) ||
      (rc = dalloc(b, &b->save_l0, nv)) || (rc = dalloc(b, &b->save_a0, np)) || (rc = alloc_lists(b, 16)) ||
      (rc = upload_tiles(b))) {
    cr_batch_destroy(b);
    return rc;
  }
  if (cudaMallocHost((void**)&b->status_h, sizeof(DevStatus)) != cudaSuccess) {
    cr_batch_destroy(b);
    return CR_ENOMEM;
  }
  std::memset(b->status_h, 0, sizeof(DevStatus));
  if (upload(b, b->vtopo, vtopo.data(), nv * sizeof(int2)) || upload(b, b->pq_pack, pqp.data(), nv * sizeof(int)) ||
      upload(b, b->ring_of, ring_of.data(), nv * sizeof(int)) || upload(b, b->vsys, vsys.data(), nv * sizeof(int)) ||
      upload(b, b->ring_sys, b->ring_sys_h.data(), np * sizeof(int)) ||
      upload(b, b->sys_v0_d, b->sys_v0.data(), S * sizeof(int)) || push_sys(b)) {
    cr_batch_destroy(b);
    return CR_ECUDA;
  }
  // reference defaults (src/DPM2D.cu:41-95)
  b->p.ea = 1e5;
  b->p.el = 20;
  b->p.eb = 10;
  b->p.ec = 1;
  refresh_params(b);
  *out = b;
  return CR_OK;
}

int cr_batch_destroy(cr_batch* b) {
  if (!b) return CR_EINVAL;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graphs(b);
  void* ptrs[] = {b->pos, b->vel, b->force, b->last_pos, b->ppos, b->rad, b->l0, b->theta0, b->a0, b->energy,
                  b->p_energy, b->theta, b->length, b->area, b->perimeter, b->vtopo, b->pq_pack, b->ring_of,
                  b->vsys, b->ring_sys, b->sys_v0_d, b->tiles, b->nbr, b->nbr_pq, b->nbr_cnt, b->cell_of, b->slot,
                  b->cell_cnt, b->cell_start, b->cell_vid, b->cell_ring, b->cell_pq, b->cell_pos, b->cell_rad,
                  b->sgrid, b->bsys, b->bfire, b->partials, b->sys_scalar, b->sys_flag, b->status, b->snap_pos,
                  b->snap_vel, b->snap_bsys, b->snap_bfire, b->save_pos, b->save_rad, b->save_l0, b->save_a0,
                  b->comp, b->sys_nv_d, b->sys_r0_d, b->sys_np_d, b->cells0_d};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (b->status_h) cudaFreeHost(b->status_h);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->cap_s2) cudaStreamDestroy(b->cap_s2);
  if (b->cap_s3) cudaStreamDestroy(b->cap_s3);
  delete b;
  return CR_OK;
}

const char* cr_batch_last_error(const cr_batch* b) { return b ? b->err.c_str() : "null batch"; }

int cr_batch_get_sizes(const cr_batch* b, long* numSystems, long* numParticles, long* numVertices) {
  if (!b) return CR_EINVAL;
  if (numSystems) *numSystems = b->S;
  if (numParticles) *numParticles = b->np;
  if (numVertices) *numVertices = b->nv;
  return CR_OK;
}

int cr_batch_set_potential_type(cr_batch* b, int v) {
  if (!b || v < 0 || v > 3) return CR_EINVAL;
  b->potential = v;
  refresh_params(b);
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_interaction_type(cr_batch* b, int v) {
  if (!b || v < 0 || v > 3) return CR_EINVAL;
  if (v == CR_INTERACTION_CELL_SMOOTH) return b->fail(CR_ENOTSUP, "cellSmooth is not part of the batched path");
  b->interaction = v;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_energy_costs(cr_batch* b, double ea, double el, double eb, double ec) {
  if (!b) return CR_EINVAL;
  b->p.ea = ea;
  b->p.el = el;
  b->p.eb = eb;
  b->p.ec = ec;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_lj_cutoff(cr_batch* b, double c) {
  if (!b || !(c > 0)) return CR_EINVAL;
  // DPM2D::setLJcutoff (src/DPM2D.cu:1923-1932), with ec as it stands
  b->p.lj_cutoff = c;
  const double ratio6 = 1.0 / std::pow(c, 6);
  b->p.lj_ecut = 4 * b->p.ec * (ratio6 * ratio6 - ratio6);
  b->p.lj_fshift = 24 * b->p.ec * (2 * ratio6 - 1) * ratio6 / c;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_attraction_constants(cr_batch* b, double l1, double l2) {
  if (!b) return CR_EINVAL;
  b->p.l1 = l1;
  b->p.l2 = l2;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_precision(cr_batch* b, int precision) {
  if (!b || (precision != CR_PRECISION_FP64 && precision != CR_PRECISION_MIXED)) return CR_EINVAL;
  b->precision = precision;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_set_tile_shape(cr_batch* b, int lanes, int block) {
  if (!b) return CR_EINVAL;
  const int cap = tile_capacity(lanes, block);
  if (!cap) return b->fail(CR_EINVAL, "unsupported tile shape");
  for (int n : b->ring_nv_h)
    if (n > cap) return b->fail(CR_EINVAL, "a ring does not fit the tile of this shape");
  int rc;
  if ((rc = pull_sys(b))) return rc;
  b->lanes = lanes;
  b->block = batch_tile_block(lanes, block);
  make_tiles(b);
  if ((rc = upload_tiles(b))) return rc;
  if ((rc = push_sys(b))) return rc;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_get_tile_shape(const cr_batch* b, int* lanes, int* block) {
  if (!b || !lanes || !block) return CR_EINVAL;
  *lanes = b->lanes;
  *block = batch_tile_block(b->lanes, b->block);
  return CR_OK;
}

int cr_batch_set_lanes(cr_batch* b, int lanes) {
  if (!b || (lanes != 1 && lanes != 2 && lanes != 4)) return CR_EINVAL;
  return cr_batch_set_tile_shape(b, lanes, 0);
}

int cr_batch_get_lanes(const cr_batch* b, int* lanes) {
  if (!b || !lanes) return CR_EINVAL;
  *lanes = b->lanes;
  return CR_OK;
}

int cr_batch_set_box_sizes(cr_batch* b, const double* boxes) {
  if (!b || !boxes) return CR_EINVAL;
  int rc;
  if ((rc = pull_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) {
    const double lx = boxes[2 * s], ly = boxes[2 * s + 1];
    if (!(lx > 0 && ly > 0)) return b->fail(CR_EINVAL, "box sizes must be positive");
    b->box_h[s] = Box{lx, ly, 1.0 / lx, 1.0 / ly};
    b->bsys_h[s].box = b->box_h[s];
  }
  drop_graphs(b);
  return push_sys(b);
}

int cr_batch_get_box_sizes(const cr_batch* b, double* boxes) {
  if (!b || !boxes) return CR_EINVAL;
  for (int s = 0; s < b->S; s++) {
    boxes[2 * s] = b->box_h[s].lx;
    boxes[2 * s + 1] = b->box_h[s].ly;
  }
  return CR_OK;
}

int cr_batch_set_vertex_positions(cr_batch* b, const double* pos) {
  return b ? set_vertex_array(b, reinterpret_cast<double*>(b->pos), pos, 2 * (size_t)b->nv) : CR_EINVAL;
}
int cr_batch_get_vertex_positions(cr_batch* b, double* pos) {
  return (b && pos) ? download(b, pos, b->pos, (size_t)b->nv * sizeof(double2)) : CR_EINVAL;
}
int cr_batch_set_vertex_velocities(cr_batch* b, const double* vel) {
  return b ? set_vertex_array(b, reinterpret_cast<double*>(b->vel), vel, 2 * (size_t)b->nv) : CR_EINVAL;
}
int cr_batch_get_vertex_velocities(cr_batch* b, double* vel) {
  return (b && vel) ? download(b, vel, b->vel, (size_t)b->nv * sizeof(double2)) : CR_EINVAL;
}
int cr_batch_get_vertex_forces(cr_batch* b, double* f) {
  return (b && f) ? download(b, f, b->force, (size_t)b->nv * sizeof(double2)) : CR_EINVAL;
}
int cr_batch_set_vertex_radii(cr_batch* b, const double* rad) {
  if (!b || !rad) return CR_EINVAL;
  compute_radius_stats(b, rad);
  drop_graphs(b);
  return set_vertex_array(b, b->rad, rad, b->nv);
}
int cr_batch_get_vertex_radii(cr_batch* b, double* rad) {
  return (b && rad) ? download(b, rad, b->rad, (size_t)b->nv * sizeof(double)) : CR_EINVAL;
}
int cr_batch_set_rest_areas(cr_batch* b, const double* a0) { return b ? set_vertex_array(b, b->a0, a0, b->np) : CR_EINVAL; }
int cr_batch_get_rest_areas(cr_batch* b, double* a0) {
  return (b && a0) ? download(b, a0, b->a0, (size_t)b->np * sizeof(double)) : CR_EINVAL;
}
int cr_batch_set_rest_lengths(cr_batch* b, const double* l0) { return b ? set_vertex_array(b, b->l0, l0, b->nv) : CR_EINVAL; }
int cr_batch_get_rest_lengths(cr_batch* b, double* l0) {
  return (b && l0) ? download(b, l0, b->l0, (size_t)b->nv * sizeof(double)) : CR_EINVAL;
}
int cr_batch_set_rest_angles(cr_batch* b, const double* t0) {
  return b ? set_vertex_array(b, b->theta0, t0, b->nv) : CR_EINVAL;
}
int cr_batch_get_vertex_energies(cr_batch* b, double* e) {
  return (b && e) ? download(b, e, b->energy, (size_t)b->nv * sizeof(double)) : CR_EINVAL;
}

int cr_batch_set_displacement_cutoff(cr_batch* b, double cutoff_, double* cutDistance) {
  if (!b || !(cutoff_ >= 0)) return CR_EINVAL;
  b->cutoff_ = cutoff_;
  int rc;
  if ((rc = refresh_radius_stats(b))) return rc;
  if ((rc = apply_cutoffs(b))) return rc;
  if (cutDistance) *cutDistance = b->cut_distance;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_calc_neighbor_lists(cr_batch* b) {
  if (!b) return CR_EINVAL;
  int rc;
  if ((rc = refresh_radius_stats(b))) return rc;
  if ((rc = apply_cutoffs(b))) return rc;
  return build_all(b);
}

int cr_batch_calc_force_energy(cr_batch* b) {
  if (!b) return CR_EINVAL;
  int rc;
  if (!b->nbr_built && (rc = cr_batch_calc_neighbor_lists(b))) return rc;
  if ((rc = force_all(b))) return rc;
  BT_TRY(cudaStreamSynchronize(b->stream));
  return CR_OK;
}

int cr_batch_get_potential_energies(cr_batch* b, double* out) {
  if (!b || !out) return CR_EINVAL;
  int rc;
  if ((rc = reduce_sys(b, 0)) || (rc = pull_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) out[s] = b->bsys_h[s].sums[S_PE];
  return CR_OK;
}

int cr_batch_get_max_unbalanced_forces(cr_batch* b, double* out) {
  if (!b || !out) return CR_EINVAL;
  int rc;
  if ((rc = reduce_sys(b, 0)) || (rc = pull_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) out[s] = std::sqrt(b->bsys_h[s].sums[S_FMAX2]);
  return CR_OK;
}

int cr_batch_get_phis(cr_batch* b, double* out) {
  if (!b || !out) return CR_EINVAL;
  int rc;
  if ((rc = pull_sys(b))) return rc;
  return phis(b, b->area, out);
}

int cr_batch_get_preferred_phis(cr_batch* b, double* out) {
  if (!b || !out) return CR_EINVAL;
  int rc;
  if ((rc = pull_sys(b))) return rc;
  return phis(b, b->a0, out);
}

int cr_batch_get_mean_particle_sizes(cr_batch* b, double* out) {
  return (b && out) ? mean_particle_sizes(b, out) : CR_EINVAL;
}

int cr_batch_init_fire(cr_batch* b, const double* prm, const double* dt, long minStep) {
  if (!b || !prm) return CR_EINVAL;
  b->fp.a_start = prm[0];
  b->fp.f_dec = prm[1];
  b->fp.f_inc = prm[2];
  b->fp.f_a = prm[3];
  b->fp.dt_max = prm[5];
  b->fp.min_step = minStep;
  b->fp.tol = -1.0;
  std::vector<double> st(8 * (size_t)b->S);
  for (int s = 0; s < b->S; s++) {
    // per-system dt keeps the ratio dt_max / dt of the parameter vector
    const double d = dt ? dt[s] : prm[4];
    const double dmax = dt ? prm[5] * (dt[s] / prm[4]) : prm[5];
    for (int par = 0; par < 2; par++) {
      st[8 * s + 4 * par + 0] = d;
      st[8 * s + 4 * par + 1] = prm[6];
      st[8 * s + 4 * par + 2] = 0.0;
      st[8 * s + 4 * par + 3] = dmax;
    }
  }
  int rc;
  if ((rc = upload(b, b->bfire, st.data(), st.size() * sizeof(double)))) return rc;
  if ((rc = pull_sys(b))) return rc;
  for (BatchSys& s : b->bsys_h) {
    s.fire_iters = 0;
    s.converged = 0;
  }
  if ((rc = push_sys(b))) return rc;
  b->fire_ready = true;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_fire_minimize(cr_batch* b, const double* tol, long maxIter, long* iterations, double* maxForce) {
  if (!b || !tol || maxIter < 0) return CR_EINVAL;
  if (!b->fire_ready) return b->fail(CR_ESTATE, "cr_batch_fire_minimize before cr_batch_init_fire");
  int rc;
  if ((rc = pull_sys(b))) return rc;
  std::vector<long long> it0(b->S);
  for (int s = 0; s < b->S; s++) {
    b->bsys_h[s].fire_tol = tol[s];
    b->bsys_h[s].converged = 0;
    b->bsys_h[s].rebuild = 0;
    b->bsys_h[s].done_ctr = 0;
    it0[s] = b->bsys_h[s].fire_iters;
    b->bsys_h[s].fire_cap = it0[s] + maxIter;  // every system stops after maxIter iterations
  }
  if ((rc = push_sys(b))) return rc;
  if ((rc = refresh_radius_stats(b)) || (rc = apply_cutoffs(b))) return rc;
  if ((rc = fire_prologue(b))) return rc;
  if ((rc = fire_loop(b, maxIter, nullptr))) return rc;
  if ((rc = reduce_sys(b, 0)) || (rc = pull_sys(b))) return rc;
  for (BatchSys& bs : b->bsys_h) bs.fire_cap = 0;
  if ((rc = push_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) {
    if (iterations) iterations[s] = (long)(b->bsys_h[s].fire_iters - it0[s]);
    if (maxForce) maxForce[s] = std::sqrt(b->bsys_h[s].sums[S_FMAX2]);
  }
  return CR_OK;
}

int cr_batch_scale_vertices(cr_batch* b, const double* scale) {
  if (!b || !scale) return CR_EINVAL;
  int rc;
  for (int s = 0; s < b->S; s++)
    if (!(scale[s] > 0)) return b->fail(CR_EINVAL, "scale factors must be positive");
  if (!b->nbr_built && (rc = build_all(b))) return rc;
  if ((rc = force_all(b))) return rc;  // ring centroids and areas of the current positions
  if ((rc = upload(b, b->sys_scalar, scale, b->S * sizeof(double)))) return rc;
  const int n = std::max(b->nv, b->np);
  k_bscale<<<(n + 255) / 256, 256, 0, b->stream>>>(b->nv, b->np, b->vsys, b->ring_sys, b->ring_of, b->ppos,
                                                   b->sys_scalar, b->pos, b->l0, b->rad, b->a0, b->area);
  b->launches++;
  BT_TRY(cudaGetLastError());
  BT_TRY(cudaStreamSynchronize(b->stream));
  drop_graphs(b);
  return refresh_radius_stats(b);
}

int cr_batch_set_active(cr_batch* b, const int* active) {
  if (!b || !active) return CR_EINVAL;
  int rc;
  if ((rc = pull_sys(b))) return rc;
  for (int s = 0; s < b->S; s++) b->bsys_h[s].active = active[s] ? 1 : 0;
  return push_sys(b);
}

// The compression protocol of compressFIRE.cpp:101-205, per system and all
// systems together.  Each step: FIRE with dt = fire_dt * sigma_s and force
// tolerance tol0 / sigma_s (sigma_s the system's mean particle size); then
//   jammed:        tol < F < 2 tol            -> the system stops
//   under-jammed:  F <= tol                   -> save the state, grow phi by dphi
//   over-jammed:   F >= 2 tol                 -> halve dphi, restore the saved
//                                                state, grow its phi by dphi
// The starting configuration counts as the first saved state (the reference
// restores zero-filled vectors when its first step is over-jammed).
// (criterion 1 reads U / N_p against energy_tol instead of F against tol,
// the energy form the reference keeps commented out beside the force form).
int cr_batch_compress(cr_batch* b, const cr_compress_params* prm, double* phiOut, long* stepsOut, int* stateOut,
                      long* fireItersOut) {
  if (!b || !prm) return CR_EINVAL;
  if (!(prm->dphi > 0) || prm->max_steps < 0 || prm->max_fire_iters <= 0) return b->fail(CR_EINVAL, "bad compress params");
  return compress_device(b, prm, phiOut, stepsOut, stateOut, fireItersOut);
}

// The same protocol driven from the host: one host round trip per chunk of
// 64 FIRE iterations and per compression step.
int cr_batch_compress_stepwise(cr_batch* b, const cr_compress_params* prm, double* phiOut, long* stepsOut,
                               int* stateOut, long* fireItersOut) {
  if (!b || !prm) return CR_EINVAL;
  if (!(prm->dphi > 0) || prm->max_steps < 0 || prm->max_fire_iters <= 0) return b->fail(CR_EINVAL, "bad compress params");
  const int S = b->S;
  std::vector<double> phi(S), prev(S), dphi(S, prm->dphi), sigma(S), tol(S), dts(S), scale(S);
  std::vector<int> state(S, 0), flag(S);
  std::vector<long> steps(S, 0), its(S);
  std::vector<long long> fire_total(S, 0);
  std::vector<double> fmax(S), upot(S);
  int rc;
  if (!b->nbr_built && (rc = cr_batch_calc_neighbor_lists(b))) return rc;
  if ((rc = force_all(b)) || (rc = pull_sys(b)) || (rc = phis(b, b->area, phi.data()))) return rc;
  prev = phi;
  {
    // the starting configuration is the first "last under-jammed" state, so
    // that a system found over-jammed at its first step steps back to it
    std::fill(flag.begin(), flag.end(), 1);
    if ((rc = upload(b, b->sys_flag, flag.data(), S * sizeof(int)))) return rc;
    const int n = std::max(b->nv, b->np);
    k_bsave<<<(n + 255) / 256, 256, 0, b->stream>>>(b->nv, b->np, b->vsys, b->ring_sys, b->sys_flag, b->pos, b->rad,
                                                    b->l0, b->a0, b->save_pos, b->save_rad, b->save_l0, b->save_a0);
    b->launches++;
    BT_TRY(cudaGetLastError());
  }
  for (long step = 0; step < prm->max_steps; step++) {
    bool any = false;
    for (int s = 0; s < S; s++) any = any || state[s] == 0;
    if (!any) break;
    if ((rc = mean_particle_sizes(b, sigma.data()))) return rc;
    for (int s = 0; s < S; s++) {
      dts[s] = prm->fire_dt * sigma[s];
      tol[s] = prm->tol0 / sigma[s];
    }
    // compressFIRE.cpp:106: {a_start, f_dec, f_inc, f_a, dt, 10 dt, a}, minStep 20
    const double fparams[7] = {0.2, 0.5, 1.1, 0.99, prm->fire_dt, 10 * prm->fire_dt, 0.2};
    if ((rc = cr_batch_init_fire(b, fparams, dts.data(), 20))) return rc;
    std::vector<int> act(S);
    for (int s = 0; s < S; s++) act[s] = state[s] == 0;
    if ((rc = cr_batch_set_active(b, act.data()))) return rc;
    if ((rc = cr_batch_fire_minimize(b, tol.data(), prm->max_fire_iters, its.data(), fmax.data()))) return rc;
    if ((rc = cr_batch_get_potential_energies(b, upot.data()))) return rc;
    for (int s = 0; s < S; s++) {
      flag[s] = 0;
      scale[s] = 1.0;
      if (state[s] != 0) continue;
      fire_total[s] += its[s];
      steps[s] += 1;
      bool jam, over, under;
      if (prm->criterion == 1) {
        const double u = upot[s] / b->sys_np[s];
        jam = u > prm->energy_tol && u < 2 * prm->energy_tol;
        over = u >= 2 * prm->energy_tol;
        under = u <= prm->energy_tol;
      } else {
        jam = fmax[s] > tol[s] && fmax[s] < 2 * tol[s];
        over = fmax[s] >= 2 * tol[s];
        under = fmax[s] <= tol[s];
      }
      if (jam) {
        state[s] = 1;
        continue;
      }
      if (under) {
        scale[s] = std::sqrt((phi[s] + dphi[s]) / phi[s]);
        prev[s] = phi[s];
        flag[s] = 1;
      } else if (over) {
        dphi[s] *= 0.5;
        scale[s] = std::sqrt((prev[s] + dphi[s]) / prev[s]);
        flag[s] = 2;
      }
      if (dphi[s] < prm->min_dphi) state[s] = 3;  // bisection resolved below the requested step
    }
    if ((rc = upload(b, b->sys_flag, flag.data(), S * sizeof(int)))) return rc;
    const int n = std::max(b->nv, b->np);
    k_bsave<<<(n + 255) / 256, 256, 0, b->stream>>>(b->nv, b->np, b->vsys, b->ring_sys, b->sys_flag, b->pos, b->rad,
                                                    b->l0, b->a0, b->save_pos, b->save_rad, b->save_l0, b->save_a0);
    b->launches++;
    BT_TRY(cudaGetLastError());
    for (int s = 0; s < S; s++)
      if (state[s] != 0) scale[s] = 1.0;
    if ((rc = refresh_radius_stats(b))) return rc;
    if ((rc = cr_batch_scale_vertices(b, scale.data()))) return rc;
    if ((rc = force_all(b)) || (rc = phis(b, b->area, phi.data()))) return rc;
    for (int s = 0; s < S; s++)
      if (state[s] == 0 && steps[s] >= prm->max_steps) state[s] = 2;
  }
  for (int s = 0; s < S; s++) {
    if (phiOut) phiOut[s] = phi[s];
    if (stepsOut) stepsOut[s] = steps[s];
    if (stateOut) stateOut[s] = state[s];
    if (fireItersOut) fireItersOut[s] = (long)fire_total[s];
  }
  std::vector<int> all(S, 1);
  return cr_batch_set_active(b, all.data());
}

// Times one batched FIRE iteration's force kernel (the tile op, `reps`
// launches after warm-up) on the current state; FIRE scalars untouched.
int cr_batch_profile_fire_tile(cr_batch* b, long reps, double* ms_per_launch) {
  if (!b || reps <= 0 || !ms_per_launch) return CR_EINVAL;
  int rc;
  if (!b->nbr_built && (rc = cr_batch_calc_neighbor_lists(b))) return rc;
  if ((rc = pull_sys(b))) return rc;
  const std::vector<BatchSys> keep = b->bsys_h;
  for (BatchSys& s : b->bsys_h) {
    s.converged = 0;
    s.fire_tol = -1.0;
  }
  if ((rc = push_sys(b))) return rc;
  std::vector<double> st(8 * (size_t)b->S);
  if ((rc = download(b, st.data(), b->bfire, st.size() * sizeof(double)))) return rc;
  double2* vel_keep = nullptr;
  BT_TRY(cudaMallocAsync((void**)&vel_keep, (size_t)b->nv * sizeof(double2), b->stream));
  BT_TRY(cudaMemcpyAsync(vel_keep, b->vel, (size_t)b->nv * sizeof(double2), cudaMemcpyDeviceToDevice, b->stream));
  cudaEvent_t e0, e1;
  BT_TRY(cudaEventCreate(&e0));
  BT_TRY(cudaEventCreate(&e1));
  for (int w = 0; w < 3; w++) enqueue_fire_tile(b, b->stream);
  BT_TRY(cudaEventRecord(e0, b->stream));
  for (long r = 0; r < reps; r++) enqueue_fire_tile(b, b->stream);
  BT_TRY(cudaEventRecord(e1, b->stream));
  BT_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  BT_TRY(cudaEventElapsedTime(&ms, e0, e1));
  *ms_per_launch = ms / (double)reps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BT_TRY(cudaMemcpyAsync(b->vel, vel_keep, (size_t)b->nv * sizeof(double2), cudaMemcpyDeviceToDevice, b->stream));
  BT_TRY(cudaFreeAsync(vel_keep, b->stream));
  if ((rc = upload(b, b->bfire, st.data(), st.size() * sizeof(double)))) return rc;
  b->bsys_h = keep;
  if ((rc = push_sys(b))) return rc;
  if ((rc = clear_flags(b))) return rc;
  return force_all(b);
}

// Times the batched tile op for each lane count whose tiles hold the largest
// ring and keeps the fastest.
int cr_batch_autotune(cr_batch* b, long reps, int* lanes_out) {
  if (!b || reps <= 0) return CR_EINVAL;
  int maxnv = 0;
  for (int n : b->ring_nv_h) maxnv = std::max(maxnv, n);
  int best_l = b->lanes, best_b = b->block;
  double best_ms = 1e300;
  int rc;
  static const int shapes[][2] = {{1, 128}, {1, 192}, {2, 128}, {2, 192}, {4, 256}};
  for (const auto& sh : shapes) {
    if (maxnv > tile_capacity(sh[0], sh[1])) continue;
    if ((rc = cr_batch_set_tile_shape(b, sh[0], sh[1]))) return rc;
    double ms = 0.0;
    if ((rc = cr_batch_profile_fire_tile(b, reps, &ms))) return rc;
    if (ms < best_ms) {
      best_ms = ms;
      best_l = sh[0];
      best_b = sh[1];
    }
  }
  if ((rc = cr_batch_set_tile_shape(b, best_l, best_b))) return rc;
  if (lanes_out) *lanes_out = best_l;
  return CR_OK;
}

int cr_batch_set_persistent(cr_batch* b, int on) {
  if (!b) return CR_EINVAL;
  b->no_persist = !on;
  drop_graphs(b);
  return CR_OK;
}

int cr_batch_get_list_capacity(const cr_batch* b, int* out) {
  if (!b || !out) return CR_EINVAL;
  *out = b->cap;
  return CR_OK;
}

int cr_batch_get_launch_count(const cr_batch* b, long long* out) {
  if (!b || !out) return CR_EINVAL;
  *out = b->launches;
  return CR_OK;
}

}  // extern "C"
