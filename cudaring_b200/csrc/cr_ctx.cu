// Context, op sequencer (CUDA graphs of step ops, each followed by the
// one-launch neighbour build that runs only when the op armed it) and the
// C ABI declared in include/cudaring.h.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "cr_launch.h"
#include "cr_tile.cuh"

using namespace cr;

#define CR_TRY(expr)                                                                     \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) return ctx->fail(CR_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

enum OpType { OP_DRIFT = 0, OP_TILE = 1, OP_FIRE_PRE = 2, OP_CHECK = 3, OP_RIGID_DRIFT = 4 };

struct Op {
  int type;
  int in_buf;     // position buffer read
  int out_buf;    // position buffer written (drift/advance), or in_buf
  int advance;    // tile: 1 = write next positions, 0 = final (store v, F)
  int check_after;  // the op's displacement check may arm a rebuild (the build follows it)
  int check_buf;    // buffer whose positions the rebuild would use
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  long long launches = 0;  // kernel launches per graph launch
};

long long pow2ceil(long long x) {
  long long p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

struct cr_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;

  int np = 0, nv = 0;
  std::vector<int> ring_first_h, ring_nv_h, ring_of_h;
  std::vector<int4> tiles_h;
  int lanes = 2;
  int precision = CR_PRECISION_FP64;

  SysParams p{};
  int potential = 0, interaction = 0, monomer = 0, particle = 0, noise_type = 0, shape = 0, geometry = 0;
  double dt = 1e-3, driving = 0.0, taup = 0.0;
  unsigned long long seed = 0x5EEDC0DEULL;
  unsigned long long rng_calls = 0;
  double cutoff = 0.0, cut_distance = 1.0;
  long long list_size_ref = 0;
  double rmax = 0.0;

  // device state
  double2* pos[2] = {nullptr, nullptr};
  int cur = 0;
  double2 *vel = nullptr, *force = nullptr, *last_pos = nullptr, *ppos = nullptr;
  double *rad = nullptr, *l0 = nullptr, *theta0 = nullptr, *a0 = nullptr;
  double *energy = nullptr, *p_energy = nullptr, *theta = nullptr, *length = nullptr, *area = nullptr,
         *perimeter = nullptr, *p_angle = nullptr, *vertex_area = nullptr;
  int *ring_of = nullptr, *ring_first = nullptr, *ring_nv = nullptr, *zero_cnt = nullptr;
  int2* pp_of = nullptr;
  int2* vtopo = nullptr;   // {ring, k | nv << 16}
  int* pq_pack = nullptr;  // packed (prev - v, prev(prev) - v)
  int4* tiles = nullptr;
  int* nbr = nullptr;
  int* nbr_pq = nullptr;   // companion of nbr: pq_pack of each listed neighbour
  int* nbr_cnt = nullptr;
  int cap = 0;
  bool nbr_built = false;
  // cell scratch
  CellGrid grid{0, 0, 0.0, 0.0};
  int ncells_alloc = 0;
  int *cell_of = nullptr, *slot = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_vid = nullptr,
      *cell_ring = nullptr, *cell_pq = nullptr;
  int* block_sum = nullptr;  // per-CTA totals of the one-launch build
  // cell buckets of the one-launch build, kCellBucket members per cell (ids,
  // positions, radii, rings, packed offsets); cell_cnt then holds two count
  // arrays of ncells_alloc entries and two control words
  int *cell_bucket = nullptr, *bucket_ring = nullptr, *bucket_pq = nullptr;
  double2* bucket_pos = nullptr;
  double* bucket_rad = nullptr;
  int fused_max = 0;         // CTAs of the one-launch build resident at once
  double2* cell_pos = nullptr;
  double* cell_rad = nullptr;
  double* partials = nullptr;
  // derivative evaluations (cr_hvp, cr_calc_pressure, cr_param_derivatives)
  double* diff_f = nullptr;   // [nv][8]
  double* diff_e = nullptr;   // [nv][4]
  double* diff_dot = nullptr; // [256] dot-product partials
  double* diff_vec = nullptr; // [5][2 nv] CG vectors
  double* diff_area = nullptr; // [np][4] hyper-dual ring areas
  CgState* cg_state = nullptr;
  double* cg_part = nullptr;   // [148][8] CG reduction partials
  double* cg_minv = nullptr;   // [nv][3] inverse diagonal Hessian blocks (block-Jacobi preconditioner)
  int cg_precond = 1;          // 1: block-Jacobi preconditioner in cr_hessian_solve; 0: none
  int partials_n = 0;
  DevStatus* status = nullptr;
  DevStatus* status_h = nullptr;  // pinned
  double* fire_state = nullptr;   // [2][4]
  // rigid rings
  double2 *p_vel = nullptr, *p_force = nullptr;
  double *p_angvel = nullptr, *p_torque = nullptr, *p_moi = nullptr, *v_torque = nullptr, *sp_angle = nullptr;
  // soft-disk pre-packing (allocated on first use)
  bool soft_ready = false;
  double* prad = nullptr;       // particle radii
  double2* plast = nullptr;     // particle positions at the last list build
  int* pid = nullptr;           // identity: every particle is its own "ring" for the list build
  int *pnbr = nullptr, *pnbr_cnt = nullptr;
  int pcap = 0;
  bool pnbr_built = false;
  long long plist_size_ref = 0;
  CellGrid pgrid{0, 0, 0.0, 0.0};
  DevStatus* pstatus = nullptr;
  SoftFire* pfire = nullptr;
  bool pfire_ready = false;
  double* pdraws = nullptr;     // 2 nv caller-supplied draws for initVerticesOnParticles
  std::map<long, GraphEntry> soft_graphs;
  double soft_key[3] = {0.0, 0.0, 0.0};  // cutDistance, cutoff, cells of the captured minimisation graphs

  // integrators
  int sim_kind = -1;  // Kind
  double T = 0.0, gamma = 1.0, noise = 0.0, gamma_factor = 1.0;
  bool fire_ready = false;
  FireParams fp{};
  bool use_graphs = true;
  bool multistep = true;  // middle steps of NVE / Langevin / BAOAB runs in k_tile_steps
  // A grid-barrier wait gave up (the GPU did not hold every CTA of a
  // one-launch build or multi-step kernel at once, e.g. because other work
  // shared it): from then on one launch per op, no graphs, and the list built
  // by the multi-kernel path, whose kernels never wait for one another.
  bool degraded = false;
  // state at the start of a multi-step sequence, restored if a barrier gives up
  double2 *snap_pos = nullptr, *snap_vel = nullptr, *snap_force = nullptr, *snap_last = nullptr;
  double* snap_angle = nullptr;

  std::map<std::tuple<int, long, int, int, unsigned long long>, GraphEntry> graphs;

  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
};

namespace {

int upload(cr_ctx* ctx, void* dst, const void* src, size_t bytes);

template <typename T>
int dalloc(cr_ctx* ctx, T** p, size_t n) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return ctx->fail(CR_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(*p, 0, n * sizeof(T));
  if (e != cudaSuccess) return ctx->fail(CR_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  return CR_OK;
}

void drop_graphs(cr_ctx* ctx) {
  for (auto& kv : ctx->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->graphs.clear();
  for (auto& kv : ctx->soft_graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
  }
  ctx->soft_graphs.clear();
}

// After a grid-barrier wait gave up: one launch per op from now on.
void enter_degraded(cr_ctx* ctx) {
  ctx->degraded = true;
  ctx->multistep = false;
  ctx->use_graphs = false;
  drop_graphs(ctx);
  // the build that gave up left its cell counts part-done: every count back
  // to zero, the first array current (the particle-list build still uses
  // the bucket form)
  if (ctx->cell_cnt && ctx->ncells_alloc > 0)
    cudaMemsetAsync(ctx->cell_cnt, 0, cell_count_words(ctx->ncells_alloc) * sizeof(int), ctx->stream);
}

void refresh_params(cr_ctx* ctx) {
  SysParams& p = ctx->p;
  p.nv = ctx->nv;
  p.np = ctx->np;
  p.inv_lx = 1.0 / p.lx;
  p.inv_ly = 1.0 / p.ly;
  p.monomer = ctx->monomer;
  p.potential = ctx->potential;
}

SysArrays arrays(cr_ctx* ctx, int buf, bool zero_list = false) {
  SysArrays a;
  a.pos = ctx->pos[buf];
  a.rad = ctx->rad;
  a.l0 = ctx->l0;
  a.theta0 = ctx->theta0;
  a.a0 = ctx->a0;
  a.ring_of = ctx->ring_of;
  a.ring_first = ctx->ring_first;
  a.ring_nv = ctx->ring_nv;
  a.pp_of = ctx->pp_of;
  a.nbr = ctx->nbr;
  a.nbr_cnt = (zero_list || !ctx->nbr_built) ? ctx->zero_cnt : ctx->nbr_cnt;
  a.tiles = ctx->tiles;
  a.nbr_cap = ctx->cap;
  a.vtopo = ctx->vtopo;
  a.nbr_pq = ctx->nbr_pq;
  return a;
}

StepArgs base_args(cr_ctx* ctx) {
  StepArgs s;
  memset(&s, 0, sizeof(s));
  s.vel = ctx->vel;
  s.force = ctx->force;
  s.last_pos = ctx->last_pos;
  s.energy = ctx->energy;
  s.p_energy = ctx->p_energy;
  s.theta_out = ctx->theta;
  s.length_out = ctx->length;
  s.area_out = ctx->area;
  s.perim_out = ctx->perimeter;
  s.ppos_out = ctx->ppos;
  s.p_angle = ctx->p_angle;
  s.partials = ctx->partials;
  s.status = ctx->status;
  s.fire_state = ctx->fire_state;
  s.dt = ctx->dt;
  s.hdt = 0.5 * ctx->dt;
  s.gamma = ctx->gamma;
  s.noise = ctx->noise;
  s.gamma_factor = ctx->gamma_factor;
  s.driving = ctx->driving;
  s.sp_amp = ctx->taup != 0.0 ? std::sqrt(2.0 * ctx->dt / ctx->taup) : 0.0;
  s.active = ctx->particle == CR_PARTICLE_ACTIVE;
  s.disp_cutoff = ctx->cutoff;
  s.seed = ctx->seed;
  s.fire_tol = -1.0;
  return s;
}

RigidArgs rigid_args(cr_ctx* ctx) {
  RigidArgs r;
  r.p_vel = ctx->p_vel;
  r.p_angle = ctx->p_angle;
  r.p_angvel = ctx->p_angvel;
  r.p_force = ctx->p_force;
  r.p_torque = ctx->p_torque;
  r.p_moi = ctx->p_moi;
  r.v_torque = ctx->v_torque;
  r.sp_angle = ctx->sp_angle;
  return r;
}

int inter_kind(cr_ctx* ctx) {
  return (ctx->interaction == CR_INTERACTION_VERTEX_VERTEX || ctx->interaction == CR_INTERACTION_ALL) ? INT_VV
                                                                                                      : INT_SMOOTH;
}

LaunchCfg tile_cfg(cr_ctx* ctx) {
  return LaunchCfg{ctx->stream, (int)ctx->tiles_h.size(), ctx->lanes, ctx->precision};
}

int ensure_partials(cr_ctx* ctx) {
  int need = std::max<int>((int)ctx->tiles_h.size(), 2048) * NSUM;
  if (ctx->partials_n >= need) return CR_OK;
  ctx->partials_n = need;
  return dalloc(ctx, &ctx->partials, need);
}

// Cell grid for the current box, radii and cutDistance (see cr_nbr.cu).
// Cell scratch for grids of up to `ncells` cells (vertex and particle grids
// share it): counts in the bucket form's layout (zeroed, the first array
// current), starts and buckets.
int alloc_cells(cr_ctx* ctx, int ncells) {
  if (ncells <= ctx->ncells_alloc) return CR_OK;
  drop_graphs(ctx);
  int rc;
  if ((rc = dalloc(ctx, &ctx->cell_cnt, cell_count_words(ncells)))) return rc;
  if ((rc = dalloc(ctx, &ctx->cell_start, ncells + 1))) return rc;
  const size_t nb = (size_t)ncells * kCellBucket;
  if ((rc = dalloc(ctx, &ctx->cell_bucket, nb)) || (rc = dalloc(ctx, &ctx->bucket_pos, nb)) ||
      (rc = dalloc(ctx, &ctx->bucket_rad, nb)) || (rc = dalloc(ctx, &ctx->bucket_ring, nb)) ||
      (rc = dalloc(ctx, &ctx->bucket_pq, nb)))
    return rc;
  ctx->ncells_alloc = ncells;
  return CR_OK;
}

// Every cell count zero and the first array current: after a build that
// stopped part-way (a grid-barrier wait gave up), whose counts are unknown.
int reset_cell_counts(cr_ctx* ctx) {
  if (ctx->cell_cnt && ctx->ncells_alloc > 0)
    CR_TRY(cudaMemsetAsync(ctx->cell_cnt, 0, cell_count_words(ctx->ncells_alloc) * sizeof(int), ctx->stream));
  return CR_OK;
}

int setup_grid(cr_ctx* ctx, double cut) {
  const double cmin = (1.0 + cut) * 2.0 * ctx->rmax * (1.0 + 1e-9);
  int ncx = cmin > 0 ? (int)std::floor(ctx->p.lx / cmin) : 0;
  int ncy = cmin > 0 ? (int)std::floor(ctx->p.ly / cmin) : 0;
  ncx = std::min(ncx, 4096);
  ncy = std::min(ncy, 4096);
  if (ncx < 3 || ncy < 3) {
    ctx->grid = CellGrid{0, 0, 0.0, 0.0};
    return CR_OK;
  }
  // The sorted-cell stencil search (the multi-kernel build, and the one-launch
  // build when a cell overflows its bucket) deals home cells to its warps in
  // rounds; a last round that only a few warps take costs a whole round.
  // When the build fills the GPU and there are more cells than warps, coarsen
  // the grid (larger cells hold every pair the smaller ones did) to a whole
  // number of rounds: the lists hold the same neighbours, in the order of the
  // coarser cells.  Smaller systems keep the finest grid.
  {
    const int blocks = nbr_fused_blocks(ctx->nv, ctx->fused_max);
    const long warps = (long)blocks * 32;
    const long cells = (long)ncx * ncy;
    if (ctx->fused_max > 0 && blocks >= ctx->fused_max && cells > warps && cells % warps != 0) {
      const double f = std::sqrt((double)((cells / warps) * warps) / (double)cells);
      const int nx = std::max(3, (int)std::floor(ncx * f)), ny = std::max(3, (int)std::floor(ncy * f));
      if ((long)nx * ny <= (cells / warps) * warps) {
        ncx = nx;
        ncy = ny;
      }
    }
  }
  ctx->grid = CellGrid{ncx, ncy, ctx->p.lx / ncx, ctx->p.ly / ncy};
  const int ncells = ncx * ncy;
  return alloc_cells(ctx, ncells);
}

NbrArgs nbr_args(cr_ctx* ctx, int buf, double cut) {
  NbrArgs n;
  n.pos = ctx->pos[buf];
  n.rad = ctx->rad;
  n.ring_of = ctx->ring_of;
  n.nbr = ctx->nbr;
  n.nbr_cnt = ctx->nbr_cnt;
  n.cap = ctx->cap;
  n.cut_distance = cut;
  n.last_pos = ctx->last_pos;
  n.cell_of = ctx->cell_of;
  n.slot = ctx->slot;
  n.cell_cnt = ctx->cell_cnt;
  n.cell_start = ctx->cell_start;
  n.cell_vid = ctx->cell_vid;
  n.cell_pos = ctx->cell_pos;
  n.cell_rad = ctx->cell_rad;
  n.cell_ring = ctx->cell_ring;
  n.pq_pack = ctx->pq_pack;
  n.nbr_pq = ctx->nbr_pq;
  n.cell_pq = ctx->cell_pq;
  n.status = ctx->status;
  n.count_op = 0;
  n.count_update = 0;
  n.block_sum = ctx->block_sum;
  n.bucket = ctx->cell_bucket;
  n.bucket_pos = ctx->bucket_pos;
  n.bucket_rad = ctx->bucket_rad;
  n.bucket_ring = ctx->bucket_ring;
  n.bucket_pq = ctx->bucket_pq;
  n.cell_stride = ctx->ncells_alloc;
  return n;
}

int read_status(cr_ctx* ctx) {
  CR_TRY(cudaMemcpyAsync(ctx->status_h, ctx->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int clear_flags(cr_ctx* ctx) {
  // abort, overflow, rebuild, converged, nonfinite <- 0 (counters kept)
  int rc = read_status(ctx);
  if (rc) return rc;
  DevStatus s = *ctx->status_h;
  s.abort = 0;
  s.overflow = 0;
  s.rebuild = 0;
  s.converged = 0;
  s.nonfinite = 0;
  s.done_ctr = 0;
  s.bar_count = 0;
  s.stalled = 0;
  s.pbar = 0;
  s.pflag[0] = s.pflag[1] = s.pflag[2] = 0;
  s.pbase = 0;
  *ctx->status_h = s;
  CR_TRY(cudaMemcpyAsync(ctx->status, ctx->status_h, sizeof(DevStatus), cudaMemcpyHostToDevice, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

// Neighbour list and its companion at capacity `cap`.
int alloc_lists(cr_ctx* ctx, int cap) {
  int rc;
  if ((rc = dalloc(ctx, &ctx->nbr, (size_t)cap * ctx->nv))) return rc;
  if ((rc = dalloc(ctx, &ctx->nbr_pq, (size_t)cap * ctx->nv))) return rc;
  ctx->cap = cap;
  return CR_OK;
}

// Build the list from positions buffer `buf`; grows capacity like the
// reference (two passes when the first overflowed).
int build_list(cr_ctx* ctx, int buf, double cut) {
  int rc;
  if ((rc = setup_grid(ctx, cut))) return rc;
  for (int pass = 0; pass < 3; pass++) {
    if (ctx->degraded) {
      // the multi-kernel build: per-cell counters start at zero
      if (ctx->grid.ncx)
        CR_TRY(cudaMemsetAsync(ctx->cell_cnt, 0, (size_t)ctx->grid.ncx * ctx->grid.ncy * sizeof(int), ctx->stream));
      launch_nbr_build(ctx->stream, ctx->p, ctx->grid, nbr_args(ctx, buf, cut));
      ctx->launches += 6;
    } else {
      launch_nbr_fused(ctx->stream, ctx->p, ctx->grid, nbr_args(ctx, buf, cut),
                       nbr_fused_blocks(ctx->nv, ctx->fused_max), 1);
      ctx->launches += 1;
    }
    CR_TRY(cudaGetLastError());
    if ((rc = read_status(ctx))) return rc;
    if (ctx->status_h->stalled) {
      if (ctx->degraded) return ctx->fail(CR_ECUDA, "neighbour-list build: a grid barrier timed out");
      // the one-launch build's CTAs were not all resident: build again with
      // the multi-kernel path (positions are untouched by a build)
      enter_degraded(ctx);
      if ((rc = clear_flags(ctx))) return rc;
      pass = -1;
      continue;
    }
    const int mc = ctx->status_h->max_count;
    if (!ctx->status_h->overflow) {
      ctx->list_size_ref = std::max<long long>(ctx->list_size_ref, mc > 0 ? pow2ceil(mc) : 0);
      ctx->nbr_built = true;
      if (mc * 2 > ctx->cap) {
        // keep headroom for rebuilds inside step sequences
        int newcap = (int)std::max<long long>(16, pow2ceil(2LL * mc));
        if ((rc = alloc_lists(ctx, newcap))) return rc;
        drop_graphs(ctx);
        if ((rc = clear_flags(ctx))) return rc;
        continue;  // rebuild into the larger list
      }
      return CR_OK;
    }
    int newcap = (int)std::max<long long>(16, pow2ceil(2LL * mc));
    if ((rc = alloc_lists(ctx, newcap))) return rc;
    drop_graphs(ctx);
    if ((rc = clear_flags(ctx))) return rc;
  }
  return ctx->fail(CR_ENBR_OVERFLOW, "neighbour list did not fit after growing");
}

void update_rmax(cr_ctx* ctx, const double* rad_h) {
  double m = 0.0;
  for (int i = 0; i < ctx->nv; i++) m = std::max(m, rad_h[i]);
  ctx->rmax = m;
}

int force_pass(cr_ctx* ctx, bool zero_list) {
  StepArgs s = base_args(ctx);
  s.kind = KIND_NONE;
  s.write_out = 1;
  s.active = 0;
  if (ctx->particle == CR_PARTICLE_ACTIVE && !zero_list) {
    // addSelfPropulsion advances the ring angles, then adds f0 (cos, sin)
    launch_advance_angles(ctx->stream, ctx->np, ctx->p_angle, s.sp_amp, ctx->seed, (1ull << 62) + ctx->rng_calls++);
    ctx->launches++;
    s.active = 1;
  }
  launch_tile(tile_cfg(ctx), ctx->potential, inter_kind(ctx), MODE_FORCE, ctx->p, arrays(ctx, ctx->cur, zero_list), s);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  return CR_OK;
}

int reduce_now(cr_ctx* ctx) {
  int rc;
  if ((rc = ensure_partials(ctx))) return rc;
  const int nb = std::min(2048, std::max(1, (ctx->nv + 255) / 256));
  launch_reduce(ctx->stream, ctx->nv, ctx->np, ctx->vel, ctx->force, ctx->energy, ctx->p_energy,
                inter_kind(ctx) == INT_SMOOTH, ctx->partials, ctx->status, nb);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  return read_status(ctx);
}

// ------------------------------------------------------------- op sequences

// Ops of one call.  NVE / Langevin / BAOAB: drift, then nsteps tile ops (the
// last one final); Brownian: a displacement check, then nsteps advancing tile
// ops; FIRE: nsteps x (pre, tile).
std::vector<Op> make_ops(cr_ctx* ctx, int kind, long nsteps) {
  std::vector<Op> ops;
  int b = ctx->cur;
  if (kind == KIND_FIRE) {
    for (long i = 0; i < nsteps; i++) {
      ops.push_back(Op{OP_FIRE_PRE, b, b, 0, 1, b});
      ops.push_back(Op{OP_TILE, b, b, 0, 0, b});
    }
  } else if (kind == KIND_NVE_RESCALE) {
    // NVERescale: rescale + first kick + drift, then force + second kick;
    // the tile op's sum of v^2 feeds the next step's rescale
    for (long i = 0; i < nsteps; i++) {
      ops.push_back(Op{OP_DRIFT, b, b ^ 1, 0, 1, b ^ 1});
      b ^= 1;
      ops.push_back(Op{OP_TILE, b, b, 0, 0, b});
    }
  } else if (kind == KIND_BROWNIAN || kind == KIND_DRIVEN_BROWNIAN) {
    ops.push_back(Op{OP_CHECK, b, b, 0, 1, b});
    for (long i = 0; i < nsteps; i++) {
      ops.push_back(Op{OP_TILE, b, b ^ 1, 1, 1, b ^ 1});
      b ^= 1;
    }
  } else {
    ops.push_back(Op{ctx->shape == CR_SHAPE_RIGID ? OP_RIGID_DRIFT : OP_DRIFT, b, b ^ 1, 0, 1, b ^ 1});
    b ^= 1;
    for (long i = 0; i < nsteps; i++) {
      const bool last = (i == nsteps - 1);
      if (last) {
        ops.push_back(Op{OP_TILE, b, b, 0, 0, b});
      } else {
        ops.push_back(Op{OP_TILE, b, b ^ 1, 1, 1, b ^ 1});
        b ^= 1;
      }
    }
  }
  return ops;
}

void enqueue_op(cr_ctx* ctx, cudaStream_t st, const Op& op, int kind, bool use_cond, cudaGraphConditionalHandle h) {
  StepArgs s = base_args(ctx);
  s.kind = kind;
  s.use_cond = use_cond ? 1 : 0;
  s.cond = h;
  s.pos_out = ctx->pos[op.out_buf];
  s.advance = op.advance;
  // per-CTA sums feed FIRE's next iteration and the rigid tail; energies
  // read by the caller are reduced afresh from the written arrays
  s.accumulate = (kind == KIND_FIRE || kind == KIND_NVE_RESCALE || ctx->shape == CR_SHAPE_RIGID) ? 1 : 0;
  s.rescale_T = (kind == KIND_NVE_RESCALE && op.type == OP_DRIFT) ? ctx->T : 0.0;
  s.write_out = (kind == KIND_FIRE || !op.advance) ? 1 : 0;
  s.fire_tol = ctx->fp.tol;
  const SysArrays a = arrays(ctx, op.in_buf);
  const int nb = (ctx->nv + 255) / 256;
  switch (op.type) {
    case OP_DRIFT:
      s.kind = kind;
      launch_drift(st, ctx->p, a, s, nb);
      break;
    case OP_CHECK:
      // a drift with dt = 0 is exactly the displacement check of current positions
      s.kind = KIND_NVE;
      s.dt = 0.0;
      s.hdt = 0.0;
      s.pos_out = ctx->pos[op.out_buf];
      launch_drift(st, ctx->p, a, s, nb);
      break;
    case OP_FIRE_PRE:
      launch_fire_pre(st, ctx->p, a, s, ctx->fp, ctx->fire_state, nb);
      break;
    case OP_TILE: {
      LaunchCfg c = tile_cfg(ctx);
      c.stream = st;
      c.pdl = true;
      if (ctx->shape == CR_SHAPE_RIGID) launch_rigid(c, ctx->potential, MODE_STEP, ctx->p, a, s, rigid_args(ctx));
      else launch_tile(c, ctx->potential, inter_kind(ctx), MODE_STEP, ctx->p, a, s);
      break;
    }
    case OP_RIGID_DRIFT: {
      LaunchCfg c = tile_cfg(ctx);
      c.stream = st;
      launch_rigid_drift(c, ctx->p, a, s, rigid_args(ctx));
      break;
    }
  }
  ctx->launches++;
}

// A step sequence as one graph.  Every op that may arm a rebuild (its
// displacement check) is followed by the one-launch build, which returns at
// once unless the check fired (DPM2D::checkDisplacement, src/DPM2D.cu:1397-1405,
// rebuilds and counts an update).
int capture_graph(cr_ctx* ctx, const std::vector<Op>& ops, int kind, GraphEntry& ge) {
  CR_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  const int fb = nbr_fused_blocks(ctx->nv, ctx->fused_max);
  ge.launches = 0;
  for (const Op& op : ops) {
    enqueue_op(ctx, ctx->stream, op, kind, false, 0);
    ge.launches++;
    if (op.check_after) {
      NbrArgs nb = nbr_args(ctx, op.check_buf, ctx->cut_distance);
      nb.count_update = 1;
      launch_nbr_fused(ctx->stream, ctx->p, ctx->grid, nb, fb, 0, ctx->shape != CR_SHAPE_RIGID);
      ge.launches++;
    }
  }
  cudaGraph_t out = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &out);
  if (e != cudaSuccess) {
    if (out) cudaGraphDestroy(out);
    return ctx->fail(CR_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  }
  CR_TRY(cudaGraphInstantiate(&ge.exec, out, 0));
  ge.graph = out;
  return CR_OK;
}

// Direct launches with a host check after every op that may arm a rebuild:
// the fallback when graphs are off, and the resume path after an abort.
int run_direct(cr_ctx* ctx, const std::vector<Op>& ops, size_t first, int kind) {
  int rc;
  for (size_t i = first; i < ops.size(); i++) {
    const Op& op = ops[i];
    enqueue_op(ctx, ctx->stream, op, kind, false, 0);
    CR_TRY(cudaGetLastError());
    if ((rc = read_status(ctx))) return rc;
    if (ctx->status_h->abort) return CR_OK;  // caller inspects
    if (op.check_after && ctx->status_h->rebuild) {
      if ((rc = build_list(ctx, op.check_buf, ctx->cut_distance))) return rc;
      ctx->status_h->update_count += 1;  // DPM2D::checkDisplacement's updateCount
      if ((rc = upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus)))) return rc;
    }
  }
  return CR_OK;
}

int launch_chunk(cr_ctx* ctx, const std::vector<Op>& ops, int kind, long n) {
  if (ctx->use_graphs) {
    auto key = std::make_tuple(kind, n, ops.front().in_buf, ctx->cap, 0ULL);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
      GraphEntry ge;
      if (capture_graph(ctx, ops, kind, ge) != CR_OK) {
        cudaGetLastError();
        ctx->use_graphs = false;  // direct launches for the life of the context
      } else {
        it = ctx->graphs.emplace(key, ge).first;
      }
    }
    if (ctx->use_graphs) {
      CR_TRY(cudaGraphLaunch(it->second.exec, ctx->stream));
      ctx->launches += it->second.launches;
      return CR_OK;
    }
  }
  return run_direct(ctx, ops, 0, kind);
}

// ---------------------------------------------------- multi-step sequences
// NVE, Langevin and BAOAB runs of deformable rings: the drift op, then the
// middle steps in k_tile_steps launches (each runs until its step budget, a
// due rebuild or the end of the sequence; the one-launch build follows
// every launch), then the final op.  Graphs of up to kStepsLaunches such
// pairs (sized to the steps left, one spare launch for a rebuild) are
// launched until the device counter of middle steps reaches zero; the step
// arithmetic is the per-op path's, so FP64 results are identical to it.
constexpr int kStepsPerLaunch = 64;
constexpr int kStepsLaunches = 16;

bool steps_eligible(cr_ctx* ctx, int kind, long nsteps) {
  if (!ctx->multistep || !ctx->use_graphs || nsteps < 2) return false;
  if (ctx->shape == CR_SHAPE_RIGID) return false;
  if (kind != KIND_NVE && kind != KIND_LANGEVIN && kind != KIND_BAOAB) return false;
  if (ctx->lanes != 1 && ctx->lanes != 2) return false;
  const int maxb = tile_steps_max_blocks(ctx->potential, inter_kind(ctx), ctx->lanes, ctx->precision);
  return maxb >= (int)ctx->tiles_h.size();
}

int capture_steps_graph(cr_ctx* ctx, int kind, int b, int launches, GraphEntry& ge) {
  StepArgs s = base_args(ctx);
  s.kind = kind;
  s.pos_out = ctx->pos[b ^ 1];
  s.advance = 1;
  s.accumulate = 0;
  s.write_out = 0;
  s.persist_max = kStepsPerLaunch;
  const SysArrays a = arrays(ctx, b);
  LaunchCfg c = tile_cfg(ctx);
  c.stream = ctx->stream;
  c.pdl = true;
  NbrArgs nb = nbr_args(ctx, b, ctx->cut_distance);
  nb.count_update = 1;
  const int fb = nbr_fused_blocks(ctx->nv, ctx->fused_max);
  CR_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaSuccess;
  for (int r = 0; r < launches && e == cudaSuccess; r++) {
    e = launch_tile_steps(c, ctx->potential, inter_kind(ctx), ctx->p, a, s);
    launch_nbr_fused(ctx->stream, ctx->p, ctx->grid, nb, fb, 0, true);
  }
  cudaGraph_t out = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &out);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&ge.exec, out, 0);
  if (e != cudaSuccess) {
    if (out) cudaGraphDestroy(out);
    return ctx->fail(CR_ECUDA, std::string("multi-step graph: ") + cudaGetErrorString(e));
  }
  ge.graph = out;
  ge.launches = 2 * launches;
  return CR_OK;
}

int run_ops(cr_ctx* ctx, int kind, long nsteps);

// The state a multi-step sequence starts from (positions, velocities,
// forces, last-build positions, self-propulsion angles), saved or restored.
int sequence_state(cr_ctx* ctx, int b, bool restore) {
  int rc;
  if (!ctx->snap_pos) {
    if ((rc = dalloc(ctx, &ctx->snap_pos, ctx->nv)) || (rc = dalloc(ctx, &ctx->snap_vel, ctx->nv)) ||
        (rc = dalloc(ctx, &ctx->snap_force, ctx->nv)) || (rc = dalloc(ctx, &ctx->snap_last, ctx->nv)) ||
        (rc = dalloc(ctx, &ctx->snap_angle, ctx->np)))
      return rc;
  }
  const size_t v2 = (size_t)ctx->nv * sizeof(double2), pa = (size_t)ctx->np * sizeof(double);
  double2* live[4] = {ctx->pos[b], ctx->vel, ctx->force, ctx->last_pos};
  double2* saved[4] = {ctx->snap_pos, ctx->snap_vel, ctx->snap_force, ctx->snap_last};
  for (int k = 0; k < 4; k++)
    CR_TRY(cudaMemcpyAsync(restore ? live[k] : saved[k], restore ? saved[k] : live[k], v2, cudaMemcpyDeviceToDevice,
                           ctx->stream));
  CR_TRY(cudaMemcpyAsync(restore ? ctx->p_angle : ctx->snap_angle, restore ? ctx->snap_angle : ctx->p_angle, pa,
                         cudaMemcpyDeviceToDevice, ctx->stream));
  return CR_OK;
}

// A grid barrier of the multi-step kernel or of its builds gave up, leaving
// the sequence's positions partly advanced: go back to the state it started
// from (counters included), rebuild the list there with the multi-kernel
// build and run the whole sequence again one launch per op.
int rerun_degraded(cr_ctx* ctx, int b0, const DevStatus& start, int kind, long nsteps) {
  int rc;
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  if ((rc = sequence_state(ctx, b0, true))) return rc;
  ctx->cur = b0;
  DevStatus s = start;
  s.abort = s.overflow = s.rebuild = s.converged = s.nonfinite = s.stalled = 0;
  s.done_ctr = s.bar_count = s.pbar = 0;
  s.pflag[0] = s.pflag[1] = s.pflag[2] = 0;
  s.pbase = s.steps_left = 0;
  *ctx->status_h = s;
  if ((rc = upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus)))) return rc;
  enter_degraded(ctx);
  if ((rc = build_list(ctx, b0, ctx->cut_distance))) return rc;
  return run_ops(ctx, kind, nsteps);
}

int run_steps(cr_ctx* ctx, int kind, long nsteps) {
  int rc;
  int b = ctx->cur;
  const int b0 = b;
  const DevStatus start = *ctx->status_h;  // read by the caller's clear_flags
  if ((rc = sequence_state(ctx, b0, false))) return rc;
  // drift (first half kick + drift) and its displacement check
  enqueue_op(ctx, ctx->stream, Op{OP_DRIFT, b, b ^ 1, 0, 1, b ^ 1}, kind, false, 0);
  {
    NbrArgs nb = nbr_args(ctx, b ^ 1, ctx->cut_distance);
    nb.count_update = 1;
    launch_nbr_fused(ctx->stream, ctx->p, ctx->grid, nb, nbr_fused_blocks(ctx->nv, ctx->fused_max), 0);
    ctx->launches++;
  }
  b ^= 1;
  const long long middle = nsteps - 1;
  CR_TRY(cudaMemcpyAsync(&ctx->status->steps_left, &middle, sizeof(middle), cudaMemcpyHostToDevice, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  long long left = middle;
  for (;;) {
    const int launches =
        (int)std::min<long long>(kStepsLaunches, std::max<long long>(2, (left + kStepsPerLaunch - 1) / kStepsPerLaunch + 1));
    auto key = std::make_tuple(kind, -(long)launches, b, ctx->cap, 1ULL);
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
      GraphEntry ge;
      if ((rc = capture_steps_graph(ctx, kind, b, launches, ge))) return rc;
      it = ctx->graphs.emplace(key, ge).first;
    }
    CR_TRY(cudaGraphLaunch(it->second.exec, ctx->stream));
    ctx->launches += it->second.launches;
    if ((rc = read_status(ctx))) return rc;
    const DevStatus& st = *ctx->status_h;
    if (st.abort) {
      if (st.stalled) return rerun_degraded(ctx, b0, start, kind, nsteps);
      if (st.nonfinite) return ctx->fail(CR_ENONFINITE, "non-finite force during the step sequence");
      if (!st.overflow) return ctx->fail(CR_ECUDA, "step sequence aborted");
      // a rebuild found more neighbours than capacity: grow the list, rebuild
      // from the positions the failed build read (pos[b]), count the update
      // as the in-graph build would have, and carry on
      if ((rc = clear_flags(ctx))) return rc;
      ctx->cap = 0;
      if ((rc = build_list(ctx, b, ctx->cut_distance))) return rc;
      if ((rc = clear_flags(ctx))) return rc;
      ctx->status_h->update_count += 1;
      if ((rc = upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus)))) return rc;
      continue;
    }
    if (st.steps_left <= 0) break;
    left = st.steps_left;
  }
  // final op: forces at the last positions and the second half kick
  enqueue_op(ctx, ctx->stream, Op{OP_TILE, b, b, 0, 0, b}, kind, false, 0);
  CR_TRY(cudaGetLastError());
  if ((rc = read_status(ctx))) return rc;
  if (ctx->status_h->nonfinite) return ctx->fail(CR_ENONFINITE, "non-finite force during the step sequence");
  ctx->cur = b;
  if (ctx->status_h->max_ever > 0)
    ctx->list_size_ref = std::max<long long>(ctx->list_size_ref, pow2ceil(ctx->status_h->max_ever));
  return CR_OK;
}

// Runs nsteps integrator steps (or FIRE iterations) as chunks of captured
// graphs.  Non-FIRE chunks are launched back to back with one status read at
// the end; FIRE reads the status after every chunk to stop at convergence.
// A neighbour-list overflow inside a chunk aborts the remaining ops (they
// become no-ops); the host then grows the list and resumes from the op after
// which the failed build ran.
int run_ops(cr_ctx* ctx, int kind, long nsteps) {
  int rc;
  if ((rc = ensure_partials(ctx))) return rc;
  if (!ctx->nbr_built) {
    if ((rc = build_list(ctx, ctx->cur, ctx->cut_distance))) return rc;
  } else if ((rc = setup_grid(ctx, ctx->cut_distance))) {
    return rc;
  }
  if (kind == KIND_NVE_RESCALE) {
    // the first rescale reads the sum of v^2 of the current velocities
    launch_reduce(ctx->stream, ctx->nv, ctx->np, ctx->vel, ctx->force, ctx->energy, ctx->p_energy,
                  inter_kind(ctx) == INT_SMOOTH, ctx->partials, ctx->status,
                  std::min(2048, std::max(1, (ctx->nv + 255) / 256)));
    ctx->launches++;
    CR_TRY(cudaGetLastError());
  }
  if ((rc = clear_flags(ctx))) return rc;
  if (steps_eligible(ctx, kind, nsteps)) return run_steps(ctx, kind, nsteps);
  const long chunk = 128;
  std::vector<std::vector<Op>> plan;
  std::vector<long> sizes;
  {
    int b = ctx->cur;
    for (long done = 0; done < nsteps;) {
      const long n = std::min(chunk, nsteps - done);
      const int keep = ctx->cur;
      ctx->cur = b;
      plan.push_back(make_ops(ctx, kind, n));
      ctx->cur = keep;
      sizes.push_back(n);
      b = plan.back().back().out_buf;
      done += n;
    }
  }
  size_t c = 0;
  while (c < plan.size()) {
    const long long ops0 = ctx->status_h->ops_done;
    size_t c_end = c;
    if (kind == KIND_FIRE) {
      if ((rc = launch_chunk(ctx, plan[c], kind, sizes[c]))) return rc;
      c_end = c + 1;
    } else {
      for (c_end = c; c_end < plan.size(); c_end++)
        if ((rc = launch_chunk(ctx, plan[c_end], kind, sizes[c_end]))) return rc;
    }
    if ((rc = read_status(ctx))) return rc;
    if (ctx->status_h->abort) {
      // a stalled one-launch build (its CTAs were not all resident) is
      // resumed like an overflowed one, one launch per op from here on
      const bool stall = ctx->status_h->stalled != 0;
      if (stall) enter_degraded(ctx);
      else if (ctx->status_h->nonfinite) return ctx->fail(CR_ENONFINITE, "non-finite force during the step sequence");
      else if (!ctx->status_h->overflow) return ctx->fail(CR_ECUDA, "step sequence aborted");
      // locate the op after which the failed build ran (builds are not ops)
      long long k = ctx->status_h->ops_done - ops0;
      size_t j = c;
      while (j < c_end && k >= (long long)plan[j].size()) k -= (long long)plan[j++].size();
      if (j >= c_end || k == 0) return ctx->fail(CR_ECUDA, "inconsistent op counter after abort");
      if ((rc = clear_flags(ctx))) return rc;
      if (!stall) ctx->cap = 0;  // build_list grows from the measured count
      if ((rc = build_list(ctx, plan[j][(size_t)k - 1].check_buf, ctx->cut_distance))) return rc;
      if ((rc = clear_flags(ctx))) return rc;
      // the failed build was a displacement-triggered rebuild: count it, as the
      // in-graph build would have (DPM2D::checkDisplacement's updateCount)
      ctx->status_h->update_count += 1;
      if ((rc = upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus)))) return rc;
      if ((rc = run_direct(ctx, plan[j], (size_t)k, kind))) return rc;
      if (ctx->status_h->nonfinite)
        return ctx->fail(CR_ENONFINITE, "non-finite force after resuming from a neighbour-list overflow");
      if (ctx->status_h->abort) return ctx->fail(CR_ENBR_OVERFLOW, "neighbour list overflow during resume");
      c = j + 1;
      continue;
    }
    c = c_end;
    if (kind == KIND_FIRE && ctx->status_h->converged) break;
  }
  ctx->cur = plan[std::min(c, plan.size()) - 1].back().out_buf;
  if (ctx->status_h->max_ever > 0)
    ctx->list_size_ref = std::max<long long>(ctx->list_size_ref, pow2ceil(ctx->status_h->max_ever));
  return CR_OK;
}

int check_ctx(const cr_ctx* ctx) { return ctx ? CR_OK : CR_EINVAL; }

// Tiles: consecutive whole rings up to the tile capacity of the lane count.
void make_tiles(cr_ctx* ctx) {
  const int tv = tile_vertices(ctx->lanes);
  ctx->tiles_h.clear();
  int r = 0;
  while (r < ctx->np) {
    int r1 = r, cnt = 0;
    while (r1 < ctx->np && cnt + ctx->ring_nv_h[r1] <= tv) cnt += ctx->ring_nv_h[r1++];
    ctx->tiles_h.push_back(make_int4(r, r1, ctx->ring_first_h[r], ctx->ring_first_h[r] + cnt));
    r = r1;
  }
}

int set_current_device(cr_ctx* ctx) {
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->fail(CR_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  return CR_OK;
}

int upload(cr_ctx* ctx, void* dst, const void* src, size_t bytes) {
  if (!src) return ctx->fail(CR_EINVAL, "NULL host pointer");
  CR_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int download(const cr_ctx* cctx, void* dst, const void* src, size_t bytes) {
  cr_ctx* ctx = const_cast<cr_ctx*>(cctx);
  if (!dst) return ctx->fail(CR_EINVAL, "NULL host pointer");
  CR_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

// double AoS <-> double2 internal: identical memory layout.
static_assert(sizeof(double2) == 2 * sizeof(double), "double2 layout");

}  // namespace

// =========================================================================== C ABI
extern "C" {

int cr_create(long numParticles, const long* nvList, cr_ctx** out) {
  if (!out || numParticles <= 0 || !nvList) return CR_EINVAL;
  *out = nullptr;
  cr_ctx* ctx = new cr_ctx();
  int rc;
  cudaError_t e = cudaGetDevice(&ctx->device);
  if (e != cudaSuccess) {
    delete ctx;
    return CR_ECUDA;
  }
  ctx->np = (int)numParticles;
  long total = 0;
  int maxnv = 0;
  for (long q = 0; q < numParticles; q++) {
    if (nvList[q] < 3) {
      delete ctx;
      return CR_EINVAL;
    }
    ctx->ring_first_h.push_back((int)total);
    ctx->ring_nv_h.push_back((int)nvList[q]);
    total += nvList[q];
    maxnv = std::max(maxnv, (int)nvList[q]);
  }
  if (total >= (1L << 30)) {
    delete ctx;
    return CR_EINVAL;
  }
  ctx->nv = (int)total;
  ctx->lanes = maxnv > tile_vertices(2) ? 1 : 2;
  if (maxnv > tile_vertices(1)) {
    delete ctx;
    return CR_ENOTSUP;
  }
  ctx->ring_of_h.resize(total);
  std::vector<int2> pp(total), vtopo(total);
  std::vector<int> pqp(total);
  for (int q = 0; q < ctx->np; q++) {
    const int f = ctx->ring_first_h[q], n = ctx->ring_nv_h[q];
    for (int k = 0; k < n; k++) {
      ctx->ring_of_h[f + k] = q;
      const int prev = f + (k == 0 ? n - 1 : k - 1);
      const int k2 = (k - 2 + 2 * n) % n;
      pp[f + k] = make_int2(prev, f + k2);
      vtopo[f + k] = make_int2(q, k | (n << 16));
      pqp[f + k] = pq_pack_of(prev - (f + k), (f + k2) - (f + k));
    }
  }
  make_tiles(ctx);
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    delete ctx;
    return CR_ECUDA;
  }
  ctx->fused_max = nbr_fused_max_blocks();
  if (ctx->fused_max <= 0) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CR_ECUDA;
  }
  const size_t nv = total, np = numParticles;
  if ((rc = dalloc(ctx, &ctx->pos[0], nv)) || (rc = dalloc(ctx, &ctx->pos[1], nv)) ||
      (rc = dalloc(ctx, &ctx->vel, nv)) || (rc = dalloc(ctx, &ctx->force, nv)) ||
      (rc = dalloc(ctx, &ctx->last_pos, nv)) || (rc = dalloc(ctx, &ctx->ppos, np)) ||
      (rc = dalloc(ctx, &ctx->rad, nv)) || (rc = dalloc(ctx, &ctx->l0, nv)) || (rc = dalloc(ctx, &ctx->theta0, nv)) ||
      (rc = dalloc(ctx, &ctx->a0, np)) || (rc = dalloc(ctx, &ctx->energy, nv)) ||
      (rc = dalloc(ctx, &ctx->p_energy, np)) || (rc = dalloc(ctx, &ctx->theta, nv)) ||
      (rc = dalloc(ctx, &ctx->length, nv)) || (rc = dalloc(ctx, &ctx->area, np)) ||
      (rc = dalloc(ctx, &ctx->perimeter, np)) || (rc = dalloc(ctx, &ctx->p_angle, np)) ||
      (rc = dalloc(ctx, &ctx->vertex_area, np)) || (rc = dalloc(ctx, &ctx->ring_of, nv)) ||
      (rc = dalloc(ctx, &ctx->ring_first, np)) || (rc = dalloc(ctx, &ctx->ring_nv, np)) ||
      (rc = dalloc(ctx, &ctx->zero_cnt, nv)) || (rc = dalloc(ctx, &ctx->pp_of, nv)) ||
      (rc = dalloc(ctx, &ctx->tiles, ctx->tiles_h.size())) || (rc = dalloc(ctx, &ctx->nbr_cnt, nv)) ||
      (rc = dalloc(ctx, &ctx->cell_of, nv)) || (rc = dalloc(ctx, &ctx->slot, nv)) ||
      (rc = dalloc(ctx, &ctx->cell_vid, nv)) || (rc = dalloc(ctx, &ctx->cell_ring, nv)) ||
      (rc = dalloc(ctx, &ctx->cell_pq, nv)) || (rc = dalloc(ctx, &ctx->vtopo, nv)) ||
      (rc = dalloc(ctx, &ctx->pq_pack, nv)) ||
      (rc = dalloc(ctx, &ctx->cell_pos, nv)) || (rc = dalloc(ctx, &ctx->cell_rad, nv)) ||
      (rc = dalloc(ctx, &ctx->status, 1)) || (rc = dalloc(ctx, &ctx->fire_state, 8)) ||
      (rc = dalloc(ctx, &ctx->block_sum, std::max(1, ctx->fused_max))) ||
      (rc = dalloc(ctx, &ctx->p_vel, np)) || (rc = dalloc(ctx, &ctx->p_force, np)) ||
      (rc = dalloc(ctx, &ctx->p_angvel, np)) || (rc = dalloc(ctx, &ctx->p_torque, np)) ||
      (rc = dalloc(ctx, &ctx->p_moi, np)) || (rc = dalloc(ctx, &ctx->v_torque, nv)) ||
      (rc = dalloc(ctx, &ctx->sp_angle, np))) {
    cr_destroy(ctx);
    return rc;
  }
  if ((rc = alloc_lists(ctx, 16))) {
    cr_destroy(ctx);
    return rc;
  }
  if (cudaMallocHost((void**)&ctx->status_h, sizeof(DevStatus)) != cudaSuccess) {
    cr_destroy(ctx);
    return CR_ENOMEM;
  }
  memset(ctx->status_h, 0, sizeof(DevStatus));
  if (upload(ctx, ctx->ring_of, ctx->ring_of_h.data(), nv * sizeof(int)) ||
      upload(ctx, ctx->ring_first, ctx->ring_first_h.data(), np * sizeof(int)) ||
      upload(ctx, ctx->ring_nv, ctx->ring_nv_h.data(), np * sizeof(int)) ||
      upload(ctx, ctx->pp_of, pp.data(), nv * sizeof(int2)) ||
      upload(ctx, ctx->vtopo, vtopo.data(), nv * sizeof(int2)) ||
      upload(ctx, ctx->pq_pack, pqp.data(), nv * sizeof(int)) ||
      upload(ctx, ctx->tiles, ctx->tiles_h.data(), ctx->tiles_h.size() * sizeof(int4))) {
    cr_destroy(ctx);
    return CR_ECUDA;
  }
  // reference defaults (src/DPM2D.cu:41-95)
  ctx->p.lx = ctx->p.ly = 1.0;
  ctx->p.ea = 1e5;
  ctx->p.el = 20;
  ctx->p.eb = 10;
  ctx->p.ec = 1;
  ctx->dt = 1e-3;
  refresh_params(ctx);
  if (ensure_partials(ctx)) {
    cr_destroy(ctx);
    return CR_ENOMEM;
  }
  *out = ctx;
  return CR_OK;
}

int cr_destroy(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  void* ptrs[] = {ctx->pos[0], ctx->pos[1], ctx->vel, ctx->force, ctx->last_pos, ctx->ppos, ctx->rad, ctx->l0,
                  ctx->theta0, ctx->a0, ctx->energy, ctx->p_energy, ctx->theta, ctx->length, ctx->area,
                  ctx->perimeter, ctx->p_angle, ctx->vertex_area, ctx->ring_of, ctx->ring_first, ctx->ring_nv,
                  ctx->zero_cnt, ctx->pp_of, ctx->vtopo, ctx->pq_pack, ctx->nbr_pq, ctx->cell_pq,
                  ctx->tiles, ctx->nbr, ctx->nbr_cnt, ctx->cell_of, ctx->slot,
                  ctx->cell_cnt, ctx->cell_start, ctx->cell_vid, ctx->cell_ring, ctx->cell_pos, ctx->cell_rad,
                  ctx->partials, ctx->status, ctx->fire_state, ctx->p_vel, ctx->p_force, ctx->p_angvel,
                  ctx->diff_f, ctx->diff_e, ctx->diff_dot, ctx->diff_vec, ctx->diff_area, ctx->cg_state,
                  ctx->cg_part, ctx->cg_minv,
                  ctx->p_torque, ctx->p_moi, ctx->v_torque, ctx->sp_angle, ctx->block_sum, ctx->cell_bucket, ctx->bucket_pos, ctx->bucket_rad,
                  ctx->bucket_ring, ctx->bucket_pq,
                  ctx->prad, ctx->plast, ctx->pid, ctx->pnbr, ctx->pnbr_cnt, ctx->pstatus, ctx->pfire, ctx->pdraws,
                  ctx->snap_pos, ctx->snap_vel, ctx->snap_force, ctx->snap_last, ctx->snap_angle};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->status_h) cudaFreeHost(ctx->status_h);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CR_OK;
}

const char* cr_last_error(const cr_ctx* ctx) { return ctx ? ctx->err.c_str() : "NULL context"; }

int cr_get_num_vertices(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = ctx->nv;
  return CR_OK;
}
int cr_get_num_particles(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = ctx->np;
  return CR_OK;
}

#define CR_ENUM_SETTER(name, field, lo, hi)                                   \
  int name(cr_ctx* ctx, int v) {                                             \
    if (!ctx) return CR_EINVAL;                                              \
    if (v < (lo) || v > (hi)) return ctx->fail(CR_EINVAL, #name ": bad value"); \
    ctx->field = v;                                                          \
    refresh_params(ctx);                                                     \
    drop_graphs(ctx);                                                        \
    return CR_OK;                                                            \
  }
CR_ENUM_SETTER(cr_set_potential_type, potential, 0, 3)
CR_ENUM_SETTER(cr_set_monomer_type, monomer, 0, 1)
CR_ENUM_SETTER(cr_set_noise_type, noise_type, 0, 3)
CR_ENUM_SETTER(cr_set_shape_type, shape, 0, 1)

int cr_set_interaction_type(cr_ctx* ctx, int v) {
  if (!ctx) return CR_EINVAL;
  if (v < 0 || v > 3) return ctx->fail(CR_EINVAL, "cr_set_interaction_type: bad value");
  if (v == CR_INTERACTION_ALL)
    return ctx->fail(CR_ENOTSUP, "interactionEnum::all (O(N^2) debug path) is served by the neighbour list path");
  ctx->interaction = v;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_particle_type(cr_ctx* ctx, int v) {
  if (!ctx) return CR_EINVAL;
  if (v < 0 || v > 2) return ctx->fail(CR_EINVAL, "cr_set_particle_type: bad value");
  if (v == CR_PARTICLE_ACTIVE_SHAPE)
    return ctx->fail(CR_ENOTSUP, "activeShape (rest-length noise) is not on the accelerated path");
  ctx->particle = v;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_geometry_type(cr_ctx* ctx, int v) {
  if (!ctx) return CR_EINVAL;
  if (v != CR_GEOMETRY_NORMAL) return ctx->fail(CR_ENOTSUP, "only periodic geometry is supported");
  ctx->geometry = v;
  return CR_OK;
}

int cr_set_box_size(cr_ctx* ctx, const double* box) {
  if (!ctx || !box || !(box[0] > 0) || !(box[1] > 0)) return ctx ? ctx->fail(CR_EINVAL, "bad box") : CR_EINVAL;
  ctx->p.lx = box[0];
  ctx->p.ly = box[1];
  refresh_params(ctx);
  drop_graphs(ctx);
  return CR_OK;
}
int cr_get_box_size(const cr_ctx* ctx, double* box) {
  if (!ctx || !box) return CR_EINVAL;
  box[0] = ctx->p.lx;
  box[1] = ctx->p.ly;
  return CR_OK;
}

int cr_set_energy_costs(cr_ctx* ctx, double ea, double el, double eb, double ec) {
  if (!ctx) return CR_EINVAL;
  ctx->p.ea = ea;
  ctx->p.el = el;
  ctx->p.eb = eb;
  ctx->p.ec = ec;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_lj_cutoff(cr_ctx* ctx, double c) {
  if (!ctx || !(c > 0)) return ctx ? ctx->fail(CR_EINVAL, "bad LJ cutoff") : CR_EINVAL;
  ctx->p.lj_cutoff = c;
  const double ratio6 = 1 / std::pow(c, 6);
  ctx->p.lj_ecut = 4 * ctx->p.ec * (ratio6 * ratio6 - ratio6);
  ctx->p.lj_fshift = 24 * ctx->p.ec * (2 * ratio6 - 1) * ratio6 / c;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_attraction_constants(cr_ctx* ctx, double l1, double l2) {
  if (!ctx) return CR_EINVAL;
  ctx->p.l1 = l1;
  ctx->p.l2 = l2;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_fene_constants(cr_ctx* ctx, double stiff, double ext) {
  if (!ctx) return CR_EINVAL;
  ctx->p.stiff = stiff;
  ctx->p.ext_sq = ext * ext;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_time_step(cr_ctx* ctx, double dt) {
  if (!ctx || !(dt > 0)) return ctx ? ctx->fail(CR_EINVAL, "bad dt") : CR_EINVAL;
  ctx->dt = dt;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_self_propulsion_params(cr_ctx* ctx, double driving, double taup) {
  if (!ctx) return CR_EINVAL;
  ctx->driving = driving;
  ctx->taup = taup;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_set_seed(cr_ctx* ctx, unsigned long long seed) {
  if (!ctx) return CR_EINVAL;
  ctx->seed = seed;
  drop_graphs(ctx);
  return CR_OK;
}

#define CR_NV2 ((size_t)ctx->nv * sizeof(double2))
#define CR_NV1 ((size_t)ctx->nv * sizeof(double))
#define CR_NP1 ((size_t)ctx->np * sizeof(double))

int cr_set_vertex_positions(cr_ctx* ctx, const double* pos) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->pos[ctx->cur], pos, CR_NV2);
}
int cr_get_vertex_positions(const cr_ctx* ctx, double* pos) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, pos, ctx->pos[ctx->cur], CR_NV2);
}
int cr_set_vertex_velocities(cr_ctx* ctx, const double* vel) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->vel, vel, CR_NV2);
}
int cr_get_vertex_velocities(const cr_ctx* ctx, double* vel) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, vel, ctx->vel, CR_NV2);
}
int cr_get_vertex_forces(const cr_ctx* ctx, double* f) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, f, ctx->force, CR_NV2);
}
int cr_set_vertex_forces(cr_ctx* ctx, const double* f) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->force, f, CR_NV2);
}
int cr_get_vertex_energies(const cr_ctx* ctx, double* e) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, e, ctx->energy, CR_NV1);
}
int cr_get_particle_energies(const cr_ctx* ctx, double* e) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, e, ctx->p_energy, CR_NP1);
}
int cr_set_vertex_radii(cr_ctx* ctx, const double* rad) {
  if (!ctx) return CR_EINVAL;
  int rc = upload(ctx, ctx->rad, rad, CR_NV1);
  if (rc == CR_OK) {
    update_rmax(ctx, rad);
    drop_graphs(ctx);
  }
  return rc;
}
int cr_get_vertex_radii(const cr_ctx* ctx, double* rad) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, rad, ctx->rad, CR_NV1);
}
int cr_set_rest_areas(cr_ctx* ctx, const double* a0) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->a0, a0, CR_NP1);
}
int cr_get_rest_areas(const cr_ctx* ctx, double* a0) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, a0, ctx->a0, CR_NP1);
}
int cr_set_rest_lengths(cr_ctx* ctx, const double* l0) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->l0, l0, CR_NV1);
}
int cr_get_rest_lengths(const cr_ctx* ctx, double* l0) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, l0, ctx->l0, CR_NV1);
}
int cr_set_rest_angles(cr_ctx* ctx, const double* t0) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->theta0, t0, CR_NV1);
}
int cr_get_rest_angles(const cr_ctx* ctx, double* t0) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, t0, ctx->theta0, CR_NV1);
}
int cr_get_areas(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->area, CR_NP1);
}
int cr_get_perimeters(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->perimeter, CR_NP1);
}
int cr_get_segment_lengths(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->length, CR_NV1);
}
int cr_get_segment_angles(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->theta, CR_NV1);
}
int cr_calc_particle_shape(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  // geometry pass only: the force outputs are restored afterwards by keeping
  // them out of this pass (a zero-length neighbour list and a scratch force)
  double2* keep_force = ctx->force;
  double* keep_energy = ctx->energy;
  double* keep_pe = ctx->p_energy;
  double2* tmpf = nullptr;
  double* tmpe = nullptr;
  double* tmpp = nullptr;
  CR_TRY(cudaMallocAsync((void**)&tmpf, CR_NV2, ctx->stream));
  CR_TRY(cudaMallocAsync((void**)&tmpe, CR_NV1, ctx->stream));
  CR_TRY(cudaMallocAsync((void**)&tmpp, CR_NP1, ctx->stream));
  ctx->force = tmpf;
  ctx->energy = tmpe;
  ctx->p_energy = tmpp;
  int particle = ctx->particle;
  ctx->particle = CR_PARTICLE_PASSIVE;
  int rc = force_pass(ctx, true);
  ctx->particle = particle;
  ctx->force = keep_force;
  ctx->energy = keep_energy;
  ctx->p_energy = keep_pe;
  cudaFreeAsync(tmpf, ctx->stream);
  cudaFreeAsync(tmpe, ctx->stream);
  cudaFreeAsync(tmpp, ctx->stream);
  if (rc) return rc;
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}
int cr_calc_particle_positions(cr_ctx* ctx) { return cr_calc_particle_shape(ctx); }
int cr_get_particle_positions(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->ppos, (size_t)ctx->np * sizeof(double2));
}
int cr_set_particle_positions(cr_ctx* ctx, const double* pp) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->ppos, pp, (size_t)ctx->np * sizeof(double2));
}

int cr_set_displacement_cutoff(cr_ctx* ctx, double cutoff, double size, double* cut_out) {
  if (!ctx) return CR_EINVAL;
  // DPM2D::setDisplacementCutoff (src/DPM2D.cu:1300-1329)
  double base = 1.0;
  switch (ctx->potential) {
    case CR_POTENTIAL_HARMONIC: base = 1.0; break;
    case CR_POTENTIAL_LENNARD_JONES: base = ctx->p.lj_cutoff; break;
    case CR_POTENTIAL_WCA: base = kWCAcut; break;
    case CR_POTENTIAL_ADHESIVE: base = 1.0 + ctx->p.l2; break;
  }
  ctx->cut_distance = base + cutoff;
  ctx->cutoff = cutoff * size;
  drop_graphs(ctx);
  if (cut_out) *cut_out = ctx->cut_distance;
  return CR_OK;
}

int cr_calc_neighbor_list(cr_ctx* ctx, double cut) {
  if (!ctx) return CR_EINVAL;
  int rc = clear_flags(ctx);
  if (rc) return rc;
  return build_list(ctx, ctx->cur, cut);
}

int cr_reset_last_positions(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  CR_TRY(cudaMemcpyAsync(ctx->last_pos, ctx->pos[ctx->cur], CR_NV2, cudaMemcpyDeviceToDevice, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int cr_check_neighbors(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc;
  if ((rc = clear_flags(ctx))) return rc;
  std::vector<Op> ops{Op{OP_CHECK, ctx->cur, ctx->cur, 0, 1, ctx->cur}};
  if ((rc = run_direct(ctx, ops, 0, KIND_NVE))) return rc;
  return CR_OK;
}

int cr_get_neighbor_list_size(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = (long)ctx->list_size_ref;
  return CR_OK;
}

int cr_get_max_neighbor_list(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<int> cnt(ctx->nv);
  int rc = download(ctx, cnt.data(), ctx->nbr_built ? ctx->nbr_cnt : ctx->zero_cnt, ctx->nv * sizeof(int));
  if (rc) return rc;
  for (int i = 0; i < ctx->nv; i++) out[i] = cnt[i];
  return CR_OK;
}

int cr_get_neighbors(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  const long ls = ctx->list_size_ref;
  if (ls == 0) return CR_OK;
  std::vector<int> cnt(ctx->nv), nb((size_t)ctx->cap * ctx->nv);
  int rc;
  if ((rc = download(ctx, cnt.data(), ctx->nbr_built ? ctx->nbr_cnt : ctx->zero_cnt, ctx->nv * sizeof(int)))) return rc;
  if ((rc = download(ctx, nb.data(), ctx->nbr, nb.size() * sizeof(int)))) return rc;
  std::vector<int> row;
  for (int i = 0; i < ctx->nv; i++) {
    row.clear();
    for (int s = 0; s < std::min(cnt[i], ctx->cap); s++) row.push_back(nb[(size_t)s * ctx->nv + i]);
    std::sort(row.begin(), row.end());
    for (long s = 0; s < ls; s++) out[(size_t)i * ls + s] = s < (long)row.size() ? row[s] : -1;
  }
  return CR_OK;
}

int cr_get_update_count(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  cr_ctx* c = const_cast<cr_ctx*>(ctx);
  int rc = read_status(c);
  if (rc) return rc;
  *out = (long)c->status_h->update_count;
  return CR_OK;
}

int cr_reset_update_count(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc = read_status(ctx);
  if (rc) return rc;
  ctx->status_h->update_count = 0;
  return upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus));
}

int cr_calc_force_energy(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc = force_pass(ctx, false);
  if (rc) return rc;
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int cr_get_potential_energy(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = ctx->status_h->sums[S_PE];
  return CR_OK;
}
int cr_get_kinetic_energy(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = 0.5 * ctx->status_h->sums[S_VV];
  return CR_OK;
}
int cr_get_energy(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = ctx->status_h->sums[S_PE] + 0.5 * ctx->status_h->sums[S_VV];
  return CR_OK;
}
int cr_get_temperature(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = 2.0 * (0.5 * ctx->status_h->sums[S_VV]) / (ctx->nv * 2.0);
  return CR_OK;
}
int cr_get_max_unbalanced_force(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = std::sqrt(ctx->status_h->sums[S_FMAX2]);
  return CR_OK;
}
int cr_get_total_force_magnitude(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = reduce_now(ctx);
  if (rc) return rc;
  *out = std::sqrt(ctx->status_h->sums[S_FF] / (ctx->nv * 2.0));
  return CR_OK;
}

static int phi_common(cr_ctx* ctx, const double* ring_area_dev, double* out) {
  std::vector<double> ar(ctx->np), va(ctx->np);
  launch_vertex_area(ctx->stream, ctx->np, ctx->ring_first, ctx->ring_nv, ctx->rad, ctx->vertex_area);
  ctx->launches++;
  int rc;
  if ((rc = download(ctx, ar.data(), ring_area_dev, CR_NP1))) return rc;
  if ((rc = download(ctx, va.data(), ctx->vertex_area, CR_NP1))) return rc;
  double s = 0.0, v = 0.0;
  for (int q = 0; q < ctx->np; q++) s += ar[q];
  for (int q = 0; q < ctx->np; q++) v += va[q];
  *out = (s + kPi * v) / (ctx->p.lx * ctx->p.ly);
  return CR_OK;
}
int cr_get_phi(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  return phi_common(ctx, ctx->area, out);
}
int cr_get_preferred_phi(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  return phi_common(ctx, ctx->a0, out);
}
int cr_get_mean_vertex_radius(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<double> r(ctx->nv);
  int rc = download(ctx, r.data(), ctx->rad, CR_NV1);
  if (rc) return rc;
  double s = 0;
  for (double x : r) s += x;
  *out = s / ctx->nv;
  return CR_OK;
}
int cr_get_mean_particle_size(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<double> a(ctx->np);
  int rc = download(ctx, a.data(), ctx->a0, CR_NP1);
  if (rc) return rc;
  double s = 0;
  for (double x : a) s += x;
  *out = 2 * std::sqrt(s / (kPi * ctx->np));  // src/DPM2D.cu:781-783
  return CR_OK;
}

int cr_scale_vertices(cr_ctx* ctx, double scale) {
  if (!ctx || !(scale > 0)) return ctx ? ctx->fail(CR_EINVAL, "bad scale") : CR_EINVAL;
  launch_scale_vertices(ctx->stream, ctx->nv, ctx->np, ctx->ring_of, ctx->ppos, ctx->pos[ctx->cur], ctx->a0,
                        ctx->area, ctx->l0, ctx->rad, scale);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->rmax *= scale;
  drop_graphs(ctx);
  return CR_OK;
}

static int reset_rng_step(cr_ctx* ctx) {
  int rc = read_status(ctx);
  if (rc) return rc;
  ctx->status_h->rng_step = 0;
  return upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus));
}

int cr_init_nve(cr_ctx* ctx, double T, int readState) {
  if (!ctx) return CR_EINVAL;
  // DPM2D::initNVE (src/DPM2D.cu:3760-3771): lastPos = pos, KE injection
  int rc = cr_reset_last_positions(ctx);
  if (rc) return rc;
  if ((rc = reset_rng_step(ctx))) return rc;
  ctx->sim_kind = KIND_NVE;
  ctx->T = T;
  if (!readState) {
    launch_inject_ke(ctx->stream, ctx->nv, ctx->ring_of, ctx->vel, std::sqrt(T), ctx->seed, (1ull << 61) + ctx->rng_calls++);
    ctx->launches++;
    CR_TRY(cudaGetLastError());
    CR_TRY(cudaStreamSynchronize(ctx->stream));
  }
  drop_graphs(ctx);
  return CR_OK;
}

int cr_init_nve_rescale(cr_ctx* ctx, double T) {
  if (!ctx) return CR_EINVAL;
  if (!(T > 0.0)) return ctx->fail(CR_EINVAL, "NVERescale needs a positive temperature");
  // DPM2D::initNVERescale (src/DPM2D.cu:3778-3817): lastPos = pos, ring-rigid
  // thermal velocities at amplitude sqrt(T), then scaled to T exactly
  int rc = cr_reset_last_positions(ctx);
  if (rc) return rc;
  if ((rc = reset_rng_step(ctx))) return rc;
  ctx->sim_kind = KIND_NVE_RESCALE;
  ctx->T = T;
  launch_inject_ke(ctx->stream, ctx->nv, ctx->ring_of, ctx->vel, std::sqrt(T), ctx->seed, (1ull << 61) + ctx->rng_calls++);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  if ((rc = reduce_now(ctx))) return rc;
  const double Tcur = ctx->status_h->sums[S_VV] / (2.0 * ctx->nv);
  if (!(Tcur > 0.0)) return ctx->fail(CR_ENONFINITE, "zero kinetic energy after the thermal draw");
  launch_affine_vel(ctx->stream, ctx->nv, ctx->vel, std::sqrt(T / Tcur), make_double2(0.0, 0.0));
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  return CR_OK;
}

int cr_nve_rescale_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (ctx->sim_kind != KIND_NVE_RESCALE) return ctx->fail(CR_ESTATE, "cr_nve_rescale_loop before cr_init_nve_rescale");
  if (nsteps == 0) return CR_OK;
  return run_ops(ctx, KIND_NVE_RESCALE, nsteps);
}

int cr_conserve_momentum(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc;
  if (ctx->shape == CR_SHAPE_RIGID) {
    // RigidLangevin / RigidNVE::conserveMomentum (src/Simulator.cu:309-312,
    // 368-371): the mean ring velocity is removed (over every ring; the
    // reference's single-CTA kernel covers only its first block of rings)
    std::vector<double2> pv(ctx->np);
    if ((rc = download(ctx, pv.data(), ctx->p_vel, ctx->np * sizeof(double2)))) return rc;
    double mx = 0.0, my = 0.0;
    for (const double2& u : pv) { mx += u.x; my += u.y; }
    launch_affine_vel(ctx->stream, ctx->np, ctx->p_vel, 1.0, make_double2(-mx / ctx->np, -my / ctx->np));
  } else {
    // Langevin::conserveMomentum (src/Simulator.cu:91-108): the mean vertex
    // velocity is removed
    std::vector<double2> v(ctx->nv);
    if ((rc = download(ctx, v.data(), ctx->vel, ctx->nv * sizeof(double2)))) return rc;
    double mx = 0.0, my = 0.0;
    for (const double2& u : v) { mx += u.x; my += u.y; }
    launch_affine_vel(ctx->stream, ctx->nv, ctx->vel, 1.0, make_double2(-mx / ctx->nv, -my / ctx->nv));
  }
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int cr_nve_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (ctx->sim_kind != KIND_NVE) return ctx->fail(CR_ESTATE, "cr_nve_loop before cr_init_nve");
  if (nsteps == 0) return CR_OK;
  return run_ops(ctx, KIND_NVE, nsteps);
}

int cr_init_langevin(cr_ctx* ctx, double T, double gamma, int readState) {
  if (!ctx) return CR_EINVAL;
  // DPM2D::initLangevin (src/DPM2D.cu:3713-3753)
  ctx->T = T;
  switch (ctx->noise_type) {
    case CR_NOISE_LANGEVIN:
      ctx->sim_kind = KIND_LANGEVIN;
      ctx->gamma = gamma;
      ctx->noise = std::sqrt(2.0 * T * gamma / ctx->dt);
      break;
    case CR_NOISE_BAOAB:
      ctx->sim_kind = KIND_BAOAB;
      ctx->gamma_factor = std::exp(-gamma * ctx->dt);
      ctx->noise = std::sqrt(1 - std::exp(-2 * gamma * ctx->dt)) * std::sqrt(T);
      break;
    case CR_NOISE_BROWNIAN:
      ctx->sim_kind = KIND_BROWNIAN;
      ctx->gamma = gamma;
      ctx->noise = std::sqrt(2.0 * T * gamma / ctx->dt);
      break;
    default:
      ctx->sim_kind = KIND_DRIVEN_BROWNIAN;
      ctx->gamma = gamma;
      ctx->noise = std::sqrt(2.0 * T * gamma / ctx->dt);
      break;
  }
  int rc = cr_reset_last_positions(ctx);
  if (rc) return rc;
  if ((rc = reset_rng_step(ctx))) return rc;
  if (!readState) {
    launch_inject_ke(ctx->stream, ctx->nv, ctx->ring_of, ctx->vel, std::sqrt(T), ctx->seed, (1ull << 61) + ctx->rng_calls++);
    ctx->launches++;
    CR_TRY(cudaGetLastError());
    CR_TRY(cudaStreamSynchronize(ctx->stream));
  }
  drop_graphs(ctx);
  return CR_OK;
}

int cr_langevin_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (ctx->sim_kind < KIND_LANGEVIN || ctx->sim_kind > KIND_DRIVEN_BROWNIAN)
    return ctx->fail(CR_ESTATE, "cr_langevin_loop before cr_init_langevin");
  if (nsteps == 0) return CR_OK;
  return run_ops(ctx, ctx->sim_kind, nsteps);
}

int cr_init_fire(cr_ctx* ctx, const double* prm, long minStep, long numStep, long numDOF) {
  if (!ctx || !prm) return CR_EINVAL;
  (void)numDOF;
  ctx->fp.a_start = prm[0];
  ctx->fp.f_dec = prm[1];
  ctx->fp.f_inc = prm[2];
  ctx->fp.f_a = prm[3];
  ctx->fp.dt_max = prm[5];
  ctx->fp.min_step = minStep;
  ctx->fp.tol = -1.0;
  double st[8] = {prm[4], prm[6], (double)numStep, 0, prm[4], prm[6], (double)numStep, 0};
  int rc = upload(ctx, ctx->fire_state, st, sizeof(st));
  if (rc) return rc;
  if ((rc = read_status(ctx))) return rc;
  ctx->status_h->fire_iters = 0;
  if ((rc = upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus)))) return rc;
  ctx->fire_ready = true;
  ctx->sim_kind = KIND_FIRE;
  drop_graphs(ctx);
  return CR_OK;
}

static int fire_run(cr_ctx* ctx, long nsteps, double tol) {
  int rc;
  ctx->fp.tol = tol;
  drop_graphs(ctx);
  if ((rc = reduce_now(ctx))) return rc;  // P, |v|^2, |F|^2 of the current state
  if ((rc = clear_flags(ctx))) return rc;
  if (tol >= 0 && ctx->status_h->sums[S_FMAX2] <= tol * tol) return CR_OK;
  return run_ops(ctx, KIND_FIRE, nsteps);
}

int cr_vertex_fire_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (!ctx->fire_ready) return ctx->fail(CR_ESTATE, "cr_vertex_fire_loop before cr_init_fire");
  if (nsteps == 0) return CR_OK;
  return fire_run(ctx, nsteps, -1.0);
}

int cr_fire_minimize(cr_ctx* ctx, double tol, long maxIter, long* iterations, double* maxForce) {
  if (!ctx || maxIter < 0) return CR_EINVAL;
  if (!ctx->fire_ready) return ctx->fail(CR_ESTATE, "cr_fire_minimize before cr_init_fire");
  int rc = read_status(ctx);
  if (rc) return rc;
  const long long it0 = ctx->status_h->fire_iters;
  rc = fire_run(ctx, maxIter, tol);
  if (rc) return rc;
  if ((rc = read_status(ctx))) return rc;
  if (iterations) *iterations = (long)(ctx->status_h->fire_iters - it0);
  double m;
  if ((rc = cr_get_max_unbalanced_force(ctx, &m))) return rc;
  if (maxForce) *maxForce = m;
  return CR_OK;
}

int cr_get_fire_state(cr_ctx* ctx, double* out3) {
  if (!ctx || !out3) return CR_EINVAL;
  int rc = read_status(ctx);
  if (rc) return rc;
  double st[8];
  if ((rc = download(ctx, st, ctx->fire_state, sizeof(st)))) return rc;
  const int b = (int)(ctx->status_h->fire_iters & 1);
  out3[0] = st[b * 4];
  out3[1] = st[b * 4 + 1];
  out3[2] = st[b * 4 + 2];
  return CR_OK;
}

// ------------------------------------------------------------------ rigid rings

int cr_calc_rigid_force_energy(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  if (ctx->interaction != CR_INTERACTION_VERTEX_VERTEX)
    return ctx->fail(CR_ENOTSUP, "rigid rings run the vertex-vertex interaction");
  StepArgs s = base_args(ctx);
  s.kind = KIND_NONE;
  launch_rigid(tile_cfg(ctx), ctx->potential, MODE_FORCE, ctx->p, arrays(ctx, ctx->cur), s, rigid_args(ctx));
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

static int rigid_init(cr_ctx* ctx, double T, int readState) {
  // DPM2D::initRigidNVE / initRigidLangevin (src/DPM2D.cu:3793-3838): angles
  // and angular velocities start at zero, lastPos = pos, centroids current
  int rc;
  if (ctx->interaction != CR_INTERACTION_VERTEX_VERTEX)
    return ctx->fail(CR_ENOTSUP, "rigid rings run the vertex-vertex interaction");
  ctx->shape = CR_SHAPE_RIGID;
  if ((rc = cr_reset_last_positions(ctx))) return rc;
  if ((rc = reset_rng_step(ctx))) return rc;
  CR_TRY(cudaMemsetAsync(ctx->p_angle, 0, CR_NP1, ctx->stream));
  CR_TRY(cudaMemsetAsync(ctx->p_angvel, 0, CR_NP1, ctx->stream));
  if (!readState) {
    launch_rigid_inject(ctx->stream, ctx->np, ctx->p_vel, std::sqrt(T), ctx->seed, (1ull << 60) + ctx->rng_calls++);
    ctx->launches++;
    CR_TRY(cudaGetLastError());
  }
  if (!ctx->nbr_built && (rc = build_list(ctx, ctx->cur, ctx->cut_distance))) return rc;
  if ((rc = cr_calc_rigid_force_energy(ctx))) return rc;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_init_rigid_nve(cr_ctx* ctx, double T, int readState) {
  if (!ctx) return CR_EINVAL;
  int rc = rigid_init(ctx, T, readState);
  if (rc) return rc;
  ctx->sim_kind = KIND_NVE;
  ctx->T = T;
  return CR_OK;
}

int cr_rigid_nve_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (ctx->shape != CR_SHAPE_RIGID || ctx->sim_kind != KIND_NVE)
    return ctx->fail(CR_ESTATE, "cr_rigid_nve_loop before cr_init_rigid_nve");
  if (nsteps == 0) return CR_OK;
  return run_ops(ctx, KIND_NVE, nsteps);
}

int cr_init_rigid_langevin(cr_ctx* ctx, double T, double gamma, int readState) {
  if (!ctx) return CR_EINVAL;
  int rc = rigid_init(ctx, T, readState);
  if (rc) return rc;
  ctx->sim_kind = KIND_LANGEVIN;
  ctx->T = T;
  ctx->gamma = gamma;
  ctx->noise = std::sqrt(2.0 * T * gamma / ctx->dt);
  return CR_OK;
}

int cr_rigid_langevin_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (ctx->shape != CR_SHAPE_RIGID || ctx->sim_kind != KIND_LANGEVIN)
    return ctx->fail(CR_ESTATE, "cr_rigid_langevin_loop before cr_init_rigid_langevin");
  if (nsteps == 0) return CR_OK;
  return run_ops(ctx, KIND_LANGEVIN, nsteps);
}

int cr_get_particle_velocities(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->p_vel, (size_t)ctx->np * sizeof(double2));
}
int cr_set_particle_velocities(cr_ctx* ctx, const double* in) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->p_vel, in, (size_t)ctx->np * sizeof(double2));
}
int cr_get_particle_angles(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->p_angle, CR_NP1);
}
int cr_set_particle_angles(cr_ctx* ctx, const double* in) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->p_angle, in, CR_NP1);
}
int cr_get_particle_angular_velocities(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->p_angvel, CR_NP1);
}
int cr_set_particle_angular_velocities(cr_ctx* ctx, const double* in) {
  if (!ctx) return CR_EINVAL;
  return upload(ctx, ctx->p_angvel, in, CR_NP1);
}
int cr_get_particle_forces(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->p_force, (size_t)ctx->np * sizeof(double2));
}
int cr_get_particle_torques(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->p_torque, CR_NP1);
}
int cr_get_vertex_torques(const cr_ctx* ctx, double* out) {
  if (!ctx) return CR_EINVAL;
  return download(ctx, out, ctx->v_torque, CR_NV1);
}
int cr_get_particle_kinetic_energy(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<double> v(2 * (size_t)ctx->np);
  int rc = download(ctx, v.data(), ctx->p_vel, v.size() * sizeof(double));
  if (rc) return rc;
  double s = 0.0;
  for (double x : v) s += x * x;
  *out = 0.5 * s;  // DPM2D::getParticleKineticEnergy (src/DPM2D.cu:1101-1106)
  return CR_OK;
}

int cr_get_stream(const cr_ctx* ctx, void** out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = (void*)ctx->stream;
  return CR_OK;
}

int cr_profile_step_kernel(cr_ctx* ctx, long reps, double* ms_per_launch) {
  if (!ctx || reps <= 0 || !ms_per_launch) return CR_EINVAL;
  if (!ctx->nbr_built) return ctx->fail(CR_ESTATE, "cr_profile_step_kernel before a neighbour list exists");
  int rc;
  if ((rc = ensure_partials(ctx))) return rc;
  // scratch copies so the context state is untouched
  double2 *pos_s = nullptr, *vel_s = nullptr, *frc_s = nullptr;
  DevStatus* st_s = nullptr;
  CR_TRY(cudaMallocAsync((void**)&pos_s, CR_NV2, ctx->stream));
  CR_TRY(cudaMallocAsync((void**)&vel_s, CR_NV2, ctx->stream));
  CR_TRY(cudaMallocAsync((void**)&frc_s, CR_NV2, ctx->stream));
  CR_TRY(cudaMallocAsync((void**)&st_s, sizeof(DevStatus), ctx->stream));
  CR_TRY(cudaMemcpyAsync(vel_s, ctx->vel, CR_NV2, cudaMemcpyDeviceToDevice, ctx->stream));
  CR_TRY(cudaMemsetAsync(st_s, 0, sizeof(DevStatus), ctx->stream));
  StepArgs s = base_args(ctx);
  s.kind = ctx->sim_kind >= 0 && ctx->sim_kind != KIND_FIRE ? ctx->sim_kind : KIND_NVE;
  s.advance = 1;
  s.accumulate = 0;  // as in an NVE / Langevin step op
  s.active = 0;  // ring angles are state; the self-propulsion term is not timed here
  s.pos_out = pos_s;
  s.vel = vel_s;
  s.force = frc_s;
  s.status = st_s;
  const SysArrays a = arrays(ctx, ctx->cur);
  cudaEvent_t e0, e1;
  CR_TRY(cudaEventCreate(&e0));
  CR_TRY(cudaEventCreate(&e1));
  for (int w = 0; w < 3; w++) launch_tile(tile_cfg(ctx), ctx->potential, inter_kind(ctx), MODE_STEP, ctx->p, a, s);
  CR_TRY(cudaEventRecord(e0, ctx->stream));
  for (long r = 0; r < reps; r++) launch_tile(tile_cfg(ctx), ctx->potential, inter_kind(ctx), MODE_STEP, ctx->p, a, s);
  CR_TRY(cudaEventRecord(e1, ctx->stream));
  CR_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  CR_TRY(cudaEventElapsedTime(&ms, e0, e1));
  *ms_per_launch = ms / (double)reps;
  ctx->launches += reps + 3;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(pos_s, ctx->stream);
  cudaFreeAsync(vel_s, ctx->stream);
  cudaFreeAsync(frc_s, ctx->stream);
  cudaFreeAsync(st_s, ctx->stream);
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

int cr_set_lanes(cr_ctx* ctx, int lanes) {
  if (!ctx) return CR_EINVAL;
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8) return ctx->fail(CR_EINVAL, "lanes must be 1, 2, 4 or 8");
  int maxnv = 0;
  for (int n : ctx->ring_nv_h) maxnv = std::max(maxnv, n);
  if (maxnv > tile_vertices(lanes)) return ctx->fail(CR_EINVAL, "a ring does not fit the tile of this lane count");
  ctx->lanes = lanes;
  make_tiles(ctx);
  int rc;
  if ((rc = dalloc(ctx, &ctx->tiles, ctx->tiles_h.size()))) return rc;
  if ((rc = upload(ctx, ctx->tiles, ctx->tiles_h.data(), ctx->tiles_h.size() * sizeof(int4)))) return rc;
  if ((rc = ensure_partials(ctx))) return rc;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_get_lanes(const cr_ctx* ctx, int* lanes) {
  if (!ctx || !lanes) return CR_EINVAL;
  *lanes = ctx->lanes;
  return CR_OK;
}

int cr_autotune(cr_ctx* ctx, long reps, int* lanes_out) {
  if (!ctx || reps <= 0) return CR_EINVAL;
  int maxnv = 0;
  for (int n : ctx->ring_nv_h) maxnv = std::max(maxnv, n);
  int best = ctx->lanes;
  double best_ms = 1e300;
  const int cand[] = {1, 2, 4, 8};
  for (int lanes : cand) {
    if (maxnv > tile_vertices(lanes)) continue;
    int rc = cr_set_lanes(ctx, lanes);
    if (rc) return rc;
    double ms = 0.0;
    if ((rc = cr_profile_step_kernel(ctx, reps, &ms))) return rc;
    if (ms < best_ms) {
      best_ms = ms;
      best = lanes;
    }
  }
  int rc = cr_set_lanes(ctx, best);
  if (rc) return rc;
  if (lanes_out) *lanes_out = best;
  return CR_OK;
}

int cr_set_precision(cr_ctx* ctx, int precision) {
  if (!ctx) return CR_EINVAL;
  if (precision != CR_PRECISION_FP64 && precision != CR_PRECISION_MIXED)
    return ctx->fail(CR_EINVAL, "precision must be CR_PRECISION_FP64 or CR_PRECISION_MIXED");
  ctx->precision = precision;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_get_precision(const cr_ctx* ctx, int* precision) {
  if (!ctx || !precision) return CR_EINVAL;
  *precision = ctx->precision;
  return CR_OK;
}

int cr_set_multistep(cr_ctx* ctx, int on) {
  if (!ctx) return CR_EINVAL;
  ctx->multistep = on != 0;
  return CR_OK;
}

int cr_set_spin_limit(cr_ctx* ctx, long long polls) {
  if (!ctx) return CR_EINVAL;
  int rc = read_status(ctx);
  if (rc) return rc;
  ctx->status_h->spin_limit = polls;
  return upload(ctx, ctx->status, ctx->status_h, sizeof(DevStatus));
}

int cr_get_degraded(const cr_ctx* ctx, int* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = ctx->degraded ? 1 : 0;
  return CR_OK;
}

int cr_set_use_graphs(cr_ctx* ctx, int on) {
  if (!ctx) return CR_EINVAL;
  ctx->use_graphs = on != 0;
  drop_graphs(ctx);
  return CR_OK;
}

// ---------------------------------------------------------------- derivatives

static int diff_ready(cr_ctx* ctx) {
  if (ctx->shape == CR_SHAPE_RIGID) return ctx->fail(CR_ENOTSUP, "derivatives are for deformable rings");
  int rc;
  if (!ctx->nbr_built && (rc = build_list(ctx, ctx->cur, ctx->cut_distance))) return rc;
  if (!ctx->diff_f) {
    if ((rc = dalloc(ctx, &ctx->diff_f, (size_t)8 * ctx->nv)) || (rc = dalloc(ctx, &ctx->diff_e, (size_t)4 * ctx->nv)) ||
        (rc = dalloc(ctx, &ctx->diff_dot, 256)) || (rc = dalloc(ctx, &ctx->diff_vec, (size_t)10 * ctx->nv)) ||
        (rc = dalloc(ctx, &ctx->diff_area, (size_t)4 * ctx->np)) || (rc = dalloc(ctx, &ctx->cg_state, 1)) ||
        (rc = dalloc(ctx, &ctx->cg_part, (size_t)8 * 148)) || (rc = dalloc(ctx, &ctx->cg_minv, (size_t)3 * ctx->nv)))
      return rc;
  }
  return CR_OK;
}

static DiffArgs diff_args(cr_ctx* ctx) {
  DiffArgs g;
  memset(&g, 0, sizeof(g));
  g.p = ctx->p;
  g.pos = ctx->pos[ctx->cur];
  g.rad = ctx->rad;
  g.l0 = ctx->l0;
  g.theta0 = ctx->theta0;
  g.a0 = ctx->a0;
  g.vtopo = ctx->vtopo;
  g.nbr = ctx->nbr;
  g.nbr_cnt = ctx->nbr_cnt;
  g.nbr_cap = ctx->cap;
  g.force_out = ctx->diff_f;
  g.energy_out = ctx->diff_e;
  g.ring_area = ctx->diff_area;
  return g;
}

static int diff_launch(cr_ctx* ctx, const DiffArgs& g) {
  launch_diff(ctx->stream, ctx->potential, inter_kind(ctx), g, ctx->ring_first, ctx->ring_nv);
  ctx->launches += 2;
  CR_TRY(cudaGetLastError());
  return CR_OK;
}

// host sums of the hyper-dual energy parts, in vertex order
static int diff_energy(cr_ctx* ctx, double out[4]) {
  std::vector<double> e((size_t)4 * ctx->nv);
  int rc = download(ctx, e.data(), ctx->diff_e, e.size() * sizeof(double));
  if (rc) return rc;
  // compensated (TwoSum) sums in vertex order: the energy and pressure
  // tangents are differences of large terms of both signs
  double c[4] = {0.0, 0.0, 0.0, 0.0};
  for (int q = 0; q < 4; q++) out[q] = 0.0;
  for (int v = 0; v < ctx->nv; v++)
    for (int q = 0; q < 4; q++) {
      const double x = e[(size_t)4 * v + q], t = out[q] + x, bp = t - out[q];
      c[q] += (out[q] - (t - bp)) + (x - bp);
      out[q] = t;
    }
  for (int q = 0; q < 4; q++) out[q] += c[q];
  return CR_OK;
}

static int dev_dot(cr_ctx* ctx, const double* a, const double* b, int n, double* out) {
  const int nb = std::min(256, std::max(1, (n + 255) / 256));
  launch_dot_partials(ctx->stream, n, a, b, ctx->diff_dot, nb);
  ctx->launches++;
  double part[256];
  int rc = download(ctx, part, ctx->diff_dot, nb * sizeof(double));
  if (rc) return rc;
  double s = 0.0;
  for (int i = 0; i < nb; i++) s += part[i];
  *out = s;
  return CR_OK;
}

static int dev_project(cr_ctx* ctx, double* x) {
  std::vector<double> h((size_t)2 * ctx->nv);
  int rc = download(ctx, h.data(), x, h.size() * sizeof(double));
  if (rc) return rc;
  double mx = 0.0, my = 0.0;
  for (int v = 0; v < ctx->nv; v++) {
    mx += h[2 * v];
    my += h[2 * v + 1];
  }
  launch_sub_mean(ctx->stream, ctx->nv, x, mx / ctx->nv, my / ctx->nv);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  return CR_OK;
}

extern "C" int cr_hvp_device(cr_ctx* ctx, const double* v_dev, double* hv_dev) {
  if (!ctx || !v_dev || !hv_dev) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  DiffArgs g = diff_args(ctx);
  g.t1 = reinterpret_cast<const double2*>(v_dev);
  if ((rc = diff_launch(ctx, g))) return rc;
  launch_extract_hv(ctx->stream, ctx->nv, ctx->diff_f, hv_dev);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

extern "C" int cr_hvp(cr_ctx* ctx, const double* v, double* hv) {
  if (!ctx || !v || !hv) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  double* vd = ctx->diff_vec;
  double* hd_ = ctx->diff_vec + (size_t)2 * ctx->nv;
  if ((rc = upload(ctx, vd, v, (size_t)2 * ctx->nv * sizeof(double)))) return rc;
  if ((rc = cr_hvp_device(ctx, vd, hd_))) return rc;
  return download(ctx, hv, hd_, (size_t)2 * ctx->nv * sizeof(double));
}

extern "C" int cr_calc_pressure(cr_ctx* ctx, double* P) {
  if (!ctx || !P) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  DiffArgs g = diff_args(ctx);
  g.t1 = ctx->pos[ctx->cur];  // affine dilation: x -> (1 + e) x, L -> (1 + e) L
  g.s1 = 1.0;
  if ((rc = diff_launch(ctx, g))) return rc;
  double e[4];
  if ((rc = diff_energy(ctx, e))) return rc;
  *P = -e[1] / (2.0 * ctx->p.lx * ctx->p.ly);
  return CR_OK;
}

extern "C" int cr_param_derivatives(cr_ctx* ctx, int param, double* dU, double* dP, double* dF, double* dPdx) {
  if (!ctx || param < 0 || param > 3) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  DiffArgs g = diff_args(ctx);
  g.t1 = ctx->pos[ctx->cur];
  g.s1 = 1.0;
  if (param < 3) g.pe2[param] = 1.0;
  else g.c2 = 1.0;
  if ((rc = diff_launch(ctx, g))) return rc;
  double e[4];
  if ((rc = diff_energy(ctx, e))) return rc;
  const double A2 = 2.0 * ctx->p.lx * ctx->p.ly;
  if (dU) *dU = e[2];
  if (dP) *dP = -e[3] / A2;
  if (dF || dPdx) {
    std::vector<double> f((size_t)8 * ctx->nv);
    if ((rc = download(ctx, f.data(), ctx->diff_f, f.size() * sizeof(double)))) return rc;
    for (int v = 0; v < ctx->nv; v++) {
      const double* q = &f[(size_t)8 * v];
      if (dF) {
        dF[2 * v] = q[2];
        dF[2 * v + 1] = q[6];
      }
      if (dPdx) {
        dPdx[2 * v] = (q[0] + q[1]) / A2;
        dPdx[2 * v + 1] = (q[4] + q[5]) / A2;
      }
    }
  }
  return CR_OK;
}

extern "C" int cr_hessian_solve(cr_ctx* ctx, const double* b, double* x, double tol, long maxIter, long* iters,
                                double* relres) {
  if (!ctx || !b || !x || maxIter < 0) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  const int n = 2 * ctx->nv;
  double* xd = ctx->diff_vec;
  double* r = xd + n;
  double* pv = r + n;
  double* hp = pv + n;
  double* zv = hp + n;
  // preconditioned conjugate gradients on the Hessian restricted to vectors
  // without a uniform translation (its null space in a periodic box): b is
  // projected, each H p and each preconditioned residual lose their means,
  // so every iterate stays in that subspace.  The preconditioner is
  // block-Jacobi: the inverse 2 x 2 diagonal block of every vertex, from one
  // hyper-dual launch seeding each vertex's own coordinates.
  const double* minv = nullptr;
  if (ctx->cg_precond) {
    DiffArgs gd = diff_args(ctx);
    gd.diag = 1;
    launch_diff(ctx->stream, ctx->potential, inter_kind(ctx), gd, ctx->ring_first, ctx->ring_nv);
    launch_cg_prec(ctx->stream, ctx->nv, ctx->diff_f, ctx->cg_minv);
    ctx->launches += 3;
    CR_TRY(cudaGetLastError());
    minv = ctx->cg_minv;
  }
  if ((rc = upload(ctx, r, b, (size_t)n * sizeof(double)))) return rc;
  if ((rc = dev_project(ctx, r))) return rc;
  CR_TRY(cudaMemsetAsync(xd, 0, (size_t)n * sizeof(double), ctx->stream));
  launch_cg_apply(ctx->stream, ctx->nv, minv, r, zv);
  CR_TRY(cudaGetLastError());
  if ((rc = dev_project(ctx, zv))) return rc;
  CR_TRY(cudaMemcpyAsync(pv, zv, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  double bb, rz;
  if ((rc = dev_dot(ctx, r, r, n, &bb)) || (rc = dev_dot(ctx, r, zv, n, &rz))) return rc;
  CgState cs;
  memset(&cs, 0, sizeof(cs));
  cs.rr = bb;
  cs.bb = bb;
  cs.rz = rz;
  cs.tol = tol;
  cs.max_iters = maxIter;
  cs.done = (maxIter == 0 || !(bb > 0.0) || !(std::sqrt(cs.rr / bb) > tol)) ? 1 : 0;
  if ((rc = upload(ctx, ctx->cg_state, &cs, sizeof(cs)))) return rc;
  // the iterations run in captured chunks: H p (hyper-dual forces along p),
  // then the CG scalars and vector updates, all on the device; every kernel
  // returns at once after the state says done, so a chunk may overrun
  constexpr int kChunk = 32;
  DiffArgs g = diff_args(ctx);
  g.t1 = reinterpret_cast<const double2*>(pv);
  g.skip = &ctx->cg_state->done;
  CgArgs a;
  a.nv = ctx->nv;
  a.x = xd;
  a.r = r;
  a.p = pv;
  a.hp = hp;
  a.fhd = ctx->diff_f;
  a.st = ctx->cg_state;
  a.partials = ctx->cg_part;
  a.nblk = cg_blocks(ctx->nv);
  a.z = zv;
  a.minv = minv;
  cudaGraphExec_t exec = nullptr;
  if (!cs.done) {
    cudaGraph_t graph = nullptr;
    CR_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < kChunk; k++) {
      launch_diff(ctx->stream, ctx->potential, inter_kind(ctx), g, ctx->ring_first, ctx->ring_nv);
      launch_cg_iteration(ctx->stream, a);
    }
    cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    CR_TRY(ce);
  }
  while (!cs.done) {
    cudaError_t ce = cudaGraphLaunch(exec, ctx->stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&cs, ctx->cg_state, sizeof(cs), cudaMemcpyDeviceToHost, ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    if (ce != cudaSuccess) {
      cudaGraphExecDestroy(exec);
      CR_TRY(ce);
    }
    ctx->launches += (long long)kChunk * 7;
  }
  if (exec) cudaGraphExecDestroy(exec);
  CR_TRY(cudaGetLastError());
  if (cs.bad) return ctx->fail(CR_ENONFINITE, "Hessian not positive along a CG direction");
  if (iters) *iters = (long)cs.iters;
  if (relres) *relres = bb > 0.0 ? std::sqrt(cs.rr / bb) : 0.0;
  return download(ctx, x, xd, (size_t)n * sizeof(double));
}

int cr_hessian_diag_blocks(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc;
  if ((rc = diff_ready(ctx))) return rc;
  DiffArgs gd = diff_args(ctx);
  gd.diag = 1;
  launch_diff(ctx->stream, ctx->potential, inter_kind(ctx), gd, ctx->ring_first, ctx->ring_nv);
  ctx->launches += 2;
  CR_TRY(cudaGetLastError());
  std::vector<double> f((size_t)8 * ctx->nv);
  if ((rc = download(ctx, f.data(), ctx->diff_f, f.size() * sizeof(double)))) return rc;
  for (int v = 0; v < ctx->nv; v++) {
    const double* q = f.data() + (size_t)8 * v;
    out[3 * v] = -q[1];
    out[3 * v + 1] = -0.5 * (q[2] + q[5]);
    out[3 * v + 2] = -q[6];
  }
  return CR_OK;
}

int cr_set_cg_preconditioner(cr_ctx* ctx, int kind) {
  if (!ctx || kind < 0 || kind > 1) return CR_EINVAL;
  ctx->cg_precond = kind;
  return CR_OK;
}

int cr_get_launch_count(const cr_ctx* ctx, long long* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = ctx->launches;
  return CR_OK;
}

}  // extern "C"

// ------------------------------------------------------- soft-disk pre-packing
// The particle-level stage of compressFIRE.cpp:53-90 (kernels in cr_soft.cu).

static int soft_ensure(cr_ctx* ctx) {
  if (ctx->soft_ready) return CR_OK;
  int rc;
  if ((rc = dalloc(ctx, &ctx->prad, ctx->np)) || (rc = dalloc(ctx, &ctx->plast, ctx->np)) ||
      (rc = dalloc(ctx, &ctx->pid, ctx->np)) || (rc = dalloc(ctx, &ctx->pnbr_cnt, ctx->np)) ||
      (rc = dalloc(ctx, &ctx->pnbr, (size_t)16 * ctx->np)) || (rc = dalloc(ctx, &ctx->pstatus, 1)) ||
      (rc = dalloc(ctx, &ctx->pfire, 1)))
    return rc;
  ctx->pcap = 16;
  std::vector<int> id(ctx->np);
  for (int i = 0; i < ctx->np; i++) id[i] = i;
  if ((rc = upload(ctx, ctx->pid, id.data(), id.size() * sizeof(int)))) return rc;
  ctx->soft_ready = true;
  return CR_OK;
}

static int soft_read_status(cr_ctx* ctx, DevStatus* out) { return download(ctx, out, ctx->pstatus, sizeof(DevStatus)); }
static int soft_clear_status(cr_ctx* ctx) {
  DevStatus s;
  int rc = soft_read_status(ctx, &s);
  if (rc) return rc;
  s.abort = 0;
  s.overflow = 0;
  s.rebuild = 0;
  s.done_ctr = 0;
  s.bar_count = 0;
  s.stalled = 0;
  return upload(ctx, ctx->pstatus, &s, sizeof(DevStatus));
}

static SysParams soft_params(cr_ctx* ctx) {
  SysParams sp = ctx->p;
  sp.nv = ctx->np;  // list stride and loop bound of the build: one entry per particle
  return sp;
}

static double soft_rmax(cr_ctx* ctx, int* rc) {
  std::vector<double> r(ctx->np);
  *rc = download(ctx, r.data(), ctx->prad, CR_NP1);
  double m = 0.0;
  for (double x : r) m = std::max(m, x);
  return m;
}

static NbrArgs soft_nbr_args(cr_ctx* ctx, double cut) {
  NbrArgs n;
  n.pos = ctx->ppos;
  n.rad = ctx->prad;
  n.ring_of = ctx->pid;
  n.nbr = ctx->pnbr;
  n.nbr_cnt = ctx->pnbr_cnt;
  n.cap = ctx->pcap;
  n.cut_distance = cut;
  n.last_pos = ctx->plast;
  n.cell_of = ctx->cell_of;
  n.slot = ctx->slot;
  n.cell_cnt = ctx->cell_cnt;
  n.cell_start = ctx->cell_start;
  n.cell_vid = ctx->cell_vid;
  n.cell_pos = ctx->cell_pos;
  n.cell_rad = ctx->cell_rad;
  n.cell_ring = ctx->cell_ring;
  n.status = ctx->pstatus;
  n.count_op = 0;
  n.count_update = 0;
  n.block_sum = ctx->block_sum;
  n.bucket = ctx->cell_bucket;
  n.bucket_pos = ctx->bucket_pos;
  n.bucket_rad = ctx->bucket_rad;
  n.bucket_ring = ctx->bucket_ring;
  n.bucket_pq = ctx->bucket_pq;
  n.cell_stride = ctx->ncells_alloc;
  n.self_rsum = 1;
  return n;
}

// cells no smaller than (1 + cut) * 2 * max particle radius, as for vertices
static int soft_setup_grid(cr_ctx* ctx, double cut) {
  int rc = CR_OK;
  const double rmax = soft_rmax(ctx, &rc);
  if (rc) return rc;
  const double cmin = (1.0 + cut) * 2.0 * rmax * (1.0 + 1e-9);
  int ncx = cmin > 0 ? (int)std::min(4096.0, std::floor(ctx->p.lx / cmin)) : 0;
  int ncy = cmin > 0 ? (int)std::min(4096.0, std::floor(ctx->p.ly / cmin)) : 0;
  if (ncx < 3 || ncy < 3) {
    ctx->pgrid = CellGrid{0, 0, 0.0, 0.0};
    return CR_OK;
  }
  ctx->pgrid = CellGrid{ncx, ncy, ctx->p.lx / ncx, ctx->p.ly / ncy};
  return alloc_cells(ctx, ncx * ncy);
}

// DPM2D::calcParticleNeighborList (DPM2D.cu:3521-3545): the list size only
// grows, to the next power of two of the largest count.
static int soft_build(cr_ctx* ctx, double cut) {
  int rc;
  if ((rc = soft_setup_grid(ctx, cut))) return rc;
  for (int pass = 0; pass < 3; pass++) {
    if ((rc = soft_clear_status(ctx))) return rc;
    launch_nbr_fused(ctx->stream, soft_params(ctx), ctx->pgrid, soft_nbr_args(ctx, cut),
                     nbr_fused_blocks(ctx->np, ctx->fused_max), 1);
    ctx->launches += 1;
    CR_TRY(cudaGetLastError());
    DevStatus st;
    if ((rc = soft_read_status(ctx, &st))) return rc;
    if (st.stalled) {
      reset_cell_counts(ctx);
      return ctx->fail(CR_ECUDA, "particle list build: a grid barrier timed out");
    }
    if (!st.overflow) {
      if (st.max_count > 0) ctx->plist_size_ref = std::max<long long>(ctx->plist_size_ref, pow2ceil(st.max_count));
      ctx->pnbr_built = true;
      return soft_clear_status(ctx);
    }
    const int newcap = (int)std::max<long long>(16, pow2ceil(2LL * st.max_count));
    if ((rc = dalloc(ctx, &ctx->pnbr, (size_t)newcap * ctx->np))) return rc;
    ctx->pcap = newcap;
    drop_graphs(ctx);
  }
  return ctx->fail(CR_ENBR_OVERFLOW, "particle neighbour list kept overflowing");
}

static SoftArgs soft_args(cr_ctx* ctx, double cutoff) {
  SoftArgs a;
  a.pos = ctx->ppos;
  a.vel = ctx->p_vel;
  a.force = ctx->p_force;
  a.energy = ctx->p_energy;
  a.rad = ctx->prad;
  a.nbr = ctx->pnbr;
  a.cnt = ctx->pnbr_built ? ctx->pnbr_cnt : ctx->zero_cnt;
  a.cap = ctx->pcap;
  a.last_pos = ctx->plast;
  a.cutoff = cutoff;
  a.fire = ctx->pfire;
  a.status = ctx->pstatus;
  a.partials = ctx->partials;
  return a;
}

extern "C" {

int cr_set_particle_radii(cr_ctx* ctx, const double* rad) {
  if (!ctx || !rad) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  ctx->pnbr_built = false;
  return upload(ctx, ctx->prad, rad, CR_NP1);
}
int cr_get_particle_radii(const cr_ctx* cctx, double* rad) {
  cr_ctx* ctx = const_cast<cr_ctx*>(cctx);
  if (!ctx || !rad) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  return download(ctx, rad, ctx->prad, CR_NP1);
}
int cr_get_mean_particle_sigma(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  std::vector<double> r(ctx->np);
  if ((rc = download(ctx, r.data(), ctx->prad, CR_NP1))) return rc;
  double s = 0.0;
  for (double x : r) s += x;
  *out = s / ctx->np;
  return CR_OK;
}
int cr_get_min_particle_sigma(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  std::vector<double> r(ctx->np);
  if ((rc = download(ctx, r.data(), ctx->prad, CR_NP1))) return rc;
  double m = 1.0;  // thrust::reduce with init 1 (DPM2D.cu:766-768)
  for (double x : r) m = std::min(m, x);
  *out = m;
  return CR_OK;
}

int cr_set_random_particles(cr_ctx* ctx, double phi0, double extraRad, long seed) {
  if (!ctx || !(phi0 > 0)) return ctx ? ctx->fail(CR_EINVAL, "bad packing fraction") : CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  double phi;
  if ((rc = cr_get_preferred_phi(ctx, &phi))) return rc;
  const double scale = std::sqrt(phi / phi0);
  const double box[2] = {1.0, 1.0};
  if ((rc = cr_set_box_size(ctx, box))) return rc;
  std::vector<double> a0(ctx->np), l0(ctx->nv), rad(ctx->nv), pr(ctx->np), pp(2 * (size_t)ctx->np);
  if ((rc = download(ctx, a0.data(), ctx->a0, CR_NP1)) || (rc = download(ctx, l0.data(), ctx->l0, CR_NV1)) ||
      (rc = download(ctx, rad.data(), ctx->rad, CR_NV1)))
    return rc;
  // the drand48() stream of srand48(seed)
  unsigned short xs[3] = {0x330E, (unsigned short)(seed & 0xFFFF), (unsigned short)((seed >> 16) & 0xFFFF)};
  for (int q = 0; q < ctx->np; q++) {
    a0[q] /= (scale * scale);
    for (int dim = 0; dim < 2; dim++) pp[2 * (size_t)q + dim] = box[dim] * erand48(xs);
    const long n = ctx->ring_nv_h[q];
    pr[q] = extraRad * std::sqrt((2. * a0[q]) / (n * std::sin(2. * kPi / n)));
  }
  for (int v = 0; v < ctx->nv; v++) {
    l0[v] /= scale;
    rad[v] /= scale;
  }
  if ((rc = upload(ctx, ctx->a0, a0.data(), CR_NP1)) || (rc = upload(ctx, ctx->area, a0.data(), CR_NP1)) ||
      (rc = upload(ctx, ctx->l0, l0.data(), CR_NV1)) || (rc = upload(ctx, ctx->rad, rad.data(), CR_NV1)) ||
      (rc = upload(ctx, ctx->prad, pr.data(), CR_NP1)) || (rc = upload(ctx, ctx->ppos, pp.data(), 2 * CR_NP1)))
    return rc;
  update_rmax(ctx, rad.data());
  ctx->nbr_built = false;
  ctx->pnbr_built = false;
  drop_graphs(ctx);
  return CR_OK;
}

int cr_calc_particle_neighbor_list(cr_ctx* ctx, double cutDistance) {
  if (!ctx || !(cutDistance > -1.0)) return ctx ? ctx->fail(CR_EINVAL, "bad cutDistance") : CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  return soft_build(ctx, cutDistance);
}
int cr_get_particle_neighbor_list_size(const cr_ctx* ctx, long* out) {
  if (!ctx || !out) return CR_EINVAL;
  *out = (long)ctx->plist_size_ref;
  return CR_OK;
}
int cr_get_particle_max_neighbor_list(const cr_ctx* cctx, long* out) {
  cr_ctx* ctx = const_cast<cr_ctx*>(cctx);
  if (!ctx || !out) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  std::vector<int> cnt(ctx->np);
  if ((rc = download(ctx, cnt.data(), ctx->pnbr_built ? ctx->pnbr_cnt : ctx->zero_cnt, ctx->np * sizeof(int))))
    return rc;
  for (int i = 0; i < ctx->np; i++) out[i] = cnt[i];
  return CR_OK;
}
int cr_get_particle_neighbors(const cr_ctx* cctx, long* out) {
  cr_ctx* ctx = const_cast<cr_ctx*>(cctx);
  if (!ctx || !out) return CR_EINVAL;
  const long ls = ctx->plist_size_ref;
  if (ls == 0 || !ctx->pnbr_built) return CR_OK;
  std::vector<int> cnt(ctx->np), nb((size_t)ctx->pcap * ctx->np);
  int rc;
  if ((rc = download(ctx, cnt.data(), ctx->pnbr_cnt, ctx->np * sizeof(int)))) return rc;
  if ((rc = download(ctx, nb.data(), ctx->pnbr, nb.size() * sizeof(int)))) return rc;
  std::vector<int> row;
  for (int i = 0; i < ctx->np; i++) {
    row.clear();
    for (int k = 0; k < std::min(cnt[i], ctx->pcap); k++) row.push_back(nb[(size_t)k * ctx->np + i]);
    std::sort(row.begin(), row.end());
    for (long k = 0; k < ls; k++) out[(size_t)i * ls + k] = k < (long)row.size() ? row[k] : -1;
  }
  return CR_OK;
}

int cr_calc_particle_force_energy(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  launch_soft_force(ctx->stream, ctx->potential, ctx->p, soft_args(ctx, 0.0), false);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}
int cr_get_particle_potential_energy(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<double> e(ctx->np);
  int rc = download(ctx, e.data(), ctx->p_energy, CR_NP1);
  if (rc) return rc;
  double s = 0.0;
  for (double x : e) s += x;
  *out = s;
  return CR_OK;
}
int cr_get_particle_max_unbalanced_force(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  std::vector<double> f(2 * (size_t)ctx->np);
  int rc = download(ctx, f.data(), ctx->p_force, 2 * CR_NP1);
  if (rc) return rc;
  double m = -1.0;
  for (double x : f) m = std::max(m, x * x);
  *out = std::sqrt(m);
  return CR_OK;
}
int cr_reset_particle_last_positions(cr_ctx* ctx) {
  if (!ctx) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  CR_TRY(cudaMemcpyAsync(ctx->plast, ctx->ppos, 2 * CR_NP1, cudaMemcpyDeviceToDevice, ctx->stream));
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}
int cr_get_particle_max_displacement(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  std::vector<double> x(2 * (size_t)ctx->np), y(2 * (size_t)ctx->np);
  if ((rc = download(ctx, x.data(), ctx->ppos, 2 * CR_NP1)) || (rc = download(ctx, y.data(), ctx->plast, 2 * CR_NP1)))
    return rc;
  double m = -1.0;
  for (int q = 0; q < ctx->np; q++) {
    double d2 = 0.0;
    for (int dim = 0; dim < 2; dim++) {
      const double L = dim ? ctx->p.ly : ctx->p.lx;
      double d = x[2 * (size_t)q + dim] - y[2 * (size_t)q + dim];
      d -= L * std::round(d / L);  // pbcDistance (include/cudaKernel.cuh:70-74)
      d2 += d * d;
    }
    m = std::max(m, std::sqrt(d2));
  }
  *out = m;
  return CR_OK;
}

int cr_init_particle_fire(cr_ctx* ctx, const double* p7, long minStep, long numStep) {
  if (!ctx || !p7) return CR_EINVAL;
  int rc = soft_ensure(ctx);
  if (rc) return rc;
  SoftFire f;
  memset(&f, 0, sizeof(f));
  f.a_start = p7[0];
  f.f_dec = p7[1];
  f.f_inc = p7[2];
  f.f_a = p7[3];
  f.dt = p7[4];
  f.dt_max = p7[5];
  f.a = p7[6];
  f.min_step = minStep;
  f.num_step = numStep;
  f.tol = -1.0;  // no convergence stop unless a minimisation sets one
  if ((rc = upload(ctx, ctx->pfire, &f, sizeof(f)))) return rc;
  ctx->pfire_ready = true;
  return cr_reset_particle_last_positions(ctx);  // DPM2D::initFIRE (DPM2D.cu:3672)
}
int cr_get_particle_fire_state(cr_ctx* ctx, double* out) {
  if (!ctx || !out) return CR_EINVAL;
  if (!ctx->pfire_ready) return ctx->fail(CR_EINVAL, "particle FIRE not initialised");
  SoftFire f;
  int rc = download(ctx, &f, ctx->pfire, sizeof(f));
  if (rc) return rc;
  out[0] = f.dt;
  out[1] = f.a;
  out[2] = (double)f.num_step;
  return CR_OK;
}

// FIRE::minimizerParticleLoop (FIRE.cu:156-171) nsteps times
int cr_particle_fire_loop(cr_ctx* ctx, long nsteps) {
  if (!ctx || nsteps < 0) return CR_EINVAL;
  if (!ctx->pfire_ready) return ctx->fail(CR_EINVAL, "particle FIRE not initialised");
  int rc;
  if ((rc = ensure_partials(ctx))) return rc;
  if (soft_blocks(ctx->np) * 4 > ctx->partials_n) return ctx->fail(CR_EINVAL, "too many particles for the partials");
  if ((rc = soft_clear_status(ctx))) return rc;
  SoftFire f;
  if ((rc = download(ctx, &f, ctx->pfire, sizeof(f)))) return rc;
  f.converged = 0;
  f.tol = -1.0;
  if ((rc = upload(ctx, ctx->pfire, &f, sizeof(f)))) return rc;
  const SoftArgs a = soft_args(ctx, 0.0);
  const SysParams sp = soft_params(ctx);
  for (long s = 0; s < nsteps; s++) {
    launch_soft_move(ctx->stream, sp, a, 0);
    launch_soft_force(ctx->stream, ctx->potential, sp, a, true);
    ctx->launches += 2;
  }
  launch_soft_bend(ctx->stream, ctx->np, a);
  ctx->launches += 1;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  return CR_OK;
}

// compressFIRE.cpp:66-78: FIRE until max |F_d| <= tol or maxIterations,
// the particle list rebuilt after an iteration that moved a particle by more
// than (1 + cutDistance) * getMinParticleSigma / 3 since the last build.  The
// caller has built the list and computed the forces, as the driver does.
int cr_particle_fire_minimize(cr_ctx* ctx, double cutDistance, double tol, long maxIterations, long* iterations) {
  if (!ctx || maxIterations < 0) return CR_EINVAL;
  if (!ctx->pfire_ready) return ctx->fail(CR_EINVAL, "particle FIRE not initialised");
  int rc;
  if ((rc = ensure_partials(ctx))) return rc;
  if (soft_blocks(ctx->np) * 4 > ctx->partials_n) return ctx->fail(CR_EINVAL, "too many particles for the partials");
  if (!ctx->pnbr_built && (rc = soft_build(ctx, cutDistance))) return rc;
  if ((rc = soft_setup_grid(ctx, cutDistance))) return rc;
  double minsig, fmax;
  if ((rc = cr_get_min_particle_sigma(ctx, &minsig))) return rc;
  if ((rc = cr_get_particle_max_unbalanced_force(ctx, &fmax))) return rc;
  const double cutoff = (1 + cutDistance) * minsig;
  SoftFire f;
  if ((rc = download(ctx, &f, ctx->pfire, sizeof(f)))) return rc;
  const long long it0 = f.iters;
  f.tol = tol;
  f.converged = !(fmax > tol) ? 1 : 0;
  if ((rc = upload(ctx, ctx->pfire, &f, sizeof(f)))) return rc;
  if ((rc = soft_clear_status(ctx))) return rc;
  const double key[3] = {cutDistance, cutoff, (double)ctx->pgrid.ncx * 8192.0 + ctx->pgrid.ncy};
  if (key[0] != ctx->soft_key[0] || key[1] != ctx->soft_key[1] || key[2] != ctx->soft_key[2]) {
    drop_graphs(ctx);
    std::copy(key, key + 3, ctx->soft_key);
  }
  long done = 0;
  const long chunk = 64;
  while (!f.converged && done < maxIterations) {
    const long n = std::min(chunk, maxIterations - done);
    auto it = ctx->soft_graphs.find(n);
    if (it == ctx->soft_graphs.end()) {
      GraphEntry ge;
      const SoftArgs a = soft_args(ctx, cutoff);
      const SysParams sp = soft_params(ctx);
      const NbrArgs na = soft_nbr_args(ctx, cutDistance);
      const int fb = nbr_fused_blocks(ctx->np, ctx->fused_max);
      CR_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      for (long s = 0; s < n; s++) {
        launch_soft_move(ctx->stream, sp, a, 1);
        launch_soft_force(ctx->stream, ctx->potential, sp, a, true);
        launch_nbr_fused(ctx->stream, sp, ctx->pgrid, na, fb, 0);
      }
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ctx->fail(CR_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      }
      CR_TRY(cudaGraphInstantiate(&ge.exec, g, 0));
      ge.graph = g;
      ge.launches = 3 * n;
      it = ctx->soft_graphs.emplace(n, ge).first;
    }
    CR_TRY(cudaGraphLaunch(it->second.exec, ctx->stream));
    ctx->launches += it->second.launches;
    DevStatus st;
    if ((rc = soft_read_status(ctx, &st))) return rc;
    if ((rc = download(ctx, &f, ctx->pfire, sizeof(f)))) return rc;
    done = (long)(f.iters - it0);
    if (st.abort) {
      if (st.stalled) return ctx->fail(CR_ECUDA, "particle list build: a grid barrier timed out");
      if (!st.overflow) return ctx->fail(CR_ECUDA, "particle FIRE aborted");
      // the list outgrew its capacity after iteration `done`: grow, rebuild
      // from the same positions and carry on
      if ((rc = soft_clear_status(ctx))) return rc;
      if ((rc = soft_build(ctx, cutDistance))) return rc;  // regrows and drops the graphs
    }
  }
  launch_soft_bend(ctx->stream, ctx->np, soft_args(ctx, cutoff));
  ctx->launches += 1;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  if ((rc = download(ctx, &f, ctx->pfire, sizeof(f)))) return rc;
  if (iterations) *iterations = (long)(f.iters - it0);
  return CR_OK;
}

// DPM2D::initVerticesOnParticles (DPM2D.cu:1678-1691).  draws: the 2 nv
// uniforms on [0, 1) of the jitter (x then y of each vertex, the order of the
// reference's drand48 calls), or NULL for the context's Philox stream.
int cr_init_vertices_on_particles(cr_ctx* ctx, const double* draws) {
  if (!ctx) return CR_EINVAL;
  int rc;
  if (draws) {
    if (!ctx->pdraws && (rc = dalloc(ctx, &ctx->pdraws, 2 * (size_t)ctx->nv))) return rc;
    if ((rc = upload(ctx, ctx->pdraws, draws, 2 * CR_NV1))) return rc;
  }
  launch_soft_vertices(ctx->stream, ctx->nv, ctx->ring_of, ctx->ring_nv, ctx->a0, ctx->l0, ctx->ppos,
                       draws ? ctx->pdraws : nullptr, ctx->seed, (1ull << 61) + ctx->rng_calls++, ctx->pos[ctx->cur],
                       ctx->vel, ctx->force, ctx->energy);
  ctx->launches++;
  CR_TRY(cudaGetLastError());
  CR_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->nbr_built = false;  // DPM2D::initNeighbors + syncNeighborsToDevice (DPM2D.cu:1689-1690)
  return CR_OK;
}

}  // extern "C"
