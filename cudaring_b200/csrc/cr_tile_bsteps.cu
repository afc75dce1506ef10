// Persistent batched FIRE: up to nmax FIRE iterations of every system of a
// batch in one launch, a grid barrier after each half of an iteration in
// place of a kernel boundary.  Each CTA owns one tile (the host launches the
// kernel only when occupancy x SMs holds the grid):
//   pre-kick of the tile's vertices (bfire_prekick: the system's FIRE
//   scalars from its sums, velocity mixing, first half kick, position
//   update, displacement check)
//   -- grid barrier --
//   a system's displacement check fired: leave with the force op pending;
//   the batched list build runs and the next launch starts with that op
//   force op of the tile (the tiled kernel's FIRE op: forces, second half
//   kick, per-system sums reduced by the system's last tile, convergence)
//   -- grid barrier --
// The arithmetic is that of one launch per op (k_bfire_pre, then the tiled
// kernel), so both give the same iterates.  FP64, tile shapes (1, 128) and
// (2, 192); other configurations keep one launch per op.  Every barrier wait
// is bounded (status.spin_limit): a CTA that gives up sets stalled and
// abort, and the host reruns the chunk one launch per op.
#include "cr_bfire.cuh"
#include "cr_launch.h"
#include "cr_tile_kernel.cuh"

namespace cr {

template <int POT, int INTER, int BLOCK, int L>
__global__ void __launch_bounds__(BLOCK, tile_threads_per_sm<PREC_FP64, L>() / BLOCK)
    k_bfire_steps(const __grid_constant__ SysParams p, const __grid_constant__ SysArrays a,
                  const __grid_constant__ StepArgs s, const __grid_constant__ BFire f, int nmax) {
  DevStatus* st = s.status;
  const volatile DevStatus* vs = st;
  __shared__ int s_stop;
  if (vs->abort) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && f.use_cond) cudaGraphSetConditional(f.cond, 0u);
    return;
  }
  const int pending = vs->bpending;  // the last launch left with its force op due
  const int4 tile = a.tiles[blockIdx.x];
  bool stalled = false;
  int rebuild = 0;
  const int n = nmax > 0 ? nmax : pending;
  for (int j = 0; j < n; j++) {
    if (!(j == 0 && pending)) {
      for (int v = tile.z + threadIdx.x; v < tile.w; v += BLOCK) bfire_prekick(f, v);
      if (!steps_barrier(st)) {
        stalled = true;
        break;
      }
      if (threadIdx.x == 0) s_stop = (vs->rebuild ? 1 : 0) | (vs->abort ? 2 : 0);
      __syncthreads();
      const int stop = s_stop;
      __syncthreads();
      if (stop) {
        rebuild = stop & 1;
        break;
      }
    }
    tile_body<POT, INTER, MODE_STEP, BLOCK, L, PREC_FP64, true, 2>(p, a, s, a.pos, s.pos_out, 0ull, nullptr);
    if (!steps_barrier(st)) {
      stalled = true;
      break;
    }
    if (threadIdx.x == 0) s_stop = vs->abort ? 1 : 0;
    __syncthreads();
    const int stop = s_stop;
    __syncthreads();
    if (stop) break;
  }
  if (stalled) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->bpending = rebuild;
    if (f.use_cond) cudaGraphSetConditional(f.cond, (rebuild && !st->abort) ? 1u : 0u);
  }
}

namespace {

template <int POT, int INTER>
BFireStepsFn fn_shape(int lanes, int block) {
  if (lanes == 1 && block == 128) return k_bfire_steps<POT, INTER, 128, 1>;
  if (lanes == 2 && block == 192) return k_bfire_steps<POT, INTER, 192, 2>;
  return nullptr;
}

template <int INTER>
BFireStepsFn fn_inter(int pot, int lanes, int block) {
  switch (pot) {
    case POT_HARMONIC: return fn_shape<POT_HARMONIC, INTER>(lanes, block);
    case POT_LJ: return fn_shape<POT_LJ, INTER>(lanes, block);
    case POT_ADHESIVE: return fn_shape<POT_ADHESIVE, INTER>(lanes, block);
    default: return fn_shape<POT_WCA, INTER>(lanes, block);
  }
}

}  // namespace

BFireStepsFn bfire_steps_fn(int pot, int inter, int lanes, int block) {
  return inter == INT_VV ? fn_inter<INT_VV>(pot, lanes, block) : fn_inter<INT_SMOOTH>(pot, lanes, block);
}

int bfire_steps_max_blocks(BFireStepsFn fn, int block) {
  int dev = 0, sms = 0, occ = 0;
  if (!fn || cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, 0) != cudaSuccess) return 0;
  return occ * sms;
}

void launch_bfire_steps(BFireStepsFn fn, const LaunchCfg& c, int block, const SysParams& p, const SysArrays& a,
                        const StepArgs& s, const BFire& f, int nmax) {
  fn<<<c.grid, block, 0, c.stream>>>(p, a, s, f, nmax);
}

}  // namespace cr
