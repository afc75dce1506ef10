// Batch-mode instantiations of the tiled force + integrator kernel (many
// independent systems in one grid; see BatchSys), FP64 and mixed precision.
#include "cr_launch.h"
#include "cr_tile_kernel.cuh"

namespace cr {

int batch_tile_block(int lanes, int block) {
  if (lanes == 1) return block == 0 ? 128 : ((block == 128 || block == 192) ? block : 0);
  if (lanes == 2) return block == 0 ? 192 : ((block == 128 || block == 192) ? block : 0);
  if (lanes == 4) return (block == 0 || block == 256) ? 256 : 0;
  return 0;
}

template <int POT, int INTER, int MODE, int PREC>
static void launch_batch_t(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s) {
  const int block = batch_tile_block(c.lanes, c.block);
  if (c.lanes == 1) {
    if (block == 192) k_tile<POT, INTER, MODE, 192, 1, PREC, true><<<c.grid, 192, 0, c.stream>>>(p, a, s);
    else k_tile<POT, INTER, MODE, 128, 1, PREC, true><<<c.grid, 128, 0, c.stream>>>(p, a, s);
  } else if (c.lanes == 4) {
    k_tile<POT, INTER, MODE, 256, 4, PREC, true><<<c.grid, 256, 0, c.stream>>>(p, a, s);
  } else {
    if (block == 128) k_tile<POT, INTER, MODE, 128, 2, PREC, true><<<c.grid, 128, 0, c.stream>>>(p, a, s);
    else k_tile<POT, INTER, MODE, 192, 2, PREC, true><<<c.grid, 192, 0, c.stream>>>(p, a, s);
  }
}

template <int PREC>
static void launch_batch_p(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                           const StepArgs& s) {
#define CR_BATCH_CASE(P)                                                                   \
  case P:                                                                                  \
    if (inter == INT_VV) {                                                                 \
      if (mode == MODE_FORCE) launch_batch_t<P, INT_VV, MODE_FORCE, PREC>(c, p, a, s);     \
      else launch_batch_t<P, INT_VV, MODE_STEP, PREC>(c, p, a, s);                         \
    } else {                                                                               \
      if (mode == MODE_FORCE) launch_batch_t<P, INT_SMOOTH, MODE_FORCE, PREC>(c, p, a, s); \
      else launch_batch_t<P, INT_SMOOTH, MODE_STEP, PREC>(c, p, a, s);                     \
    }                                                                                      \
    break;
  switch (pot) {
    CR_BATCH_CASE(POT_HARMONIC)
    CR_BATCH_CASE(POT_LJ)
    CR_BATCH_CASE(POT_ADHESIVE)
    CR_BATCH_CASE(POT_WCA)
    default: break;
  }
#undef CR_BATCH_CASE
}

void launch_tile_batch(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p_in, const SysArrays& a,
                       const StepArgs& s) {
  const SysParams p = with_f32_constants(p_in);
  if (c.precision == CR_PRECISION_MIXED) launch_batch_p<PREC_MIXED>(c, pot, inter, mode, p, a, s);
  else launch_batch_p<PREC_FP64>(c, pot, inter, mode, p, a, s);
}

}  // namespace cr
