// Mixed-precision instantiations of the tiled force + integrator kernel:
// FP64 positions, velocities, shape terms, integration and reductions; FP32
// pair terms on FP64-formed offsets.
#include "cr_launch.h"
#include "cr_tile_kernel.cuh"

namespace cr {

template <int POT, int INTER, int MODE>
static void launch_mixed_t(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s) {
  if (c.lanes == 1) launch_k(c.pdl, k_tile<POT, INTER, MODE, 128, 1, PREC_MIXED>, dim3(c.grid), dim3(128), c.stream, p, a, s);
  else if (c.lanes == 4) launch_k(c.pdl, k_tile<POT, INTER, MODE, 256, 4, PREC_MIXED>, dim3(c.grid), dim3(256), c.stream, p, a, s);
  else if (c.lanes == 8) launch_k(c.pdl, k_tile<POT, INTER, MODE, 256, 8, PREC_MIXED>, dim3(c.grid), dim3(256), c.stream, p, a, s);
  else launch_k(c.pdl, k_tile<POT, INTER, MODE, 192, 2, PREC_MIXED>, dim3(c.grid), dim3(192), c.stream, p, a, s);
}

void launch_tile_mixed(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p, const SysArrays& a,
                       const StepArgs& s) {
#define CR_MIXED_CASE(P)                                                                \
  case P:                                                                               \
    if (inter == INT_VV) {                                                              \
      if (mode == MODE_FORCE) launch_mixed_t<P, INT_VV, MODE_FORCE>(c, p, a, s);        \
      else launch_mixed_t<P, INT_VV, MODE_STEP>(c, p, a, s);                            \
    } else {                                                                            \
      if (mode == MODE_FORCE) launch_mixed_t<P, INT_SMOOTH, MODE_FORCE>(c, p, a, s);    \
      else launch_mixed_t<P, INT_SMOOTH, MODE_STEP>(c, p, a, s);                        \
    }                                                                                   \
    break;
  switch (pot) {
    CR_MIXED_CASE(POT_HARMONIC)
    CR_MIXED_CASE(POT_LJ)
    CR_MIXED_CASE(POT_ADHESIVE)
    CR_MIXED_CASE(POT_WCA)
    default: break;
  }
#undef CR_MIXED_CASE
}

}  // namespace cr
