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


// Multi-step kernel (k_tile_steps) for one or two lanes per vertex; nullptr
// for other lane counts.
template <int POT, int INTER>
static TileStepsFn steps_fn_l(int lanes) {
  if (lanes == 1) return k_tile_steps<POT, INTER, 128, 1, PREC_MIXED>;
  if (lanes == 2) return k_tile_steps<POT, INTER, 192, 2, PREC_MIXED>;
  return nullptr;
}

TileStepsFn tile_steps_fn_mixed(int pot, int inter, int lanes) {
  const bool vv = inter == INT_VV;
  switch (pot) {
    case POT_HARMONIC: return vv ? steps_fn_l<POT_HARMONIC, INT_VV>(lanes) : steps_fn_l<POT_HARMONIC, INT_SMOOTH>(lanes);
    case POT_LJ: return vv ? steps_fn_l<POT_LJ, INT_VV>(lanes) : steps_fn_l<POT_LJ, INT_SMOOTH>(lanes);
    case POT_ADHESIVE: return vv ? steps_fn_l<POT_ADHESIVE, INT_VV>(lanes) : steps_fn_l<POT_ADHESIVE, INT_SMOOTH>(lanes);
    case POT_WCA: return vv ? steps_fn_l<POT_WCA, INT_VV>(lanes) : steps_fn_l<POT_WCA, INT_SMOOTH>(lanes);
    default: return nullptr;
  }
}

}  // namespace cr
