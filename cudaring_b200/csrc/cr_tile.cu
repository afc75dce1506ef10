// FP64 instantiations of the tiled force + integrator kernel and the launcher
// that dispatches on potential, interaction, mode, lanes and precision.
#include "cr_launch.h"
#include "cr_tile_kernel.cuh"

namespace cr {

template <int POT, int INTER, int MODE>
static void launch_tile_t(const LaunchCfg& c, const SysParams& p, const SysArrays& a, const StepArgs& s) {
  if (c.lanes == 1) launch_k(c.pdl, k_tile<POT, INTER, MODE, 128, 1, PREC_FP64>, dim3(c.grid), dim3(128), c.stream, p, a, s);
  else if (c.lanes == 4) launch_k(c.pdl, k_tile<POT, INTER, MODE, 256, 4, PREC_FP64>, dim3(c.grid), dim3(256), c.stream, p, a, s);
  else if (c.lanes == 8) launch_k(c.pdl, k_tile<POT, INTER, MODE, 256, 8, PREC_FP64>, dim3(c.grid), dim3(256), c.stream, p, a, s);
  else launch_k(c.pdl, k_tile<POT, INTER, MODE, 192, 2, PREC_FP64>, dim3(c.grid), dim3(192), c.stream, p, a, s);
}

void launch_tile(const LaunchCfg& c, int pot, int inter, int mode, const SysParams& p_in, const SysArrays& a,
                 const StepArgs& s) {
  // both paths read the FP32 range constants in the unit skip test
  const SysParams p = with_f32_constants(p_in);
  if (c.precision == CR_PRECISION_MIXED) {
    launch_tile_mixed(c, pot, inter, mode, p, a, s);
    return;
  }
#define CR_TILE_CASE(P)                                                                 \
  case P:                                                                               \
    if (inter == INT_VV) {                                                              \
      if (mode == MODE_FORCE) launch_tile_t<P, INT_VV, MODE_FORCE>(c, p, a, s);         \
      else launch_tile_t<P, INT_VV, MODE_STEP>(c, p, a, s);                             \
    } else {                                                                            \
      if (mode == MODE_FORCE) launch_tile_t<P, INT_SMOOTH, MODE_FORCE>(c, p, a, s);     \
      else launch_tile_t<P, INT_SMOOTH, MODE_STEP>(c, p, a, s);                         \
    }                                                                                   \
    break;
  switch (pot) {
    CR_TILE_CASE(POT_HARMONIC)
    CR_TILE_CASE(POT_LJ)
    CR_TILE_CASE(POT_ADHESIVE)
    CR_TILE_CASE(POT_WCA)
    default: break;
  }
#undef CR_TILE_CASE
}

// Tile capacity (vertices of whole rings per CTA) for a lane count:
// 1 -> 128 threads x 1, 2 -> 192 x 2, 4 -> 256 x 4, 8 -> 256 x 8.
int tile_vertices(int lanes) { return lanes >= 4 ? 256 / lanes : (lanes == 2 ? 96 : 128); }


// Multi-step kernel (k_tile_steps) for one or two lanes per vertex; nullptr
// for other lane counts.
template <int POT, int INTER>
static TileStepsFn steps_fn_l(int lanes) {
  if (lanes == 1) return k_tile_steps<POT, INTER, 128, 1, PREC_FP64>;
  if (lanes == 2) return k_tile_steps<POT, INTER, 192, 2, PREC_FP64>;
  return nullptr;
}

TileStepsFn tile_steps_fn_fp64(int pot, int inter, int lanes) {
  const bool vv = inter == INT_VV;
  switch (pot) {
    case POT_HARMONIC: return vv ? steps_fn_l<POT_HARMONIC, INT_VV>(lanes) : steps_fn_l<POT_HARMONIC, INT_SMOOTH>(lanes);
    case POT_LJ: return vv ? steps_fn_l<POT_LJ, INT_VV>(lanes) : steps_fn_l<POT_LJ, INT_SMOOTH>(lanes);
    case POT_ADHESIVE: return vv ? steps_fn_l<POT_ADHESIVE, INT_VV>(lanes) : steps_fn_l<POT_ADHESIVE, INT_SMOOTH>(lanes);
    case POT_WCA: return vv ? steps_fn_l<POT_WCA, INT_VV>(lanes) : steps_fn_l<POT_WCA, INT_SMOOTH>(lanes);
    default: return nullptr;
  }
}

static TileStepsFn steps_fn(int pot, int inter, int lanes, int precision) {
  return precision == CR_PRECISION_MIXED ? tile_steps_fn_mixed(pot, inter, lanes) : tile_steps_fn_fp64(pot, inter, lanes);
}

int tile_steps_max_blocks(int pot, int inter, int lanes, int precision) {
  TileStepsFn k = steps_fn(pot, inter, lanes, precision);
  if (!k) return 0;
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, lanes == 1 ? 128 : 192, 0) != cudaSuccess) return 0;
  return occ * sms;
}

cudaError_t launch_tile_steps(const LaunchCfg& c, int pot, int inter, const SysParams& p_in, const SysArrays& a,
                              const StepArgs& s) {
  TileStepsFn k = steps_fn(pot, inter, c.lanes, c.precision);
  if (!k) return cudaErrorInvalidValue;
  const SysParams p = with_f32_constants(p_in);
  return launch_k(c.pdl, k, dim3(c.grid), dim3(c.lanes == 1 ? 128 : 192), c.stream, p, a, s);
}

}  // namespace cr
