// wg_agg_static.cu — the fused kernel instantiated for every compiled query
// shape (wg_shapes.cuh): one-row, vector and tile-staged variants.
#include "wg_internal.h"
#include "wg_launch.cuh"
#include "wg_star.cuh"

#include <cstdlib>

namespace wg {

// The star-join shape's lean kernel (wg_star.cuh) when the launch is the
// vector kernel with a shared table and the plan has its physical form
// (WG_STAR_LEAN=0 keeps the generic vector kernel).
template <int REP>
static void launch_star_dense(const LaunchSpec& ls, cudaStream_t st) {
  cudaFuncSetAttribute(wgd::starjoin_dense_kernel<REP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)ls.smem_bytes);
  wgd::starjoin_dense_kernel<REP><<<ls.grid, 768, ls.smem_bytes, st>>>(ls.P);
}

static bool launch_star_lean(const LaunchSpec& ls, cudaStream_t st) {
  static const bool on = [] {
    const char* v = std::getenv("WG_STAR_LEAN");
    return !v || std::atoi(v) != 0;
  }();
  if (!on || ls.vec == 0 || !ls.smem || ls.tile || ls.stage || ls.block != 768 || !wgd::starjoin_dense_ok(ls.P))
    return false;
  switch (ls.P.smem_rep) {
    case 1: launch_star_dense<1>(ls, st); return true;
    case 2: launch_star_dense<2>(ls, st); return true;
    case 4: launch_star_dense<4>(ls, st); return true;
    default: launch_star_dense<8>(ls, st); return true;
  }
}

void launch_static_shape(const LaunchSpec& ls, cudaStream_t st) {
  using namespace wgd;
  switch (ls.P.shape) {
    case SHAPE_STARJOIN:
      if (launch_star_lean(ls, st)) return;
      launch_pipeline_t<ShapeStarJoin::n_aggs, StatShape<ShapeStarJoin>>(ls, st);
      return;
    case SHAPE_GROUPBY: launch_pipeline_t<ShapeGroupBy::n_aggs, StatShape<ShapeGroupBy>>(ls, st); return;
    case SHAPE_HIGHCARD: launch_pipeline_t<ShapeHighCard::n_aggs, StatShape<ShapeHighCard>>(ls, st); return;
    case SHAPE_BATCH_I64: launch_pipeline_t<ShapeBatchI64::n_aggs, StatShape<ShapeBatchI64>>(ls, st); return;
    case SHAPE_BATCH_F64: launch_pipeline_t<ShapeBatchF64::n_aggs, StatShape<ShapeBatchF64>>(ls, st); return;
    case SHAPE_IPV4: launch_pipeline_t<ShapeIPv4::n_aggs, StatShape<ShapeIPv4>>(ls, st); return;
    default: return;
  }
}

}  // namespace wg
