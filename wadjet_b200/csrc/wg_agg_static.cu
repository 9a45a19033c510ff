// wg_agg_static.cu — the fused kernel instantiated for every compiled query
// shape (wg_shapes.cuh): one-row, vector and tile-staged variants.
#include "wg_internal.h"
#include "wg_launch.cuh"

namespace wg {

void launch_static_shape(const LaunchSpec& ls, cudaStream_t st) {
  using namespace wgd;
  switch (ls.P.shape) {
    case SHAPE_STARJOIN: launch_pipeline_t<ShapeStarJoin::n_aggs, StatShape<ShapeStarJoin>>(ls, st); return;
    case SHAPE_GROUPBY: launch_pipeline_t<ShapeGroupBy::n_aggs, StatShape<ShapeGroupBy>>(ls, st); return;
    case SHAPE_HIGHCARD: launch_pipeline_t<ShapeHighCard::n_aggs, StatShape<ShapeHighCard>>(ls, st); return;
    case SHAPE_BATCH_I64: launch_pipeline_t<ShapeBatchI64::n_aggs, StatShape<ShapeBatchI64>>(ls, st); return;
    case SHAPE_BATCH_F64: launch_pipeline_t<ShapeBatchF64::n_aggs, StatShape<ShapeBatchF64>>(ls, st); return;
    case SHAPE_IPV4: launch_pipeline_t<ShapeIPv4::n_aggs, StatShape<ShapeIPv4>>(ls, st); return;
    default: return;
  }
}

}  // namespace wg
