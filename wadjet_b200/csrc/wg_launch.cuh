// wg_launch.cuh — launch descriptions of the fused aggregate kernels and the
// host templates that launch one kernel variant for a query shape. The
// compiled-shape instantiations live in wg_agg_static.cu (their own
// translation unit, built in parallel with wg_agg.cu).
#pragma once

#include "wg_shapes.cuh"

#include <type_traits>

namespace wg {

constexpr int kAggBlock = 512;

// One launch description (device input already resident).
struct LaunchSpec {
  wgd::Plan P;
  bool smem = false;
  int block = kAggBlock;
  unsigned grid = 1;
  size_t smem_bytes = 0;
  bool tile = false;          // TMA-staged tile kernel
  wgd::TileCfg cfg{};
  int vec = 0;                // compiled shapes: rows per lane of the vector kernel (0 = one-row kernel)
  bool stage = false;         // vector kernel with a shared table: the self-staged variant (1024 threads, 1 CTA/SM)
};

template <int NA, bool SMEM, class Sh, int U, int MB, int BLK>
static void launch_vec_one(const LaunchSpec& ls, cudaStream_t st) {
  const size_t dyn = SMEM ? ls.smem_bytes : 0;
  if (SMEM) cudaFuncSetAttribute(wgd::pipeline_vec_kernel<NA, SMEM, Sh, U, MB, BLK>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
  wgd::pipeline_vec_kernel<NA, SMEM, Sh, U, MB, BLK><<<ls.grid, BLK, dyn, st>>>(ls.P);
}

// Two CTAs of 512 threads per SM, or one of 1024 when a shared table takes the
// whole SM's shared memory.
template <int NA, class Sh, bool SMEM>
static void launch_vec_s(const LaunchSpec& ls, cudaStream_t st) {
  if (ls.block == 1024) launch_vec_one<NA, SMEM, Sh, 2, 1, 1024>(ls, st);
  else if (ls.block == 768) launch_vec_one<NA, SMEM, Sh, 2, 2, 768>(ls, st);
  else launch_vec_one<NA, SMEM, Sh, 2, 2, 512>(ls, st);
}

// Self-staged vector kernel: smem_bytes covers the shared table and the
// staging buffers at P.stage_off.
template <int NA, class Sh>
static void launch_stage_one(const LaunchSpec& ls, cudaStream_t st) {
  cudaFuncSetAttribute(wgd::pipeline_stage_kernel<NA, Sh, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)ls.smem_bytes);
  wgd::pipeline_stage_kernel<NA, Sh, 2><<<ls.grid, 1024, ls.smem_bytes, st>>>(ls.P);
}

// The vector kernel exists for compiled shapes only (DynShape never gets here).
template <int NA, class Sh>
static void launch_vec_t(const LaunchSpec& ls, cudaStream_t st, bool smem) {
  if constexpr (std::is_same<Sh, wgd::DynShape>::value) {
    (void)ls; (void)st; (void)smem;
  } else {
    if constexpr (Sh::smem_ok) {
      if (smem && ls.stage) { launch_stage_one<NA, Sh>(ls, st); return; }
      if (smem) { launch_vec_s<NA, Sh, true>(ls, st); return; }
    }
    launch_vec_s<NA, Sh, false>(ls, st);
  }
}

template <int NA, class Sh>
static void launch_pipeline_t(const LaunchSpec& ls, cudaStream_t st) {
  const bool smem = Sh::smem_ok && ls.smem;
  if (ls.tile) {
    const size_t dyn = (size_t)ls.cfg.table_off + (smem ? (size_t)ls.P.smem_slots * ls.P.L.slot_words * 8 : 0);
    const unsigned threads = 32u * (1u + (unsigned)ls.cfg.consumers);
    if constexpr (Sh::smem_ok) {
      if (smem) {
        cudaFuncSetAttribute(wgd::tile_pipeline_kernel<NA, true, Sh>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dyn);
        wgd::tile_pipeline_kernel<NA, true, Sh><<<ls.grid, threads, dyn, st>>>(ls.P, ls.cfg);
        return;
      }
    }
    cudaFuncSetAttribute(wgd::tile_pipeline_kernel<NA, false, Sh>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    wgd::tile_pipeline_kernel<NA, false, Sh><<<ls.grid, threads, dyn, st>>>(ls.P, ls.cfg);
    return;
  }
  if (ls.vec > 0) {
    launch_vec_t<NA, Sh>(ls, st, smem);
    return;
  }
  if constexpr (Sh::smem_ok) {
    if (smem) {
      cudaFuncSetAttribute(wgd::pipeline_kernel<NA, true, Sh>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ls.smem_bytes);
      wgd::pipeline_kernel<NA, true, Sh><<<ls.grid, ls.block, ls.smem_bytes, st>>>(ls.P);
      return;
    }
  }
  wgd::pipeline_kernel<NA, false, Sh><<<ls.grid, ls.block, 0, st>>>(ls.P);
}


// Launch a compiled shape (defined in wg_agg_static.cu).
void launch_static_shape(const LaunchSpec& ls, cudaStream_t st);

}  // namespace wg
