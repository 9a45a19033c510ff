// wg_star.cuh — the compiled star-join shape in its common physical form, with
// every runtime choice of the generic vector kernel fixed at compile time.
//
// ShapeStarJoin is `qty > c` → probe `fk` in a unique int32 dimension index →
// GROUP BY the dimension's payload, SUM(price * (1 - disc)) as float64 and
// SUM(price) as Int128 (`price` DECIMAL, `disc` float64). When the dimension's
// keys fill their range (the payload-only dense index, JoinView.dense == 2)
// and the payload's value range fits the shared table (dense groups,
// Plan.gdense), each row is: two vector loads' worth of columns, one compare,
// one dependent 4-byte load, one DECIMAL-to-float64 conversion and division,
// and three shared-memory updates. pipeline_vec_kernel does the same work
// through the generic plan (join flavour, group placement, float-SUM copies and
// NULL handling decided per row from the plan) and issues about 2.8x the
// instructions; this kernel keeps only the per-row work, so it is bound by the
// shared-memory atomics instead of instruction issue.
//
// Semantics are the generic kernel's, operation for operation: the filter and
// the probe drop the row; the DECIMAL operand is Int128.ToFloat64 then the
// correctly rounded division by 10^scale (div_by_recip with the plan's divisor
// pair); the projection is RN(price * RN(c1 - disc)) with c1 the program's
// constant; a zero float contribution is skipped as apply() skips it; the
// DECIMAL sum goes limb by limb; the row count is the slot's 32-bit counter;
// float-SUM copies are lane-striped (copy lane % REP) and folded by the flush.
#pragma once

#include "wg_shapes.cuh"

namespace wgd {

// Whether a plan (already matched to ShapeStarJoin, on the vector path with a
// shared table) has the physical form the lean kernel serves.
__host__ __forceinline__ bool starjoin_dense_ok(const Plan& P) {
  return P.gdense && P.join.dense == 2 && P.smem_slots > 0 && P.smem_combine == 0 && P.sel == nullptr &&
         (P.smem_rep == 1 || P.smem_rep == 2 || P.smem_rep == 4 || P.smem_rep == 8);
}

template <int REP>
__global__ void __launch_bounds__(768, 2) starjoin_dense_kernel(const __grid_constant__ Plan P) {
  using C = ShapeStarJoin;
  static_assert(C::key_words == 1 && C::slot_words == 5 && C::agg_off(0) == 2 && C::agg_off(1) == 3,
                "slot layout of the star-join shape");
  extern __shared__ unsigned long long sm[];
  __shared__ int s_groups;
  Credit cr;
  const int S = P.smem_slots;
  smem_table_init(P, sm, S, &s_groups);
  __syncthreads();
  const int ssw = smem_stride(P);
  const int lane = threadIdx.x & 31;
  const int copy = lane & (REP - 1);  // this lane's float-SUM copy
  // columns: 0 qty int32, 1 fk int32, 2 price DECIMAL, 3 disc float64
  const int32_t* qty = (const int32_t*)P.in[0].data;
  const int32_t* fk = (const int32_t*)P.in[1].data;
  const longlong2* price = (const longlong2*)P.in[2].data;
  const double* disc = (const double*)P.in[3].data;
  const int32_t cq = (int32_t)P.filt[0].ci;
  const uint32_t jbase = (uint32_t)P.join.base;
  const uint32_t jspan = (uint32_t)P.join.mask;
  const uint32_t* pay = (const uint32_t*)P.join.slots;
  const bool keep = P.join.l2keep != 0;
  const uint32_t gmin = (uint32_t)P.gmin;
  const double db = P.vdiv_b[2], dy = P.vdiv_y[2];
  const double c1 = as_f((unsigned long long)P.expr[0].imm[1]);
  const int64_t n = P.n_items;
  const int64_t wpb = blockDim.x >> 5;
  const int64_t step = (int64_t)gridDim.x * wpb * 64;
  for (int64_t base = ((int64_t)blockIdx.x * wpb + (threadIdx.x >> 5)) * 64; base < n; base += step) {
    const int64_t r0 = base + 2 * lane;
    int32_t q[2], f[2];
    long long ph[2];
    unsigned long long pl[2];
    double d[2];
    bool act[2];
    if (r0 + 2 <= n) {
      const int2 qv = __ldcs((const int2*)(qty + r0));
      const int2 fv = __ldcs((const int2*)(fk + r0));
      const longlong2 p0 = __ldcs(price + r0), p1 = __ldcs(price + r0 + 1);
      const double2 dv = __ldcs((const double2*)(disc + r0));
      q[0] = qv.x; q[1] = qv.y; f[0] = fv.x; f[1] = fv.y;
      ph[0] = p0.x; pl[0] = (unsigned long long)p0.y; ph[1] = p1.x; pl[1] = (unsigned long long)p1.y;
      d[0] = dv.x; d[1] = dv.y;
      act[0] = act[1] = true;
    } else {
      act[0] = r0 < n;
      act[1] = false;
      q[0] = act[0] ? qty[r0] : 0; f[0] = act[0] ? fk[r0] : 0;
      const longlong2 p0 = act[0] ? price[r0] : make_longlong2(0, 0);
      ph[0] = p0.x; pl[0] = (unsigned long long)p0.y;
      d[0] = act[0] ? disc[r0] : 0.0;
      q[1] = 0; f[1] = 0; ph[1] = 0; pl[1] = 0; d[1] = 0.0;
    }
    uint32_t g[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {  // filter, then the probe (both payload loads in flight together)
      act[u] = act[u] && cmp_op<int32_t>(q[u], cq, C::filt_op(0));
      const uint32_t i = (uint32_t)f[u] - jbase;
      act[u] = act[u] && i < jspan;
      g[u] = act[u] ? (keep ? ld_keep_u32(pay + i) : __ldg(pay + i)) - gmin : 0u;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (!act[u]) continue;
      if (g[u] >= (uint32_t)S) {  // a payload outside the range the table was sized for
        set_error(P.err, WG_DERR_TABLE_FULL);
        continue;
      }
      unsigned long long* s = sm + (size_t)g[u] * ssw;
      const double pf = div_by_recip(int128_to_f64(ph[u], pl[u]), db, dy);
      const double v = __dmul_rn(pf, __dsub_rn(c1, d[u]));
      atomicAdd((unsigned*)(s + 1), 1u);
      if (v != 0.0) atomicAdd((double*)(copy == 0 ? s + 2 : s + 5 + (copy - 1)), v);
      smem_add_limbs((unsigned*)(s + 3), 4, pl[u], (unsigned long long)ph[u]);
    }
  }
  __syncthreads();
  smem_table_flush<2>(P, sm, S, cr);
  cr.release(P.T);
}

}  // namespace wgd
