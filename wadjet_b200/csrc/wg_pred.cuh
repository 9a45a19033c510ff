// wg_pred.cuh — typed `col OP const` predicates (kernel.compareFilterImpl,
// internal/engine/exec/kernel/compare.go:47-90). The constant is resolved on the
// host to the column's storage type exactly as ResolveFilterKernel does
// (compare.go:145-182); comparisons are IEEE for floats (NaN compares false
// except !=), signed for integers.
#pragma once

#include "wg_device.cuh"

namespace wgd {

struct Pred {
  int32_t col;
  int32_t op;
  int32_t cls;        // storage class of the column
  int32_t _pad;
  long long ci;       // constant for integer classes (already truncated to int32 for I32)
  double cf;          // constant for float classes (already rounded to float32 for F32)
};

template <typename T>
__device__ __forceinline__ bool cmp_op(T a, T b, int op) {
  switch (op) {
    case 0: return a == b;
    case 1: return a != b;
    case 2: return a < b;
    case 3: return a <= b;
    case 4: return a > b;
    case 5: return a >= b;
    default: return false;
  }
}

// Evaluate the predicate on row i of column c (NULL never matches).
__device__ __forceinline__ bool pred_row(const Pred& p, const DCol& c, int64_t i) {
  if (is_null(c, i)) return false;
  switch (p.cls) {
    case WG_CLS_I32: return cmp_op<int32_t>(__ldg((const int32_t*)c.data + i), (int32_t)p.ci, p.op);
    case WG_CLS_I64: return cmp_op<long long>(__ldg((const long long*)c.data + i), p.ci, p.op);
    case WG_CLS_F32: return cmp_op<float>(__ldg((const float*)c.data + i), (float)p.cf, p.op);
    case WG_CLS_F64: return cmp_op<double>(__ldg((const double*)c.data + i), p.cf, p.op);
    default: return false;
  }
}

}  // namespace wgd
