// spmv_row.cuh -- one block-row of a BCSR product with LPR cooperating lanes.
#pragma once
#include "maspcg_internal.cuh"

namespace maspcg {

template <typename T>
struct AccOf {
  using type = float;
};
template <>
struct AccOf<double> {
  using type = double;
};

__device__ __forceinline__ float ldv(const float* p) { return __ldg(p); }
__device__ __forceinline__ double ldv(const double* p) { return __ldg(p); }

// y_row = sum_t B_t x_{col_t} over the row, reduced over LPR lanes (all lanes
// of the group get the result).  Blocks are row-major.
template <typename Tm, typename Tv, int LPR>
__device__ __forceinline__ void row_product(int rs, int re, const int* __restrict__ colidx, const Tm* __restrict__ val,
                                            const Tv* __restrict__ x, int sub, typename AccOf<Tm>::type acc[3])
{
  using A = typename AccOf<Tm>::type;
  A a0 = 0, a1 = 0, a2 = 0;
  for (int t = rs + sub; t < re; t += LPR) {
    const int c = __ldg(colidx + t);
    const Tm* B = val + 9 * (size_t)t;
    const A x0 = (A)ldv(x + 3 * (size_t)c), x1 = (A)ldv(x + 3 * (size_t)c + 1), x2 = (A)ldv(x + 3 * (size_t)c + 2);
    const A b0 = (A)ldv(B), b1 = (A)ldv(B + 1), b2 = (A)ldv(B + 2), b3 = (A)ldv(B + 3), b4 = (A)ldv(B + 4),
            b5 = (A)ldv(B + 5), b6 = (A)ldv(B + 6), b7 = (A)ldv(B + 7), b8 = (A)ldv(B + 8);
    a0 += b0 * x0 + b1 * x1 + b2 * x2;
    a1 += b3 * x0 + b4 * x1 + b5 * x2;
    a2 += b6 * x0 + b7 * x1 + b8 * x2;
  }
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(kFull, a0, o, LPR);
    a1 += __shfl_xor_sync(kFull, a1, o, LPR);
    a2 += __shfl_xor_sync(kFull, a2, o, LPR);
  }
  acc[0] = a0;
  acc[1] = a1;
  acc[2] = a2;
}

}  // namespace maspcg
