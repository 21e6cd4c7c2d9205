// Matvec accumulators: plain FMA in FP64; in FP32 the compensated dot product of Ogita, Rump
// and Oishi (SIAM J. Sci. Comput. 26, 2005): TwoProduct via fma and TwoSum, so the FP32 result is
// as accurate as if accumulated in twice the working precision.
#pragma once
#include "common.cuh"

namespace sqd {

template <typename R>
struct Acc {
  R s = 0, c = 0;
  __device__ __forceinline__ void add_prod(R a, R b) {
    if constexpr (sizeof(R) == 8) {
      s = fma(a, b, s);
    } else {
      const R p = a * b;
      const R ep = fmaf(a, b, -p);
      const R t = s + p;
      const R bp = t - s;
      const R es = (s - (t - bp)) + (p - bp);
      s = t;
      c += ep + es;
    }
  }
  __device__ __forceinline__ void add_neg_prod(R a, R b) { add_prod(-a, b); }
  __device__ __forceinline__ void merge_lanes(int width) {
    for (int o = width >> 1; o > 0; o >>= 1) {
      const R os = __shfl_xor_sync(kFullMask, s, o);
      if constexpr (sizeof(R) == 8) {
        s += os;
      } else {
        const R oc = __shfl_xor_sync(kFullMask, c, o);
        const R t = s + os;
        const R bp = t - s;
        const R es = (s - (t - bp)) + (os - bp);
        s = t;
        c += oc + es;
      }
    }
  }
  __device__ __forceinline__ R value() const { return sizeof(R) == 8 ? s : s + c; }
};

template <typename R, int NCV, int NCA>
struct CAcc {
  Acc<R> re, im;
  __device__ __forceinline__ void add(Cx<R> a, Cx<R> x) {
    re.add_prod(a.re, x.re);
    if constexpr (NCV == 2) re.add_neg_prod(a.im, x.im);
    if constexpr (NCV == 2) {
      im.add_prod(a.re, x.im);
      if constexpr (NCA == 2) im.add_prod(a.im, x.re);
    }
  }
  __device__ __forceinline__ void merge(int width) {
    re.merge_lanes(width);
    if constexpr (NCV == 2) im.merge_lanes(width);
  }
};

// One lane's share of a CSR row: pairs i0, i0 + LPR, ... below e.  Four pairs per step with
// independent index -> amplitude gathers in flight, then the remainder.
template <typename R, int NCV, int NCA, int LPR>
__device__ __forceinline__ void csr_row_dot(const uint32_t* __restrict__ cols,
                                            const R* __restrict__ vals,
                                            const R* __restrict__ v, int64_t i0, int64_t e,
                                            CAcc<R, NCV, NCA>& acc) {
  int64_t i = i0;
  for (; i + 3 * LPR < e; i += 4 * LPR) {
    uint32_t c[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) c[u] = __ldg(cols + i + u * LPR);
    Cx<R> a[4], x[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = ld_elem<R, NCA>(vals, i + u * LPR);
      x[u] = ld_elem<R, NCV>(v, c[u]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) acc.add(a[u], x[u]);
  }
  for (; i < e; i += LPR) acc.add(ld_elem<R, NCA>(vals, i), ld_elem<R, NCV>(v, __ldg(cols + i)));
}

}  // namespace sqd
