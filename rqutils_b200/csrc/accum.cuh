// Matvec accumulators: plain FMA in FP64; in FP32 a compensated sum after Ogita, Rump and Oishi
// (SIAM J. Sci. Comput. 26, 2005).  Single products (add) use their Dot2 step: TwoProduct via
// fma and TwoSum, as accurate as twice the working precision.  The unrolled loops (add4) sum
// four products by an FMA chain and compensate only the running sum: the elements are FP32
// numbers already rounded once, so the chain's few roundings stay at that level, and the sum
// over the row keeps a bounded error however long the row is.
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
  // s + p with the rounding error of the addition kept in c (TwoSum).
  __device__ __forceinline__ void add_sum(R p) {
    if constexpr (sizeof(R) == 8) {
      s += p;
    } else {
      const R t = s + p;
      const R bp = t - s;
      const R es = (s - (t - bp)) + (p - bp);
      s = t;
      c += es;
    }
  }
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
  // Partial sums kept in FP64 between kernels: the FP32 state (s, c) is exact in a double up
  // to the double's rounding, and a double splits back into (hi, lo) floats.
  __device__ __forceinline__ double value_d() const {
    return sizeof(R) == 8 ? double(s) : double(s) + double(c);
  }
  __device__ __forceinline__ void add_d(double d) {
    if constexpr (sizeof(R) == 8) {
      s += d;
    } else {
      const R hi = static_cast<R>(d);
      const R lo = static_cast<R>(d - double(hi));
      add_sum(hi);
      c += lo;
    }
  }
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
  // Four products at once.  FP64: four FMAs.  FP32: the products are summed by an FMA chain
  // whose result enters the compensated sum.
  __device__ __forceinline__ void add4(const Cx<R>* a, const Cx<R>* x) {
    if constexpr (sizeof(R) == 8) {
#pragma unroll
      for (int u = 0; u < 4; ++u) add(a[u], x[u]);
    } else {
      R pr = 0, pi = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        pr = fmaf(a[u].re, x[u].re, pr);
        if constexpr (NCV == 2) {
          if constexpr (NCA == 2) pr = fmaf(-a[u].im, x[u].im, pr);
          pi = fmaf(a[u].re, x[u].im, pi);
          if constexpr (NCA == 2) pi = fmaf(a[u].im, x[u].re, pi);
        }
      }
      re.add_sum(pr);
      if constexpr (NCV == 2) im.add_sum(pi);
    }
  }
  __device__ __forceinline__ void merge(int width) {
    re.merge_lanes(width);
    if constexpr (NCV == 2) im.merge_lanes(width);
  }
  // FP64 partial at element i of a double array (NCV doubles per element).
  __device__ __forceinline__ void add_partial(const double* p, int64_t i) {
    if constexpr (NCV == 2) {
      const double2 d = reinterpret_cast<const double2*>(p)[i];
      re.add_d(d.x);
      im.add_d(d.y);
    } else {
      re.add_d(p[i]);
    }
  }
  __device__ __forceinline__ void store_partial(double* p, int64_t i) const {
    if constexpr (NCV == 2)
      reinterpret_cast<double2*>(p)[i] = make_double2(re.value_d(), im.value_d());
    else
      p[i] = re.value_d();
  }
};

// One lane's share of a CSR row: pairs i0, i0 + LPR, ... below e.  Four pairs per step with
// independent index -> amplitude gathers in flight, then the remainder.
// CG: read v through L2 (v written earlier in the same launch by other blocks).
template <typename R, int NCV, int NCA, int LPR, bool CG = false>
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
      x[u] = CG ? ld_elem_cg<R, NCV>(v, c[u]) : ld_elem<R, NCV>(v, c[u]);
    }
    acc.add4(a, x);
  }
  // The remainder (fewer than four pairs): for FP32 rows shared by at most four lanes (short
  // rows, such as the two-half tails at 48 qubits) one predicated step, so its gathers are in
  // flight together, absent pairs adding exact zeros; otherwise one pair at a time (measured
  // faster there: FP64 tails, and FP32 rows spread over 8-16 lanes).
  if constexpr (sizeof(R) == 4 && LPR <= 4) {
    if (i < e) {
      uint32_t c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = (i + u * LPR < e) ? __ldg(cols + i + u * LPR) : 0u;
      Cx<R> a[4], x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const bool ok = i + u * LPR < e;
        a[u] = ok ? ld_elem<R, NCA>(vals, i + u * LPR) : cx_make<R>(R(0), R(0));
        x[u] = ok ? (CG ? ld_elem_cg<R, NCV>(v, c[u]) : ld_elem<R, NCV>(v, c[u]))
                  : cx_make<R>(R(0), R(0));
      }
      acc.add4(a, x);
    }
  } else {
    for (; i < e; i += LPR)
      acc.add(ld_elem<R, NCA>(vals, i),
              CG ? ld_elem_cg<R, NCV>(v, __ldg(cols + i)) : ld_elem<R, NCV>(v, __ldg(cols + i)));
  }
}

}  // namespace sqd
