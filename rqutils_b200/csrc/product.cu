// Product-subspace layout of the cached matvec (cache_strategy (1, 2)).
//
// SQD subspaces are usually the Cartesian product of strings on the high half of the qubits
// (beta) and strings on the low half (alpha).  Sorted, row r = h * nl + l holds H[h] | L[l].
// The stored pairs of a row come in three classes (k_gpre_flags, operator.cu):
//   H: x on the high half only, source (h', l) with H[h'] = H[h] ^ x.  Every row of slab h has
//      the same H sources in the same order;
//   L: the diagonal group and x on the low half only, source (h, l') with L[l'] = L[l] ^ x.
//      Every row with low string l has the same L sources in the same order;
//   M: the rest (both halves change).
// An H or L source is implied by (slab, position), so the elements of those pairs are laid out
// again as dense slabs and the matvec streams them with coalesced loads and gathers v (or its
// transpose vT[l][h]) with coalesced loads too, instead of one scattered gather and one index
// per pair.  One matvec is five launches:
//   1. vT = transpose(v)                                (32 x 32 tiles through shared memory)
//   2. t2[l][h] = sum_e VL(lo[l] + e, h) vT[l'_e][h]     (L part; FP64 partial)
//   3. t2' = transpose(t2) into the vT buffer           (now [h][l])
//   4. t3[r] = sum of the row's M pairs                  (FP64 partial; see below)
//   5. out[h][l] = t2'[h][l] + t3[r] + sum_k VH(ho[h] + k, l) v[h'_k][l]
// Steps 2 and 5 are one kernel (k_slab) over an A x B grid of outputs (A slabs of B rows each,
// A = nh for H, A = nl for L): a warp owns one slab a and 32 consecutive b (one "panel"), a
// block 8 slabs of the same panel, and blocks run panel-major, so the 32-wide panel of the
// gathered vector stays in L2 while all slabs pass over it.  The elements are stored in the
// same panel-major order, VH(k, l) at ((l / 32) * KH + k) * 32 + l % 32 (KH = entries of all
// slabs), so the element stream of a panel pass is one contiguous sweep.  Source indices are
// kept premultiplied (h' * nl, l' * nh).  At 48 qubits the FP64 passes stream their elements
// at ~5 TB/s while L2 serves one amplitude per entry (~19 TB/s).  The FP32 copies of the slabs
// of even-sized halves use 64-wide panels, read by k_slab2 with two adjacent positions per
// lane (paired 16-byte amplitude loads).
// Step 4: when all M source slabs of every slab fit in shared memory together (small slabs,
// e.g. 512 strings per half), k_tail_smem stages them per block and gathers from shared
// memory through 16-bit indices of a compact copy of the row tails; otherwise (and under
// SQD_LAYOUT_PRODUCT_CSR) the CSR kernel runs over the row tails, gathering from global
// memory: from a contiguous copy of the tails (row offsets, elements, source rows) when they
// average at most kCompactTailMax pairs per row, else inside the rows' pair lists.
// FP32 vectors keep the compensated accumulation in every part and pass partials in FP64, so
// the result is rounded once.  The elements are the same numbers as in the CSR arrays; only
// the summation order of a row changes (L and M pairs before H pairs).
//
// The file also builds the connectivity itself for such subspaces (op_connect_product): the
// partners of every string of each half, then each row's pairs assembled from them.
#include <cstdlib>
#include <algorithm>
#include <climits>
#include <type_traits>
#include <vector>

#include "internal.cuh"
#include "dispatch.cuh"
#include "accum.cuh"

namespace sqd {
namespace {

__device__ __forceinline__ void warp_count_add(unsigned long long c, unsigned long long* dst) {
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFullMask, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(dst, c);
}

// Number of distinct high strings (rows whose high half differs from the previous row's).
__global__ void k_count_slabs(const uint64_t* __restrict__ s, int64_t n, uint64_t mhi,
                              unsigned long long* cnt) {
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x)
    if (r == 0 || ((s[r] ^ s[r - 1]) & mhi) != 0) ++c;
  warp_count_add(c, cnt);
}

// Rows that are not H[r / nl] | L[r % nl].
__global__ void k_check_product(const uint64_t* __restrict__ s, int64_t n, int64_t nl,
                                uint64_t mlo, uint64_t mhi, unsigned long long* bad) {
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t l = r % nl;
    const uint64_t v = s[r];
    if (((v ^ s[l]) & mlo) != 0 || ((v ^ s[r - l]) & mhi) != 0) ++c;
  }
  warp_count_add(c, bad);
}

// Per row: the H pairs that follow the diagonal entry and the L pairs after them; a pair of
// another class before the M pairs end counts as an error.
__global__ void k_row_kinds(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ grps,
                            const uint64_t* __restrict__ group_x, int64_t n, int d, uint64_t mlo,
                            uint64_t mhi, int32_t* rkh, int32_t* rkl, unsigned long long* bad) {
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    int64_t i = row_ptr[r];
    const int64_t e = row_ptr[r + 1];
    bool ok = true;
    if (d) {
      ok = i < e && grps[i] == 0;
      ++i;
    }
    const int64_t b = i;
    while (i < e && (__ldg(group_x + grps[i]) & mlo) == 0) ++i;
    const int64_t b2 = i;
    while (i < e && (__ldg(group_x + grps[i]) & mhi) == 0) ++i;
    const int64_t b3 = i;
    for (; i < e; ++i) {
      const uint64_t x = __ldg(group_x + grps[i]);
      if ((x & mlo) == 0 || (x & mhi) == 0) ok = false;
    }
    rkh[r] = static_cast<int32_t>(b2 - b);
    rkl[r] = static_cast<int32_t>(b3 - b2);
    if (!ok) ++c;
  }
  warp_count_add(c, bad);
}

// Entries per slab (from the slab's first row) and per low string (from slab 0, diagonal
// included); every row must agree with both.
__global__ void k_slab_meta(const int32_t* __restrict__ rkh, const int32_t* __restrict__ rkl,
                            int64_t n, int64_t nl, int d, int64_t* kh, int64_t* kl,
                            unsigned long long* bad) {
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = r / nl, l = r - h * nl;
    if (l == 0) kh[h] = rkh[r];
    if (h == 0) kl[l] = d + rkl[r];
    if (rkh[r] != rkh[h * nl] || rkl[r] != rkl[l]) ++c;
  }
  warp_count_add(c, bad);
}

// H sources as offsets h' * nl: the sources of row (h, 0) itself.
__global__ void k_hsrc(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                       int64_t nh, int64_t nl, int d, const int64_t* __restrict__ ho,
                       uint32_t* hsrc) {
  for (int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; h < nh;
       h += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = row_ptr[h * nl] + d;
    for (int64_t k = 0; k < ho[h + 1] - ho[h]; ++k) hsrc[ho[h] + k] = cols[b + k];
  }
}

// L sources as offsets l' * nh (into the transposed vector), from row (0, l).
__global__ void k_lsrc(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                       int64_t nh, int64_t nl, int d, const int64_t* __restrict__ ho,
                       const int64_t* __restrict__ lo, uint32_t* lsrc) {
  const int64_t kh0 = ho[1] - ho[0];
  for (int64_t l = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; l < nl;
       l += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = row_ptr[l];
    for (int64_t e = 0; e < lo[l + 1] - lo[l]; ++e) {
      const int64_t lp = (d && e == 0) ? l : int64_t(cols[b + kh0 + e]);
      lsrc[lo[l] + e] = static_cast<uint32_t>(lp * nh);
    }
  }
}

// Panel-major slab index of entry k at contiguous position b.
__device__ __forceinline__ int64_t panel_index(int64_t k, int64_t b, int64_t total_k) {
  return ((b >> 5) * total_k + k) * 32 + (b & 31);
}

// Copies every H and L element into its slab and checks that its stored source is the one the
// slab position implies.
template <int NCA>
__global__ void k_prod_extract(const int64_t* __restrict__ row_ptr,
                               const uint32_t* __restrict__ cols, const double* __restrict__ vals,
                               int64_t n, int64_t nh, int64_t nl, int d,
                               const int64_t* __restrict__ ho, const int64_t* __restrict__ lo,
                               const uint32_t* __restrict__ hsrc,
                               const uint32_t* __restrict__ lsrc, double* vh, double* vl,
                               int check, unsigned long long* bad) {
  const int64_t th = ho[nh], tl = lo[nl];
  unsigned long long c = 0;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = r / nl, l = r - h * nl;
    const int64_t b = row_ptr[r];
    const int64_t h0 = ho[h], nkh = ho[h + 1] - h0, l0 = lo[l], nkl = lo[l + 1] - l0;
    if (check && row_ptr[r + 1] < b + nkh + nkl) {
      ++c;
      continue;
    }
    for (int64_t k = 0; k < nkh; ++k) {
      const int64_t p = b + d + k;
      if (check && int64_t(cols[p]) != int64_t(hsrc[h0 + k]) + l) ++c;
      const int64_t q = panel_index(h0 + k, l, th);
#pragma unroll
      for (int t = 0; t < NCA; ++t) vh[NCA * q + t] = vals[NCA * p + t];
    }
    for (int64_t e = 0; e < nkl; ++e) {
      const int64_t p = (d && e == 0) ? b : b + nkh + e;
      if (check && int64_t(cols[p]) != h * nl + int64_t(lsrc[l0 + e]) / nh) ++c;
      const int64_t q = panel_index(l0 + e, h, tl);
#pragma unroll
      for (int t = 0; t < NCA; ++t) vl[NCA * q + t] = vals[NCA * p + t];
    }
  }
  warp_count_add(c, bad);
}

__global__ void k_to_float32(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}

// FP32 copy of a slab in 64-wide panels: out[((b / 64) * total_k + k) * 64 + b % 64] =
// in[panel_index(k, b, total_k)] for b < B, zero in the padding of the last panel.
template <int NCA>
__global__ void k_float_panels64(const double* __restrict__ in, int64_t total_k, int64_t B,
                                 float* __restrict__ out) {
  const int64_t n = ((B + 63) / 64) * total_k * 64;
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < n;
       q += int64_t(gridDim.x) * blockDim.x) {
    const int64_t rest = q >> 6, pos = q & 63;   // rest = panel * total_k + k
    const int64_t p = rest / total_k, k = rest - p * total_k;
    const int64_t b = p * 64 + pos;
    const int64_t src = b < B ? panel_index(k, b, total_k) : 0;
#pragma unroll
    for (int t = 0; t < NCA; ++t)
      out[NCA * q + t] = b < B ? static_cast<float>(in[NCA * src + t]) : 0.0f;
  }
}

// out[c][r] = in[r][c] for an rows x cols matrix of elements E (32 x 32 tiles, 256 threads).
template <typename E>
__global__ void __launch_bounds__(256)
k_transpose(const E* __restrict__ in, E* __restrict__ out, int64_t rows, int64_t cols) {
  __shared__ E tile[32][33];
  const int64_t tr = (rows + 31) / 32, tc = (cols + 31) / 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int64_t t = blockIdx.x; t < tr * tc; t += gridDim.x) {
    const int64_t r0 = (t / tc) * 32, c0 = (t % tc) * 32;
    for (int i = ty; i < 32; i += 8) {
      const int64_t r = r0 + i, c = c0 + tx;
      if (r < rows && c < cols) tile[i][tx] = in[r * cols + c];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
      const int64_t c = c0 + i, r = r0 + tx;
      if (c < cols && r < rows) out[c * rows + r] = tile[tx][i];
    }
    __syncthreads();
  }
}

// One slab pass over an A x B grid: element (a, b) accumulates VS(k, b) * x[src[k] + b] over
// k in [off[a], off[a + 1]) (VS panel-major over total_k entries, src premultiplied).  Warp =
// one slab a and a 32-wide panel of b; block = 8 slabs of one panel; blocks panel-major.
//   FINAL = false: store the FP64 partial at out_part[a * B + b];
//   FINAL = true:  start from part_t[a * B + b] (+ part_m[a * B + b] when HAS_M) and store the
//                  result at out[a * B + b].
// Eight entries per step keep eight independent index -> amplitude chains in flight.
template <typename R, int NCV, int NCA, bool FINAL, bool HAS_M>
__global__ void __launch_bounds__(256)
k_slab(int64_t A, int64_t B, int64_t total_k, int64_t a_tiles, const int64_t* __restrict__ off,
       const uint32_t* __restrict__ src, const R* __restrict__ V, const R* __restrict__ x,
       const double* __restrict__ part_t, const double* __restrict__ part_m, R* __restrict__ out,
       double* __restrict__ out_part, int prefetch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t panels = (B + 31) >> 5;
  // A step's elements are one contiguous chunk of 8 x 32 entries (2 or 4 KB).  The chunk about
  // 2 KB ahead is prefetched into L2, one 128-byte line per lane, so the element loads wait on
  // L2 rather than on DRAM (measured: C3 FP64 matvec 5.9 -> 5.1 ms, C2 0.370 -> 0.324 ms; 4 KB
  // ahead was slightly slower, 8 KB no better than none).
  constexpr int kChunkLines = 8 * 32 * NCA * static_cast<int>(sizeof(R)) / 128;
  constexpr int pv = kChunkLines >= 16 ? 1 : 16 / kChunkLines;   // steps ahead
  for (int64_t blk = blockIdx.x; blk < panels * a_tiles; blk += gridDim.x) {
    const int64_t p = blk / a_tiles;
    const int64_t a = (blk - p * a_tiles) * 8 + warp;
    const int64_t b = p * 32 + lane;
    if (a >= A || b >= B) continue;
    CAcc<R, NCV, NCA> acc;
    if constexpr (FINAL) {
      acc.add_partial(part_t, a * B + b);
      if constexpr (HAS_M) acc.add_partial(part_m, a * B + b);
    }
    const int64_t k1 = __ldg(off + a + 1);
    int64_t k = __ldg(off + a);
    const R* vp = V + ((p * total_k + k) * 32 + lane) * NCA;
    for (; k + 7 < k1; k += 8) {
      // prefetch: the next step's source offsets (one 32-byte sector) into L1 ahead of use
      if (prefetch && k + 15 < k1) asm volatile("prefetch.global.L1 [%0];" ::"l"(src + k + 8));
      if (lane < kChunkLines && k + 8 * pv + 7 < k1)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(
            reinterpret_cast<const char*>(vp - lane * NCA + 8 * 32 * NCA * pv) + lane * 128));
      uint32_t si[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) si[u] = __ldg(src + k + u);
      Cx<R> m[8], xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        m[u] = ld_elem<R, NCA>(vp, 32 * u);
        xv[u] = ld_elem<R, NCV>(x, int64_t(si[u]) + b);
      }
      acc.add4(m, xv);
      acc.add4(m + 4, xv + 4);
      vp += 8 * 32 * NCA;
    }
    // remainder: one entry at a time (a predicated eight-entry step measured 5-11 % slower
    // for FP64 at 32 and 48 qubits)
    for (; k < k1; ++k) {
      acc.add(ld_elem<R, NCA>(vp, 0), ld_elem<R, NCV>(x, int64_t(__ldg(src + k)) + b));
      vp += 32 * NCA;
    }
    if constexpr (FINAL) st_elem<R, NCV>(out, a * B + b, cx_make<R>(acc.re.value(), acc.im.value()));
    else acc.store_partial(out_part, a * B + b);
  }
}

// FP32 slabs in 64-wide panels: a lane owns two adjacent positions b, b + 1, so one 16-byte
// (complex64) or 8-byte (float) load reads both amplitudes and one 8- or 16-byte load both
// elements; four entries per step.  Same sums per position as k_slab (FMA chains of four
// products into the compensated sums).  VEC: x and out allow the paired vector accesses
// (source offsets and B even, pointers aligned), else each position is read on its own.
template <typename R, int NCA>
__device__ __forceinline__ void pair_elem(const R* p, Cx<R>& e0, Cx<R>& e1) {
  if constexpr (NCA == 2) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    e0 = cx_make<R>(v.x, v.y);
    e1 = cx_make<R>(v.z, v.w);
  } else {
    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
    e0 = cx_make<R>(v.x, R(0));
    e1 = cx_make<R>(v.y, R(0));
  }
}

template <typename R, int NCV, bool VEC>
__device__ __forceinline__ void pair_vec(const R* x, int64_t i, Cx<R>& v0, Cx<R>& v1) {
  if constexpr (VEC && NCV == 2) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(x + 2 * i));
    v0 = cx_make<R>(v.x, v.y);
    v1 = cx_make<R>(v.z, v.w);
  } else if constexpr (VEC) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(x + i));
    v0 = cx_make<R>(v.x, R(0));
    v1 = cx_make<R>(v.y, R(0));
  } else {
    v0 = ld_elem<R, NCV>(x, i);
    v1 = ld_elem<R, NCV>(x, i + 1);
  }
}

template <typename R, int NCV, int NCA, bool FINAL, bool HAS_M, bool VEC>
__global__ void __launch_bounds__(256)
k_slab2(int64_t A, int64_t B, int64_t total_k, int64_t a_tiles, const int64_t* __restrict__ off,
        const uint32_t* __restrict__ src, const R* __restrict__ V, const R* __restrict__ x,
        const double* __restrict__ part_t, const double* __restrict__ part_m, R* __restrict__ out,
        double* __restrict__ out_part) {
  static_assert(sizeof(R) == 4, "two positions per lane: FP32 slabs");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t panels = (B + 63) >> 6;
  // element chunk of a step (4 x 64 entries, 1 or 2 KB) prefetched into L2 about 2 KB ahead,
  // as in k_slab (C3 FP32 matvec 3.32 -> 2.78 ms, C2 0.234 -> 0.210 ms; 1 KB ahead: 2.95 ms);
  // in the first pass only: the final pass, which also reads both FP64 partials, measured
  // slower with it (c3_small 90.5 -> 104.9 us, C3 1171 -> 1295 us)
  constexpr int kChunkLines = FINAL ? 0 : 4 * 64 * NCA * static_cast<int>(sizeof(R)) / 128;
  constexpr int pv = kChunkLines >= 16 ? 1 : kChunkLines > 0 ? 16 / kChunkLines : 1;
  for (int64_t blk = blockIdx.x; blk < panels * a_tiles; blk += gridDim.x) {
    const int64_t p = blk / a_tiles;
    const int64_t a = (blk - p * a_tiles) * 8 + warp;
    const int64_t b = p * 64 + 2 * lane;  // positions b and b + 1 (B is even)
    if (a >= A || b >= B) continue;
    CAcc<R, NCV, NCA> acc0, acc1;
    if constexpr (FINAL) {
      acc0.add_partial(part_t, a * B + b);
      acc1.add_partial(part_t, a * B + b + 1);
      if constexpr (HAS_M) {
        acc0.add_partial(part_m, a * B + b);
        acc1.add_partial(part_m, a * B + b + 1);
      }
    }
    const int64_t k1 = __ldg(off + a + 1);
    int64_t k = __ldg(off + a);
    const R* vp = V + ((p * total_k + k) * 64 + 2 * lane) * NCA;
    for (; k + 3 < k1; k += 4) {
      if (lane < kChunkLines && k + 4 * pv + 3 < k1)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(
            reinterpret_cast<const char*>(vp - 2 * lane * NCA + 4 * 64 * NCA * pv) + lane * 128));
      uint32_t si[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) si[u] = __ldg(src + k + u);
      Cx<R> m0[4], m1[4], x0[4], x1[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        pair_elem<R, NCA>(vp + 64 * NCA * u, m0[u], m1[u]);
        pair_vec<R, NCV, VEC>(x, int64_t(si[u]) + b, x0[u], x1[u]);
      }
      acc0.add4(m0, x0);
      acc1.add4(m1, x1);
      vp += 4 * 64 * NCA;
    }
    // remainder (fewer than four entries): one predicated step
    if (k < k1) {
      uint32_t si[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) si[u] = (k + u < k1) ? __ldg(src + k + u) : 0u;
      Cx<R> m0[4], m1[4], x0[4], x1[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (k + u < k1) {
          pair_elem<R, NCA>(vp + 64 * NCA * u, m0[u], m1[u]);
          pair_vec<R, NCV, VEC>(x, int64_t(si[u]) + b, x0[u], x1[u]);
        } else {
          m0[u] = m1[u] = x0[u] = x1[u] = cx_make<R>(R(0), R(0));
        }
      }
      acc0.add4(m0, x0);
      acc1.add4(m1, x1);
    }
    if constexpr (FINAL) {
      if constexpr (VEC && NCV == 2) {
        reinterpret_cast<float4*>(out)[(a * B + b) >> 1] =
            make_float4(acc0.re.value(), acc0.im.value(), acc1.re.value(), acc1.im.value());
      } else if constexpr (VEC) {
        reinterpret_cast<float2*>(out)[(a * B + b) >> 1] =
            make_float2(acc0.re.value(), acc1.re.value());
      } else {
        st_elem<R, NCV>(out, a * B + b, cx_make<R>(acc0.re.value(), acc0.im.value()));
        st_elem<R, NCV>(out, a * B + b + 1, cx_make<R>(acc1.re.value(), acc1.im.value()));
      }
    } else {
      acc0.store_partial(out_part, a * B + b);
      acc1.store_partial(out_part, a * B + b + 1);
    }
  }
}

// M pairs of every row, FP64 partial per row.  Same schedule as the CSR matvec: LPR lanes per
// row, interleaved or chunked rows.  The pairs are the row's CSR tail after its H and L entries
// (row_ptr, cols, vals: the operator's arrays; ho, lo give the H and L counts) or, COMPACT, the
// contiguous copy of the tails (row_ptr = mptr, cols = mcol, vals = mval; ho, lo unused).
template <typename R, int NCV, int NCA, int LPR, bool COMPACT>
__global__ void __launch_bounds__(256)
k_mv_mixed(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
           const R* __restrict__ vals, const R* __restrict__ v, const int64_t* __restrict__ ho,
           const int64_t* __restrict__ lo, int64_t nl, double* __restrict__ part,
           int64_t n_rows, int64_t chunk) {
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane % LPR, slot = lane / LPR;
  auto one_step = [&](int64_t rb, int64_t lim) {
    const int64_t row = rb + slot;
    CAcc<R, NCV, NCA> acc;
    if (row < lim) {
      int64_t b = __ldg(row_ptr + row);
      const int64_t e = __ldg(row_ptr + row + 1);
      if constexpr (!COMPACT) {
        const int64_t h = row / nl, l = row - h * nl;
        b += (__ldg(ho + h + 1) - __ldg(ho + h)) + (__ldg(lo + l + 1) - __ldg(lo + l));
      }
      csr_row_dot<R, NCV, NCA, LPR>(cols, vals, v, b + sub, e, acc);
    }
    acc.merge(LPR);
    if (sub == 0 && row < lim) acc.store_partial(part, row);
  };
  if (chunk <= 0) {
    const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t rb = w0 * RPW; rb < n_rows; rb += nw * RPW) one_step(rb, n_rows);
  } else {
    const int nwb = blockDim.x >> 5;
    for (int64_t c0 = int64_t(blockIdx.x) * chunk; c0 < n_rows; c0 += int64_t(gridDim.x) * chunk) {
      const int64_t lim = min(c0 + chunk, n_rows);
      for (int64_t rb = c0 + int64_t(warp) * RPW; rb < lim; rb += int64_t(nwb) * RPW)
        one_step(rb, lim);
    }
  }
}

// ---- M pairs through shared memory ----------------------------------------------------
constexpr int kTailThreads = 512;
constexpr size_t kTailSmemMax = 200 * 1024;

__device__ __forceinline__ int64_t tail_begin(const int64_t* row_ptr, const int64_t* ho,
                                              const int64_t* lo, int64_t r, int64_t nl) {
  const int64_t h = r / nl, l = r - h * nl;
  return row_ptr[r] + (ho[h + 1] - ho[h]) + (lo[l + 1] - lo[l]);
}

// Per-row tail lengths and, when bits is given, bits[h][h' / 32] |= 1 << (h' % 32) for every M
// source slab h' of slab h.
__global__ void k_tail_mark(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                            const int64_t* __restrict__ ho, const int64_t* __restrict__ lo,
                            int64_t n, int64_t nl, int64_t words, uint32_t* bits, int64_t* len) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = r / nl;
    const int64_t b = tail_begin(row_ptr, ho, lo, r, nl), e = row_ptr[r + 1];
    len[r] = e - b;
    if (bits == nullptr) continue;
    for (int64_t i = b; i < e; ++i) {
      const uint32_t hs = static_cast<uint32_t>(cols[i] / nl);
      atomicOr(bits + h * words + (hs >> 5), 1u << (hs & 31));
    }
  }
}

__global__ void k_tail_counts(const uint32_t* __restrict__ bits, int64_t nh, int64_t words,
                              int64_t* counts, unsigned* max_count) {
  for (int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; h < nh;
       h += int64_t(gridDim.x) * blockDim.x) {
    int64_t c = 0;
    for (int64_t w = 0; w < words; ++w) c += __popc(bits[h * words + w]);
    counts[h] = c;
    atomicMax(max_count, static_cast<unsigned>(c));
  }
}

__global__ void k_tail_slist(const uint32_t* __restrict__ bits, int64_t nh, int64_t words,
                             const int64_t* __restrict__ soff, uint32_t* slist) {
  for (int64_t h = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; h < nh;
       h += int64_t(gridDim.x) * blockDim.x) {
    int64_t k = soff[h];
    for (int64_t w = 0; w < words; ++w) {
      uint32_t m = bits[h * words + w];
      while (m) {
        const int bit = __ffs(m) - 1;
        m &= m - 1;
        slist[k++] = static_cast<uint32_t>(w * 32 + bit);
      }
    }
  }
}

// Compact tail copy: the element, and the source row (mcol, when given) or the shared-memory
// index (slot of h' among h's sources; with_index).
template <int NCA>
__global__ void k_tail_fill(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
                            const double* __restrict__ vals, const int64_t* __restrict__ ho,
                            const int64_t* __restrict__ lo, const uint32_t* __restrict__ bits,
                            int64_t n, int64_t nl, int64_t words,
                            const int64_t* __restrict__ mptr, uint16_t* msidx, double* mval,
                            int with_index, uint32_t* mcol) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = r / nl;
    const int64_t b = tail_begin(row_ptr, ho, lo, r, nl), e = row_ptr[r + 1];
    int64_t j = mptr[r];
    for (int64_t i = b; i < e; ++i, ++j) {
#pragma unroll
      for (int t = 0; t < NCA; ++t) mval[NCA * j + t] = vals[NCA * i + t];
      if (mcol != nullptr) mcol[j] = cols[i];
      if (!with_index) continue;
      const int64_t c = cols[i];
      const int64_t hs = c / nl;
      int64_t slot = 0;
      for (int64_t w = 0; w < (hs >> 5); ++w) slot += __popc(bits[h * words + w]);
      slot += __popc(bits[h * words + (hs >> 5)] & ((1u << (hs & 31)) - 1u));
      msidx[j] = static_cast<uint16_t>(slot * nl + (c - hs * nl));
    }
  }
}

template <typename R, int NC>
__device__ __forceinline__ Cx<R> sm_elem(const R* p, int64_t i) {
  if constexpr (NC == 2) {
    if constexpr (sizeof(R) == 8) {
      const double2 d = reinterpret_cast<const double2*>(p)[i];
      return cx_make<R>(d.x, d.y);
    } else {
      const float2 d = reinterpret_cast<const float2*>(p)[i];
      return cx_make<R>(d.x, d.y);
    }
  } else {
    return cx_make<R>(p[i], R(0));
  }
}

// M pairs of the rows of slab h (split in `chunks` row ranges, one block each): the block
// copies all M source slabs of h into shared memory once, then LPR lanes per row stream the
// compact tail (element + 16-bit shared-memory index) and gather from shared memory.
template <typename R, int NCV, int NCA, int LPR>
__global__ void __launch_bounds__(kTailThreads)
k_tail_smem(const int64_t* __restrict__ mptr, const uint16_t* __restrict__ msidx,
            const R* __restrict__ mval, const R* __restrict__ v, const int64_t* __restrict__ soff,
            const uint32_t* __restrict__ slist, int64_t nh, int64_t nl, int64_t chunks,
            double* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char tail_raw[];
  using E = std::conditional_t<NCV == 2, std::conditional_t<sizeof(R) == 8, double2, float2>, R>;
  E* vse = reinterpret_cast<E*>(tail_raw);
  const R* vs = reinterpret_cast<const R*>(tail_raw);
  const E* ve = reinterpret_cast<const E*>(v);
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane % LPR, slot = lane / LPR;
  const int nwarps = blockDim.x >> 5;
  const int64_t per_chunk = (nl + chunks - 1) / chunks;
  for (int64_t blk = blockIdx.x; blk < nh * chunks; blk += gridDim.x) {
    const int64_t h = blk / chunks, c = blk - h * chunks;
    const int64_t s0 = __ldg(soff + h), s1 = __ldg(soff + h + 1);
    __syncthreads();  // the previous block's slabs are consumed
    for (int64_t s = s0; s < s1; ++s) {
      const int64_t base = int64_t(__ldg(slist + s)) * nl;
      E* dst = vse + (s - s0) * nl;
      for (int64_t i = threadIdx.x; i < nl; i += blockDim.x) dst[i] = ve[base + i];
    }
    __syncthreads();
    const int64_t l0 = c * per_chunk, l1 = min(nl, l0 + per_chunk);
    for (int64_t lb = l0 + int64_t(warp) * RPW; lb < l1; lb += int64_t(nwarps) * RPW) {
      const int64_t l = lb + slot;
      CAcc<R, NCV, NCA> acc;
      if (l < l1) {
        const int64_t r = h * nl + l;
        const int64_t e = __ldg(mptr + r + 1);
        int64_t i = __ldg(mptr + r) + sub;
        for (; i + 3 * LPR < e; i += 4 * LPR) {
          uint16_t si[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) si[u] = __ldg(msidx + i + u * LPR);
          Cx<R> a[4], x[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            a[u] = ld_elem<R, NCA>(mval, i + u * LPR);
            x[u] = sm_elem<R, NCV>(vs, si[u]);
          }
          acc.add4(a, x);
        }
        for (; i < e; i += LPR) acc.add(ld_elem<R, NCA>(mval, i), sm_elem<R, NCV>(vs, __ldg(msidx + i)));
      }
      acc.merge(LPR);
      if (sub == 0 && l < l1) acc.store_partial(part, h * nl + l);
    }
  }
}

template <typename R, int NCV, int NCA>
void allow_tail_smem() {
  const int bytes = static_cast<int>(kTailSmemMax);
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 1>, attr, bytes));
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 2>, attr, bytes));
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 4>, attr, bytes));
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 8>, attr, bytes));
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 16>, attr, bytes));
  SQD_CUDA(cudaFuncSetAttribute(k_tail_smem<R, NCV, NCA, 32>, attr, bytes));
}

void allow_tail_smem_all() {
  allow_tail_smem<double, 1, 1>();
  allow_tail_smem<double, 2, 1>();
  allow_tail_smem<double, 2, 2>();
  allow_tail_smem<float, 1, 1>();
  allow_tail_smem<float, 2, 1>();
  allow_tail_smem<float, 2, 2>();
}

unsigned capped_grid(int64_t blocks) {
  return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, INT_MAX)));
}

// wide: FP32 slabs in 64-wide panels (k_slab2); vec: x and out allow its paired accesses.
template <typename R, int NCV, int NCA, bool FINAL, bool HAS_M>
void launch_slab(int64_t A, int64_t B, int64_t total_k, const int64_t* off, const uint32_t* src,
                 const R* V, const R* x, const double* part_t, const double* part_m, R* out,
                 double* out_part, cudaStream_t st, bool wide = false, bool vec = false) {
  if (A == 0 || B == 0) return;
  if constexpr (sizeof(R) == 4) {
    if (wide) {
      const int64_t a_tiles = (A + 7) / 8, panels = (B + 63) / 64;
      if (vec)
        k_slab2<R, NCV, NCA, FINAL, HAS_M, true><<<capped_grid(a_tiles * panels), 256, 0, st>>>(
            A, B, total_k, a_tiles, off, src, V, x, part_t, part_m, out, out_part);
      else
        k_slab2<R, NCV, NCA, FINAL, HAS_M, false><<<capped_grid(a_tiles * panels), 256, 0, st>>>(
            A, B, total_k, a_tiles, off, src, V, x, part_t, part_m, out, out_part);
      SQD_CHECK_LAUNCH();
      return;
    }
  }
  const int64_t a_tiles = (A + 7) / 8, panels = (B + 31) / 32;
  // With at most two waves of warps (64 per SM) too few warps hide the latency of each step's
  // source-offset load, which the gathers wait on, so it is prefetched one step ahead (C2:
  // 8,192 warps, FP64 matvec 0.348 -> 0.320 ms); on larger grids the other warps hide it and
  // the extra requests cost 2-4 % (C3, 524,288 warps).
  const int prefetch = A * panels <= 2 * 64 * int64_t(num_sms()) ? 1 : 0;
  k_slab<R, NCV, NCA, FINAL, HAS_M><<<capped_grid(a_tiles * panels), 256, 0, st>>>(
      A, B, total_k, a_tiles, off, src, V, x, part_t, part_m, out, out_part, prefetch);
  SQD_CHECK_LAUNCH();
}

template <typename E>
void launch_transpose(const void* in, void* out, int64_t rows, int64_t cols, cudaStream_t st) {
  const unsigned G = capped_grid(
      std::min<int64_t>(((rows + 31) / 32) * ((cols + 31) / 32), int64_t(num_sms()) * 32));
  k_transpose<E><<<G, 256, 0, st>>>(static_cast<const E*>(in), static_cast<E*>(out), rows, cols);
  SQD_CHECK_LAUNCH();
}

unsigned mixed_grid(int64_t rows, int lpr) {
  const int64_t warps = (rows * lpr + 31) / 32;
  const int64_t blocks = (warps + 7) / 8;
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min(blocks, cap)));
}

void extract(sqd_op_s* op, cudaStream_t st, int check, unsigned long long* bad) {
  ProductLayout& L = op->prod;
  const int64_t n = L.nh * L.nl;
  const unsigned G = grid_for(n, 256, 16384);
  if (op->value_complex)
    k_prod_extract<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, n, L.nh,
                                         L.nl, op->has_diag_group, L.ho.ptr, L.lo.ptr,
                                         L.hsrc.ptr, L.lsrc.ptr, L.vh.ptr, L.vl.ptr, check, bad);
  else
    k_prod_extract<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, n, L.nh,
                                         L.nl, op->has_diag_group, L.ho.ptr, L.lo.ptr,
                                         L.hsrc.ptr, L.lsrc.ptr, L.vh.ptr, L.vl.ptr, check, bad);
  SQD_CHECK_LAUNCH();
}

void to_float(const DevBuf<double>& in, DevBuf<float>& out, cudaStream_t st) {
  out.alloc(in.count, st);
  k_to_float32<<<grid_for(static_cast<int64_t>(in.count), 256, 16384), 256, 0, st>>>(
      in.ptr, out.ptr, static_cast<int64_t>(in.count));
  SQD_CHECK_LAUNCH();
}

// FP32 copies of both slab sets: 64-wide panels when wide32, else the FP64 layout.
void slabs_to_float(sqd_op_s* op, cudaStream_t st) {
  ProductLayout& L = op->prod;
  if (!L.wide32) {
    to_float(L.vh, L.vh32, st);
    to_float(L.vl, L.vl32, st);
    return;
  }
  const int nca = op->value_complex ? 2 : 1;
  auto conv = [&](const DevBuf<double>& in, int64_t total_k, int64_t B, DevBuf<float>& out) {
    const int64_t n = ((B + 63) / 64) * total_k * 64;
    out.alloc(static_cast<size_t>(std::max<int64_t>(n, 1)) * nca, st);
    const unsigned G = grid_for(std::max<int64_t>(n, 1), 256, 16384);
    if (nca == 2)
      k_float_panels64<2><<<G, 256, 0, st>>>(in.ptr, total_k, B, out.ptr);
    else
      k_float_panels64<1><<<G, 256, 0, st>>>(in.ptr, total_k, B, out.ptr);
    SQD_CHECK_LAUNCH();
  };
  conv(L.vh, L.th, L.nl, L.vh32);
  conv(L.vl, L.tl, L.nh, L.vl32);
}

// A row tail read in place is a short segment of the row's long pair list (C3-like subspaces:
// ~11 M pairs among ~160), so its element and source loads use few bytes of the sectors they
// fetch.  Tails up to this many pairs per row on average are also copied contiguously.
constexpr int64_t kCompactTailMax = 32;

// Shared-memory form of the M pairs, when every slab's M source slabs fit in kTailSmemMax
// together (at 8 bytes per amplitude) and 16-bit indices reach them.  Fills len (per-row tail
// lengths) either way; returns whether the form was built.
bool build_tail_smem(sqd_op_s* op, DevBuf<int64_t>& len, cudaStream_t st) {
  ProductLayout& L = op->prod;
  const int64_t nh = L.nh, nl = L.nl, n = nh * nl;
  const unsigned G = grid_for(n, 256, 16384);
  if (nh > 65536) {
    k_tail_mark<<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, L.ho.ptr, L.lo.ptr, n, nl, 0,
                                   nullptr, len.ptr);
    SQD_CHECK_LAUNCH();
    return false;
  }
  const int64_t words = (nh + 31) / 32;
  DevBuf<uint32_t> bits;
  bits.alloc(static_cast<size_t>(nh * words), st);
  SQD_CUDA(cudaMemsetAsync(bits.ptr, 0, sizeof(uint32_t) * nh * words, st));
  DevBuf<int64_t> counts;
  counts.alloc(nh, st);
  DevBuf<unsigned> maxc;
  maxc.alloc(1, st);
  SQD_CUDA(cudaMemsetAsync(maxc.ptr, 0, sizeof(unsigned), st));
  k_tail_mark<<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, L.ho.ptr, L.lo.ptr, n, nl, words,
                                 bits.ptr, len.ptr);
  SQD_CHECK_LAUNCH();
  k_tail_counts<<<grid_for(nh, 256, 4096), 256, 0, st>>>(bits.ptr, nh, words, counts.ptr,
                                                          maxc.ptr);
  SQD_CHECK_LAUNCH();
  unsigned slots = 0;
  copy_to_host(&slots, maxc.ptr, 1, st);
  const int64_t span = static_cast<int64_t>(slots) * nl;
  if (slots == 0 || span > 65535 || static_cast<size_t>(span) * 8 > kTailSmemMax) return false;
  L.soff.alloc(nh + 1, st);
  exclusive_scan_i64(counts.ptr, L.soff.ptr, nh, true, st);
  int64_t total = 0;
  copy_to_host(&total, L.soff.ptr + nh, 1, st);
  L.slist.alloc(std::max<int64_t>(total, 1), st);
  k_tail_slist<<<grid_for(nh, 256, 4096), 256, 0, st>>>(bits.ptr, nh, words, L.soff.ptr,
                                                         L.slist.ptr);
  SQD_CHECK_LAUNCH();
  L.mptr.alloc(n + 1, st);
  exclusive_scan_i64(len.ptr, L.mptr.ptr, n, true, st);
  const int nca = op->value_complex ? 2 : 1;
  L.msidx.alloc(static_cast<size_t>(L.pairs_m), st);
  L.mval.alloc(static_cast<size_t>(L.pairs_m) * nca, st);
  if (nca == 2)
    k_tail_fill<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, bits.ptr, n, nl, words, L.mptr.ptr, L.msidx.ptr,
                                      L.mval.ptr, 1, nullptr);
  else
    k_tail_fill<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, bits.ptr, n, nl, words, L.mptr.ptr, L.msidx.ptr,
                                      L.mval.ptr, 1, nullptr);
  SQD_CHECK_LAUNCH();
  allow_tail_smem_all();
  SQD_CUDA(cudaStreamSynchronize(st));
  L.tail_slots = static_cast<int>(slots);
  return true;
}

// Compact forms of the M pairs: the shared-memory form where it applies, and the short-tail
// form (source rows beside the same contiguous elements, for the CSR tail kernel) when the
// tails average at most kCompactTailMax pairs per row.  Longer tails are read in place.
void build_tail(sqd_op_s* op, cudaStream_t st) {
  ProductLayout& L = op->prod;
  const int64_t n = L.nh * L.nl;
  if (L.pairs_m <= 0) return;
  DevBuf<int64_t> len;
  len.alloc(n, st);
  const bool smem = build_tail_smem(op, len, st);
  if (L.pairs_m > kCompactTailMax * n) return;
  const int nca = op->value_complex ? 2 : 1;
  // The copy is optional: without device memory for it the tails are read in place.
  try {
    if (!smem) {
      L.mptr.alloc(n + 1, st);
      L.mval.alloc(static_cast<size_t>(L.pairs_m) * nca, st);
    }
    L.mcol.alloc(static_cast<size_t>(L.pairs_m), st);
  } catch (const Error& e) {
    if (e.status != SQD_ERR_MEMORY) throw;
    (void)cudaGetLastError();  // the failed pool allocation
    if (!smem) {
      L.mptr = DevBuf<int64_t>();
      L.mval = DevBuf<double>();
    }
    L.mcol = DevBuf<uint32_t>();
    return;
  }
  if (!smem) exclusive_scan_i64(len.ptr, L.mptr.ptr, n, true, st);
  const unsigned G = grid_for(n, 256, 16384);
  if (nca == 2)
    k_tail_fill<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, nullptr, n, L.nl, 0, L.mptr.ptr, nullptr,
                                      L.mval.ptr, 0, L.mcol.ptr);
  else
    k_tail_fill<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, nullptr, n, L.nl, 0, L.mptr.ptr, nullptr,
                                      L.mval.ptr, 0, L.mcol.ptr);
  SQD_CHECK_LAUNCH();
  SQD_CUDA(cudaStreamSynchronize(st));
  L.compact_tail = 1;
}

// Tail elements again after a coefficient update (sources unchanged).
void refill_tail(sqd_op_s* op, cudaStream_t st) {
  ProductLayout& L = op->prod;
  if (L.mval.ptr == nullptr) return;
  const int64_t n = L.nh * L.nl;
  const unsigned G = grid_for(n, 256, 16384);
  if (op->value_complex)
    k_tail_fill<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, nullptr, n, L.nl, 0, L.mptr.ptr, nullptr,
                                      L.mval.ptr, 0, nullptr);
  else
    k_tail_fill<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->values.ptr, L.ho.ptr,
                                      L.lo.ptr, nullptr, n, L.nl, 0, L.mptr.ptr, nullptr,
                                      L.mval.ptr, 0, nullptr);
  SQD_CHECK_LAUNCH();
}

template <typename R, int NCV, int NCA>
bool launch_tail_smem(sqd_op_s* op, int prec, const R* vin, cudaStream_t st) {
  ProductLayout& L = op->prod;
  if (!L.tail_slots) return false;
  const size_t bytes = static_cast<size_t>(L.tail_slots) * L.nl * NCV * sizeof(R);
  if (bytes > kTailSmemMax) return false;
  const R* mv;
  if constexpr (sizeof(R) == 8) mv = L.mval.ptr;
  else mv = L.mval32.ptr;
  if (mv == nullptr) return false;
  const int64_t chunks =
      std::max<int64_t>(1, std::min<int64_t>(8, (4 * int64_t(num_sms()) + L.nh - 1) / L.nh));
  dispatch_lpr(op->lanes_per_row[prec], [&](auto lpr_t) {
    constexpr int LPR = decltype(lpr_t)::value;
    k_tail_smem<R, NCV, NCA, LPR><<<capped_grid(L.nh * chunks), kTailThreads, bytes, st>>>(
        L.mptr.ptr, L.msidx.ptr, mv, vin, L.soff.ptr, L.slist.ptr, L.nh, L.nl, chunks, L.t.ptr);
    SQD_CHECK_LAUNCH();
  });
  return true;
}

// ---- connectivity of a product subspace -------------------------------------------------
// The (row, group) sweep tests every group against every row.  In a product subspace a group
// acting on one half connects a row iff the row's string of that half has a partner, so the
// partners are searched once per string of the half, and a two-half group connects (h, l) iff
// both halves have partners.  The pairs are then assembled per row in the sweep's order:
// diagonal, H groups, L groups, M groups, each class in ascending group index (= ascending x:
// for M groups, ascending high part, then low part).

__device__ __forceinline__ int64_t sorted_find(const uint64_t* __restrict__ a, int64_t n,
                                               uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1; else hi = mid;
  }
  return (lo < n && __ldg(a + lo) == key) ? lo : -1;
}

// Partners of every string s of one half under the masks xs[k]: entries (k, partner) with
// strs[partner] == strs[s] ^ xs[k], in k order.  One warp per string, lanes over k, ballots
// keep the order.  COUNT: count[s]; FILL: writes at off[s].
template <bool FILL>
__global__ void k_half_partners(const uint64_t* __restrict__ strs, int64_t nstr,
                                const uint64_t* __restrict__ xs, int64_t nx,
                                const int64_t* __restrict__ off, int64_t* count,
                                uint32_t* out_k, uint32_t* out_p) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = w0; s < nstr; s += nw) {
    const uint64_t base = __ldg(strs + s);
    int64_t pos = FILL ? off[s] : 0;
    for (int64_t k0 = 0; k0 < nx; k0 += 32) {
      const int64_t k = k0 + lane;
      int64_t found = -1;
      if (k < nx) found = sorted_find(strs, nstr, base ^ __ldg(xs + k));
      const unsigned b = __ballot_sync(kFullMask, found >= 0);
      if (FILL && found >= 0) {
        const int64_t idx = pos + __popc(b & lt);
        out_k[idx] = static_cast<uint32_t>(k);
        out_p[idx] = static_cast<uint32_t>(found);
      }
      pos += __popc(b);
    }
    if (!FILL && lane == 0) count[s] = pos;
  }
}

struct ProdConnect {
  int64_t nh, nl;
  int d;
  const int64_t *hoff, *loff, *aoff, *boff;          // H, L, M-high, M-low lists per string
  const uint32_t *hk, *hp, *lk, *lp, *ak, *ap, *bk, *bp;
  const int32_t *gh, *gl;                            // group index of H / L list entry k
  const int32_t* table;                              // [na * nb] M group or -1 (dense form)
  int64_t na, nb;
  const uint64_t *xa, *xb, *xm;                      // sparse form: M masks, sorted
  const int32_t* gm;
  int64_t nm;
};

__device__ __forceinline__ int32_t m_group(const ProdConnect& c, uint32_t a, uint32_t b) {
  if (c.table) return __ldg(c.table + int64_t(a) * c.nb + b);
  const int64_t i = sorted_find(c.xm, c.nm, __ldg(c.xa + a) | __ldg(c.xb + b));
  return i >= 0 ? __ldg(c.gm + i) : -1;
}

template <bool FILL>
__global__ void k_prod_rows(ProdConnect c, int64_t* counts, const int64_t* __restrict__ row_ptr,
                            uint32_t* cols, uint32_t* grps) {
  const int64_t n = c.nh * c.nl;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int64_t h = r / c.nl, l = r - h * c.nl;
    const int64_t h0 = c.hoff[h], h1 = c.hoff[h + 1], l0 = c.loff[l], l1 = c.loff[l + 1];
    const int64_t a0 = c.aoff[h], a1 = c.aoff[h + 1], b0 = c.boff[l], b1 = c.boff[l + 1];
    if (!FILL) {
      int64_t m = 0;
      for (int64_t i = a0; i < a1; ++i)
        for (int64_t j = b0; j < b1; ++j) m += m_group(c, c.ak[i], c.bk[j]) >= 0;
      counts[r] = c.d + (h1 - h0) + (l1 - l0) + m;
      continue;
    }
    int64_t p = row_ptr[r];
    if (c.d) {
      cols[p] = static_cast<uint32_t>(r);
      grps[p] = 0;
      ++p;
    }
    for (int64_t i = h0; i < h1; ++i, ++p) {
      cols[p] = static_cast<uint32_t>(int64_t(c.hp[i]) * c.nl + l);
      grps[p] = static_cast<uint32_t>(c.gh[c.hk[i]]);
    }
    for (int64_t i = l0; i < l1; ++i, ++p) {
      cols[p] = static_cast<uint32_t>(h * c.nl + c.lp[i]);
      grps[p] = static_cast<uint32_t>(c.gl[c.lk[i]]);
    }
    for (int64_t i = a0; i < a1; ++i) {
      const int64_t src_h = int64_t(c.ap[i]) * c.nl;
      for (int64_t j = b0; j < b1; ++j) {
        const int32_t g = m_group(c, c.ak[i], c.bk[j]);
        if (g < 0) continue;
        cols[p] = static_cast<uint32_t>(src_h + c.bp[j]);
        grps[p] = static_cast<uint32_t>(g);
        ++p;
      }
    }
  }
}

__global__ void k_half_strings(const uint64_t* __restrict__ s, int64_t count, int64_t stride,
                               uint64_t mask, uint64_t* out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = s[i * stride] & mask;
}

// Device copy of a host vector.
template <typename T>
void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t st) {
  d.alloc(std::max<size_t>(h.size(), 1), st);
  if (!h.empty())
    SQD_CUDA(cudaMemcpyAsync(d.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

// Partner lists of one half: counts, offsets, (k, partner) entries.
struct HalfLists {
  DevBuf<int64_t> off;
  DevBuf<uint32_t> k, p;
};

void half_lists(const DevBuf<uint64_t>& strs, int64_t nstr, const DevBuf<uint64_t>& xs,
                int64_t nx, HalfLists& out, cudaStream_t st) {
  DevBuf<int64_t> cnt;
  cnt.alloc(std::max<int64_t>(nstr, 1), st);
  const unsigned G = grid_for(nstr * 32, 256, 8192);
  k_half_partners<false><<<G, 256, 0, st>>>(strs.ptr, nstr, xs.ptr, nx, nullptr, cnt.ptr,
                                             nullptr, nullptr);
  SQD_CHECK_LAUNCH();
  out.off.alloc(nstr + 1, st);
  exclusive_scan_i64(cnt.ptr, out.off.ptr, nstr, true, st);
  int64_t total = 0;
  copy_to_host(&total, out.off.ptr + nstr, 1, st);
  out.k.alloc(std::max<int64_t>(total, 1), st);
  out.p.alloc(std::max<int64_t>(total, 1), st);
  k_half_partners<true><<<G, 256, 0, st>>>(strs.ptr, nstr, xs.ptr, nx, out.off.ptr, nullptr,
                                            out.k.ptr, out.p.ptr);
  SQD_CHECK_LAUNCH();
}

}  // namespace

bool op_product_detect(sqd_op_s* op, cudaStream_t st, int64_t* nh_out, int64_t* nl_out) {
  sqd_space_s* sp = op->s;
  const int64_t n = sp->n_unique;
  *nh_out = *nl_out = 0;
  if (n == 0 || sp->states_size != n || sp->num_qubits < 2) return false;
  const uint64_t mlo = half_mask_low(sp->num_qubits), mhi = sp->fill_state & ~mlo;
  DevBuf<unsigned long long> cnt;
  cnt.alloc(2, st);
  SQD_CUDA(cudaMemsetAsync(cnt.ptr, 0, 2 * sizeof(unsigned long long), st));
  const unsigned G = grid_for(n, 256, 4096);
  k_count_slabs<<<G, 256, 0, st>>>(sp->states.ptr, n, mhi, cnt.ptr);
  SQD_CHECK_LAUNCH();
  unsigned long long nh = 0;
  copy_to_host(&nh, cnt.ptr, 1, st);
  if (nh == 0 || n % static_cast<int64_t>(nh) != 0) return false;
  const int64_t nl = n / static_cast<int64_t>(nh);
  k_check_product<<<G, 256, 0, st>>>(sp->states.ptr, n, nl, mlo, mhi, cnt.ptr + 1);
  SQD_CHECK_LAUNCH();
  unsigned long long bad = 0;
  copy_to_host(&bad, cnt.ptr + 1, 1, st);
  if (bad) return false;
  *nh_out = static_cast<int64_t>(nh);
  *nl_out = nl;
  return true;
}

bool op_connect_product(sqd_op_s* op, cudaStream_t st) {
  int64_t nh = 0, nl = 0;
  if (!op_product_detect(op, st, &nh, &nl)) return false;
  sqd_space_s* sp = op->s;
  const int64_t n = nh * nl;
  if (n > (int64_t(1) << 32)) return false;
  const uint64_t mlo = half_mask_low(sp->num_qubits), mhi = sp->fill_state & ~mlo;
  // Group lists per class from the preprocessed groups (class order, ascending group index).
  std::vector<GroupPre> gp(static_cast<size_t>(op->n_gpre));
  copy_to_host(gp.data(), op->gpre.ptr, gp.size(), st);
  const int64_t n0 = op->n_gpre_cls[0], n1 = op->n_gpre_cls[1];
  std::vector<uint64_t> xh, xl, xm;
  std::vector<int32_t> gh, gl, gm;
  for (int64_t i = 0; i < op->n_gpre; ++i) {
    const GroupPre& g = gp[static_cast<size_t>(i)];
    if (i < n0) { xh.push_back(g.x); gh.push_back(g.group); }
    else if (i < n0 + n1) { xl.push_back(g.x); gl.push_back(g.group); }
    else { xm.push_back(g.x); gm.push_back(g.group); }
  }
  // Distinct high and low parts of the M masks (ascending), and the M group lookup.
  std::vector<uint64_t> xa, xb;
  for (uint64_t x : xm) { xa.push_back(x & mhi); xb.push_back(x & mlo); }
  std::sort(xa.begin(), xa.end());
  xa.erase(std::unique(xa.begin(), xa.end()), xa.end());
  std::sort(xb.begin(), xb.end());
  xb.erase(std::unique(xb.begin(), xb.end()), xb.end());
  const bool dense = !xm.empty() && double(xa.size()) * double(xb.size()) <= double(1 << 24);
  std::vector<int32_t> table;
  if (dense) {
    table.assign(xa.size() * xb.size(), -1);
    for (size_t i = 0; i < xm.size(); ++i) {
      const size_t a = std::lower_bound(xa.begin(), xa.end(), xm[i] & mhi) - xa.begin();
      const size_t b = std::lower_bound(xb.begin(), xb.end(), xm[i] & mlo) - xb.begin();
      table[a * xb.size() + b] = gm[i];
    }
  }
  DevBuf<uint64_t> hstr, lstr, dxh, dxl, dxa, dxb, dxm;
  DevBuf<int32_t> dgh, dgl, dgm, dtable;
  hstr.alloc(nh, st);
  lstr.alloc(nl, st);
  k_half_strings<<<grid_for(nh, 256, 4096), 256, 0, st>>>(sp->states.ptr, nh, nl, mhi, hstr.ptr);
  k_half_strings<<<grid_for(nl, 256, 4096), 256, 0, st>>>(sp->states.ptr, nl, 1, mlo, lstr.ptr);
  SQD_CHECK_LAUNCH();
  upload(dxh, xh, st);
  upload(dxl, xl, st);
  upload(dxa, xa, st);
  upload(dxb, xb, st);
  upload(dxm, xm, st);
  upload(dgh, gh, st);
  upload(dgl, gl, st);
  upload(dgm, gm, st);
  if (dense) upload(dtable, table, st);
  HalfLists H, Lh, A, Bl;
  half_lists(hstr, nh, dxh, static_cast<int64_t>(xh.size()), H, st);
  half_lists(lstr, nl, dxl, static_cast<int64_t>(xl.size()), Lh, st);
  half_lists(hstr, nh, dxa, static_cast<int64_t>(xa.size()), A, st);
  half_lists(lstr, nl, dxb, static_cast<int64_t>(xb.size()), Bl, st);
  ProdConnect c{};
  c.nh = nh;
  c.nl = nl;
  c.d = op->has_diag_group;
  c.hoff = H.off.ptr;
  c.loff = Lh.off.ptr;
  c.aoff = A.off.ptr;
  c.boff = Bl.off.ptr;
  c.hk = H.k.ptr;
  c.hp = H.p.ptr;
  c.lk = Lh.k.ptr;
  c.lp = Lh.p.ptr;
  c.ak = A.k.ptr;
  c.ap = A.p.ptr;
  c.bk = Bl.k.ptr;
  c.bp = Bl.p.ptr;
  c.gh = dgh.ptr;
  c.gl = dgl.ptr;
  c.table = dense ? dtable.ptr : nullptr;
  c.na = static_cast<int64_t>(xa.size());
  c.nb = static_cast<int64_t>(xb.size());
  c.xa = dxa.ptr;
  c.xb = dxb.ptr;
  c.xm = dxm.ptr;
  c.gm = dgm.ptr;
  c.nm = static_cast<int64_t>(xm.size());
  DevBuf<int64_t> counts;
  counts.alloc(n, st);
  const unsigned G = grid_for(n, 256, 16384);
  k_prod_rows<false><<<G, 256, 0, st>>>(c, counts.ptr, nullptr, nullptr, nullptr);
  SQD_CHECK_LAUNCH();
  op->row_ptr.alloc(n + 1, st);
  exclusive_scan_i64(counts.ptr, op->row_ptr.ptr, n, true, st);
  copy_to_host(&op->nnz, op->row_ptr.ptr + n, 1, st);
  counts.release();
  op->cols.alloc(op->nnz > 0 ? op->nnz : 1, st);
  op->grps.alloc(op->nnz > 0 ? op->nnz : 1, st);
  k_prod_rows<true><<<G, 256, 0, st>>>(c, nullptr, op->row_ptr.ptr, op->cols.ptr, op->grps.ptr);
  SQD_CHECK_LAUNCH();
  SQD_CUDA(cudaStreamSynchronize(st));  // the host vectors above go out of scope
  op->product_built = 1;
  return true;
}

void op_product_build(sqd_op_s* op, cudaStream_t st) {
  if (op->prod.built) return;
  SQD_REQUIRE(op->x_cache == 1 && op->z_cache == 2,
              "the product layout needs cache_strategy (1, 2)");
  SQD_REQUIRE(op->nnz == 0 || op->grps.ptr != nullptr,
              "the operator released its group indices; create a new operator");
  int64_t nh = 0, nl = 0;
  if (!op_product_detect(op, st, &nh, &nl))
    throw Error(SQD_ERR_UNSUPPORTED,
                "the subspace is not a product of high-half and low-half strings without "
                "fill-in slots; the product layout does not apply");
  sqd_space_s* sp = op->s;
  const uint64_t mlo = half_mask_low(sp->num_qubits), mhi = sp->fill_state & ~mlo;
  const int d = op->has_diag_group;
  const int64_t n = nh * nl;
  ProductLayout L;
  L.nh = nh;
  L.nl = nl;
  L.wide32 = (nh % 2 == 0 && nl % 2 == 0) ? 1 : 0;
  DevBuf<unsigned long long> bad;
  bad.alloc(1, st);
  SQD_CUDA(cudaMemsetAsync(bad.ptr, 0, sizeof(unsigned long long), st));
  {
    DevBuf<int32_t> rkh, rkl;
    rkh.alloc(n, st);
    rkl.alloc(n, st);
    DevBuf<int64_t> kh, kl;
    kh.alloc(nh, st);
    kl.alloc(nl, st);
    const unsigned G = grid_for(n, 256, 16384);
    k_row_kinds<<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, op->p->group_x.ptr, n, d, mlo,
                                   mhi, rkh.ptr, rkl.ptr, bad.ptr);
    SQD_CHECK_LAUNCH();
    k_slab_meta<<<G, 256, 0, st>>>(rkh.ptr, rkl.ptr, n, nl, d, kh.ptr, kl.ptr, bad.ptr);
    SQD_CHECK_LAUNCH();
    unsigned long long hbad = 0;
    copy_to_host(&hbad, bad.ptr, 1, st);
    if (hbad)
      throw Error(SQD_ERR_DEVICE, "stored pairs do not follow the product structure (" +
                                      std::to_string(hbad) + " rows)");
    L.ho.alloc(nh + 1, st);
    L.lo.alloc(nl + 1, st);
    exclusive_scan_i64(kh.ptr, L.ho.ptr, nh, true, st);
    exclusive_scan_i64(kl.ptr, L.lo.ptr, nl, true, st);
  }
  int64_t th = 0, tl = 0;
  copy_to_host(&th, L.ho.ptr + nh, 1, st);
  copy_to_host(&tl, L.lo.ptr + nl, 1, st);
  L.th = th;
  L.tl = tl;
  L.hsrc.alloc(std::max<int64_t>(th, 1), st);
  L.lsrc.alloc(std::max<int64_t>(tl, 1), st);
  k_hsrc<<<grid_for(nh, 256, 4096), 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, nh, nl, d,
                                                   L.ho.ptr, L.hsrc.ptr);
  SQD_CHECK_LAUNCH();
  k_lsrc<<<grid_for(nl, 256, 4096), 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, nh, nl, d,
                                                   L.ho.ptr, L.lo.ptr, L.lsrc.ptr);
  SQD_CHECK_LAUNCH();
  L.pairs_h = th * nl;
  L.pairs_l = tl * nh;
  L.pairs_m = op->nnz - L.pairs_h - L.pairs_l;
  const int nca = op->value_complex ? 2 : 1;
  // Panel-major slabs, each panel padded to 32 positions (the padding is never read).
  const size_t nvh = static_cast<size_t>(std::max<int64_t>(th * ((nl + 31) / 32) * 32, 1)) * nca;
  const size_t nvl = static_cast<size_t>(std::max<int64_t>(tl * ((nh + 31) / 32) * 32, 1)) * nca;
  L.vh.alloc(nvh, st);
  L.vl.alloc(nvl, st);
  SQD_CUDA(cudaMemsetAsync(L.vh.ptr, 0, nvh * sizeof(double), st));
  SQD_CUDA(cudaMemsetAsync(L.vl.ptr, 0, nvl * sizeof(double), st));
  L.vt.alloc(static_cast<size_t>(n) * 2, st);
  L.tt.alloc(static_cast<size_t>(n) * 2, st);
  L.t.alloc(L.pairs_m > 0 ? static_cast<size_t>(n) * 2 : 1, st);
  op->prod = std::move(L);
  extract(op, st, 1, bad.ptr);
  unsigned long long hbad = 0;
  copy_to_host(&hbad, bad.ptr, 1, st);
  if (hbad) {
    op->prod = ProductLayout();
    throw Error(SQD_ERR_DEVICE, "stored sources do not follow the product structure (" +
                                    std::to_string(hbad) + " pairs)");
  }
  build_tail(op, st);
  if (op->values32.ptr && op->layout[1] != SQD_LAYOUT_CSR) {
    slabs_to_float(op, st);
    if (op->prod.mval.ptr) to_float(op->prod.mval, op->prod.mval32, st);
  }
  op->prod.built = 1;
  SQD_CUDA(cudaStreamSynchronize(st));
}

// Elements again after a coefficient update (sources unchanged).
void op_product_values(sqd_op_s* op, cudaStream_t st) {
  if (!op->prod.built) return;
  extract(op, st, 0, nullptr);
  refill_tail(op, st);
  if (op->prod.vh32.ptr) {
    slabs_to_float(op, st);
    if (op->prod.mval.ptr) to_float(op->prod.mval, op->prod.mval32, st);
  }
}

void op_product_values32(sqd_op_s* op, cudaStream_t st) {
  if (!op->prod.built || op->prod.vh32.ptr) return;
  slabs_to_float(op, st);
  if (op->prod.mval.ptr) to_float(op->prod.mval, op->prod.mval32, st);
}

void op_product_matvec(sqd_op_s* op, const void* v, void* out, int dtype, cudaStream_t st) {
  ProductLayout& L = op->prod;
  const bool dbl = dtype_is_double(dtype);
  SQD_REQUIRE(dbl || L.vh32.ptr != nullptr, "FP32 product-layout elements were not prepared");
  const int64_t nh = L.nh, nl = L.nl, n = nh * nl;
  const int prec = dbl ? 0 : 1;
  dispatch_vec(dtype, op->value_complex, [&](auto rt, auto ncv_t, auto nca_t) {
    using R = typename decltype(rt)::type;
    constexpr int NCV = decltype(ncv_t)::value;
    constexpr int NCA = decltype(nca_t)::value;
    using E = std::conditional_t<NCV == 2, std::conditional_t<sizeof(R) == 8, double2, float2>, R>;
    using ED = std::conditional_t<NCV == 2, double2, double>;
    const R* vin = static_cast<const R*>(v);
    R* vout = static_cast<R*>(out);
    const R* VH;
    const R* VL;
    const R* VC;
    if constexpr (sizeof(R) == 8) {
      VH = L.vh.ptr;
      VL = L.vl.ptr;
      VC = op->values.ptr;
    } else {
      VH = L.vh32.ptr;
      VL = L.vl32.ptr;
      VC = op->values32.ptr;
    }
    R* vt = reinterpret_cast<R*>(L.vt.ptr);
    // FP32 slabs in 64-wide panels (both halves even): paired accesses to the library's own
    // buffers always, to v and Hv when their addresses allow
    const bool wide = sizeof(R) == 4 && L.wide32;
    const uintptr_t pair_bytes = 2 * NCV * sizeof(R);
    const bool vec_io = reinterpret_cast<uintptr_t>(vin) % pair_bytes == 0 &&
                        reinterpret_cast<uintptr_t>(vout) % pair_bytes == 0;
    // 1. vT[l][h] = v[h][l]
    launch_transpose<E>(vin, vt, nh, nl, st);
    // 2. L part: t2[l][h]
    launch_slab<R, NCV, NCA, false, false>(nl, nh, L.tl, L.lo.ptr, L.lsrc.ptr, VL, vt, nullptr,
                                           nullptr, nullptr, L.tt.ptr, st, wide, true);
    // 3. t2 back in row order, into the vT buffer
    launch_transpose<ED>(L.tt.ptr, L.vt.ptr, nl, nh, st);
    // 4. M part: t3[r]
    if (L.pairs_m > 0) {
      if (op->layout[prec] == SQD_LAYOUT_PRODUCT_CSR ||
          !launch_tail_smem<R, NCV, NCA>(op, prec, vin, st)) {
        const R* MV = nullptr;  // the short-tail copy's elements, when it exists
        if (L.compact_tail) {
          if constexpr (sizeof(R) == 8) MV = L.mval.ptr;
          else MV = L.mval32.ptr;
        }
        dispatch_lpr(op->lanes_per_row[prec], [&](auto lpr_t) {
          constexpr int LPR = decltype(lpr_t)::value;
          if (MV != nullptr)
            k_mv_mixed<R, NCV, NCA, LPR, true><<<mixed_grid(n, LPR), 256, 0, st>>>(
                L.mptr.ptr, L.mcol.ptr, MV, vin, nullptr, nullptr, nl, L.t.ptr, n,
                op->chunk_rows[prec]);
          else
            k_mv_mixed<R, NCV, NCA, LPR, false><<<mixed_grid(n, LPR), 256, 0, st>>>(
                op->row_ptr.ptr, op->cols.ptr, VC, vin, L.ho.ptr, L.lo.ptr, nl, L.t.ptr, n,
                op->chunk_rows[prec]);
          SQD_CHECK_LAUNCH();
        });
      }
      // 5. H part plus both partials
      launch_slab<R, NCV, NCA, true, true>(nh, nl, L.th, L.ho.ptr, L.hsrc.ptr, VH, vin, L.vt.ptr,
                                           L.t.ptr, vout, nullptr, st, wide, vec_io);
    } else {
      launch_slab<R, NCV, NCA, true, false>(nh, nl, L.th, L.ho.ptr, L.hsrc.ptr, VH, vin,
                                            L.vt.ptr, nullptr, vout, nullptr, st, wide, vec_io);
    }
  });
}

}  // namespace sqd

using namespace sqd;

extern "C" int sqd_op_set_layout(sqd_op_t op, int precision, int layout, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    SQD_REQUIRE(layout == SQD_LAYOUT_CSR || layout == SQD_LAYOUT_PRODUCT ||
                    layout == SQD_LAYOUT_PRODUCT_CSR,
                "unknown layout");
    if (layout != SQD_LAYOUT_CSR) {
      cudaStream_t st = as_stream(stream);
      op_product_build(op, st);
      if (precision == 1) {
        const int prev = op->layout[1];
        op->layout[1] = layout;
        try {
          op_ensure_values32(op, st);
          SQD_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
          op->layout[1] = prev;
          throw;
        }
      }
    }
    op->layout[precision] = layout;
    ++op->schedule_version;
  });
}

extern "C" int sqd_op_get_layout(sqd_op_t op, int precision, int* layout) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && layout != nullptr, "NULL argument");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    *layout = op->layout[precision];
  });
}

extern "C" int sqd_op_product_info(sqd_op_t op, void* stream, int64_t* n_high, int64_t* n_low,
                                   int64_t* pairs_high, int64_t* pairs_low,
                                   int64_t* pairs_mixed) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    int64_t nh = 0, nl = 0, ph = -1, pl = -1, pm = -1;
    if (op->prod.built) {
      nh = op->prod.nh;
      nl = op->prod.nl;
      ph = op->prod.pairs_h;
      pl = op->prod.pairs_l;
      pm = op->prod.pairs_m;
    } else if (op->x_cache == 1 && op->z_cache == 2) {
      op_product_detect(op, as_stream(stream), &nh, &nl);
    }
    if (n_high) *n_high = nh;
    if (n_low) *n_low = nl;
    if (pairs_high) *pairs_high = ph;
    if (pairs_low) *pairs_low = pl;
    if (pairs_mixed) *pairs_mixed = pm;
  });
}
