// Hv on the subspace: (Hv)_i = sum_j C^(j)_i v[src_j(i)]  (sqd.py:65-68, apply_h* :643-743).
//
// Row-oriented gather, no atomics.  A warp serves 32 / LPR rows at a time, LPR lanes per row
// stride over the row's stored pairs (coalesced loads of the pair arrays), gather the source
// amplitudes with 128-bit (c128) / 64-bit (c64) loads, and reduce with warp shuffles.
//
//  * k_mv_csr  (cache_strategy (1, 2)): matrix elements cached per stored pair.
//  * k_mv_xc   (cache_strategy (1, 0) / (1, 1)): sources cached, composed diagonal recomputed
//               from popcount(s & z) per pair (the reference's default, apply_h_x_cached).
//               The diagonal group (x = 0, K_0 terms, the largest group) is split over the LPR
//               lanes of the row.
//  * sweep APPLY (cache_strategy (0, *)): sources searched inside the matvec (apply_h).
// FP32 vectors accumulate with error-free transformations (TwoProduct via fma, TwoSum), i.e.
// the compensated dot product of Ogita, Rump and Oishi (SIAM J. Sci. Comput. 26, 2005), so the
// FP32 result is as accurate as if accumulated in twice the working precision.
#include "internal.cuh"
#include "dispatch.cuh"
#include "accum.cuh"
#include "sweep.cuh"

namespace sqd {
namespace {

template <typename R, int NCV, int NCA, int LPR>
__global__ void __launch_bounds__(256)
k_mv_csr(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
         const R* __restrict__ vals, const R* __restrict__ v, R* __restrict__ out,
         int64_t n_rows, int64_t chunk) {
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane % LPR, slot = lane / LPR;
  auto one_step = [&](int64_t rb, int64_t lim) {
    const int64_t row = rb + slot;
    CAcc<R, NCV, NCA> acc;
    if (row < lim) {
      const int64_t b = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
      csr_row_dot<R, NCV, NCA, LPR>(cols, vals, v, b + sub, e, acc);
    }
    acc.merge(LPR);
    if (sub == 0 && row < lim) st_elem<R, NCV>(out, row, cx_make<R>(acc.re.value(), acc.im.value()));
  };
  if (chunk <= 0) {
    // Interleaved: consecutive warps of the grid take consecutive row groups.
    const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t rb = w0 * RPW; rb < n_rows; rb += nw * RPW) one_step(rb, n_rows);
  } else {
    // Chunked: a block owns `chunk` consecutive rows at a time, so the source amplitudes its
    // rows share (same high-sector block, neighbouring rows) are reused from its L1.
    const int nwb = blockDim.x >> 5;
    for (int64_t c0 = int64_t(blockIdx.x) * chunk; c0 < n_rows; c0 += int64_t(gridDim.x) * chunk) {
      const int64_t lim = min(c0 + chunk, n_rows);
      for (int64_t rb = c0 + int64_t(warp) * RPW; rb < lim; rb += int64_t(nwb) * RPW)
        one_step(rb, lim);
    }
  }
}

template <typename R, int NCV, int NCA, int LPR>
__global__ void __launch_bounds__(256)
k_mv_xc(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
        const uint32_t* __restrict__ grps, const uint64_t* __restrict__ states, int64_t n_unique,
        uint64_t fill_state, int has_diag, const int64_t* __restrict__ gs,
        const int32_t* __restrict__ ge, const uint64_t* __restrict__ tz,
        const double* __restrict__ tc, const R* __restrict__ v, R* __restrict__ out,
        int64_t n_rows) {
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31;
  const int sub = lane % LPR, slot = lane / LPR;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t rb = w0 * RPW; rb < n_rows; rb += nw * RPW) {
    const int64_t row = rb + slot;
    const bool live = row < n_rows;
    CAcc<R, NCV, NCA> acc;
    int64_t b = 0, e = 0;
    uint64_t s = 0;
    if (live) {
      b = __ldg(row_ptr + row);
      e = __ldg(row_ptr + row + 1);
      s = row < n_unique ? __ldg(states + row) : fill_state;
    }
    // Diagonal group, lanes of the row split its terms.
    const bool diag = live && has_diag && e > b;
    double dr = 0.0, di = 0.0;
    if (diag) {
      const int64_t tb = __ldg(gs);
      const int32_t K = __ldg(ge);
      for (int32_t t = sub; t < K; t += LPR) {
        const bool neg = parity64(s & __ldg(tz + tb + t));
        const double cr = __ldg(tc + 2 * (tb + t));
        dr += neg ? -cr : cr;
        if constexpr (NCA == 2) {
          const double ci = __ldg(tc + 2 * (tb + t) + 1);
          di += neg ? -ci : ci;
        }
      }
    }
    for (int o = LPR >> 1; o > 0; o >>= 1) {
      dr += __shfl_xor_sync(kFullMask, dr, o);
      if constexpr (NCA == 2) di += __shfl_xor_sync(kFullMask, di, o);
    }
    if (diag && sub == 0) {
      const Cx<R> x = ld_elem<R, NCV>(v, __ldg(cols + b));
      acc.add(cx_make<R>(R(dr), R(di)), x);
    }
    if (live) {
      for (int64_t i = b + (diag ? 1 : 0) + sub; i < e; i += LPR) {
        const uint32_t c = __ldg(cols + i);
        const uint32_t j = __ldg(grps + i);
        const int64_t tb = __ldg(gs + j);
        const int32_t K = __ldg(ge + j);
        double er = 0.0, ei = 0.0;
        for (int32_t t = 0; t < K; ++t) {
          const bool neg = parity64(s & __ldg(tz + tb + t));
          const double cr = __ldg(tc + 2 * (tb + t));
          er += neg ? -cr : cr;
          if constexpr (NCA == 2) {
            const double ci = __ldg(tc + 2 * (tb + t) + 1);
            ei += neg ? -ci : ci;
          }
        }
        const Cx<R> x = ld_elem<R, NCV>(v, c);
        acc.add(cx_make<R>(R(er), R(ei)), x);
      }
    }
    acc.merge(LPR);
    if (sub == 0 && live) st_elem<R, NCV>(out, row, cx_make<R>(acc.re.value(), acc.im.value()));
  }
}

template <typename R, int NCV>
__global__ void k_zero_tail(R* out, int64_t from, int64_t to) {
  for (int64_t i = from + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < to;
       i += int64_t(gridDim.x) * blockDim.x)
    st_elem<R, NCV>(out, i, cx_make<R>(0, 0));
}

// Fill-in slots under the uncached matvec: only the last slot connects (to the first fill-in
// slot, through the diagonal group evaluated at the all-ones state).
template <typename R, int NCV, int NCA>
__global__ void k_fill_tail(const R* v, R* out, int64_t n_unique, int64_t size,
                            uint64_t fill_state, const int64_t* gs, const int32_t* ge,
                            const uint64_t* tz, const double* tc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int64_t b = gs[0];
  const int32_t K = ge[0];
  double dr = 0.0, di = 0.0;
  for (int32_t t = 0; t < K; ++t) {
    const bool neg = parity64(fill_state & tz[b + t]);
    dr += neg ? -tc[2 * (b + t)] : tc[2 * (b + t)];
    if constexpr (NCA == 2) di += neg ? -tc[2 * (b + t) + 1] : tc[2 * (b + t) + 1];
  }
  const Cx<R> x = ld_elem_rw<R, NCV>(v, n_unique);
  Cx<R> o;
  o.re = R(dr) * x.re - R(di) * x.im;
  o.im = R(dr) * x.im + R(di) * x.re;
  st_elem<R, NCV>(out, size - 1, o);
}

unsigned mv_grid(int64_t rows, int lpr) {
  const int64_t warps = (rows * lpr + 31) / 32;
  const int64_t blocks = (warps + 7) / 8;
  const int64_t cap = static_cast<int64_t>(num_sms()) * 16;
  return static_cast<unsigned>(std::max<int64_t>(1, std::min(blocks, cap)));
}

}  // namespace

void op_matvec(sqd_op_s* op, const void* v, void* out, int dtype, cudaStream_t st) {
  sqd_paulis_s* p = op->p;
  sqd_space_s* sp = op->s;
  const int64_t size = sp->states_size;
  if (op->x_cache == 1 && op->z_cache == 2 && !dtype_is_double(dtype)) op_ensure_values32(op, st);
  if (op->x_cache == 1 && op->z_cache == 2 && op->prod.built &&
      op->layout[dtype_is_double(dtype) ? 0 : 1] != SQD_LAYOUT_CSR) {
    op_product_matvec(op, v, out, dtype, st);
    return;
  }
  dispatch_vec(dtype, op->value_complex, [&](auto rt, auto ncv_t, auto nca_t) {
    using R = typename decltype(rt)::type;
    constexpr int NCV = decltype(ncv_t)::value;
    constexpr int NCA = decltype(nca_t)::value;
    const R* vin = static_cast<const R*>(v);
    R* vout = static_cast<R*>(out);
    if (op->x_cache == 1) {
      dispatch_lpr(op->lanes_per_row[sizeof(R) == 8 ? 0 : 1], [&](auto lpr_t) {
        constexpr int LPR = decltype(lpr_t)::value;
        const unsigned G = mv_grid(size, LPR);
        if (op->z_cache == 2) {
          const R* vals;
          if constexpr (sizeof(R) == 8) vals = op->values.ptr;
          else vals = op->values32.ptr;
          const int64_t chunk = op->chunk_rows[sizeof(R) == 8 ? 0 : 1];
          k_mv_csr<R, NCV, NCA, LPR><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, vals,
                                                        vin, vout, size, chunk);
        } else {
          k_mv_xc<R, NCV, NCA, LPR><<<G, 256, 0, st>>>(
              op->row_ptr.ptr, op->cols.ptr, op->grps.ptr, sp->states.ptr, sp->n_unique,
              sp->fill_state, op->has_diag_group, p->group_start.ptr, p->group_eff.ptr,
              p->term_z.ptr, p->term_c.ptr, vin, vout, size);
        }
        SQD_CHECK_LAUNCH();
      });
      return;
    }
    // Uncached: sources searched in the matvec.
    SweepParams P{};
    P.states = sp->states.ptr;
    P.n_unique = sp->n_unique;
    P.gpre = op->gpre.ptr;
    P.n_gpre = op->n_gpre;
    P.hkeys = sp->hkeys.ptr;
    P.hvals = sp->hvals.ptr;
    P.hmask = sp->hmask;
    P.lookup = op->lookup == SQD_LOOKUP_BSEARCH ? SQD_LOOKUP_BSEARCH : SQD_LOOKUP_HASH;
    P.nsec = sp->num_sectors;
    P.m0 = sp->sector_mask[0];
    P.m1 = sp->sector_mask[1];
    P.sh0 = sp->num_sectors > 0 ? __builtin_ctzll(sp->sector_mask[0]) : 0;
    P.sh1 = sp->num_sectors > 1 ? __builtin_ctzll(sp->sector_mask[1]) : 0;
    P.ex0 = sp->num_sectors > 0 && __builtin_popcountll(sp->sector_mask[0]) <= kBitmapLog2;
    P.ex1 = sp->num_sectors > 1 && __builtin_popcountll(sp->sector_mask[1]) <= kBitmapLog2;
    P.bitmap = sp->bitmap.ptr;
    P.group_start = p->group_start.ptr;
    P.group_eff = p->group_eff.ptr;
    P.term_z = p->term_z.ptr;
    P.term_c = p->term_c.ptr;
    P.vin = v;
    P.vout = out;
    P.has_diag = op->has_diag_group;
    const size_t dyn = P.bitmap ? (static_cast<size_t>(sp->num_sectors) << kBitmapLog2) / 8 : 0;
    auto kern = k_sweep<SWEEP_APPLY, R, NCV, NCA>;
    SQD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dyn)));
    if (sp->n_unique > 0) {
      kern<<<grid_for(sp->n_unique, SW_TILE), SW_THREADS, dyn, st>>>(P);
      SQD_CHECK_LAUNCH();
    }
    if (size > sp->n_unique) {
      k_zero_tail<R, NCV><<<grid_for(size - sp->n_unique, 256, 1024), 256, 0, st>>>(
          vout, sp->n_unique, size);
      SQD_CHECK_LAUNCH();
      if (op->has_diag_group) {
        k_fill_tail<R, NCV, NCA><<<1, 32, 0, st>>>(vin, vout, sp->n_unique, size, sp->fill_state,
                                                  p->group_start.ptr, p->group_eff.ptr,
                                                  p->term_z.ptr, p->term_c.ptr);
        SQD_CHECK_LAUNCH();
      }
    }
  });
}

}  // namespace sqd

using namespace sqd;

extern "C" int sqd_matvec(sqd_op_t op, const void* v, void* out, int dtype, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && v != nullptr && out != nullptr, "NULL argument");
    SQD_REQUIRE(v != out, "sqd_matvec cannot work in place");
    op_matvec(op, v, out, dtype, as_stream(stream));
  });
}
