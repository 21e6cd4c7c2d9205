// The projected operator: connectivity cache, matrix elements, diagonals, vinit, CSR export and
// the Hellmann-Feynman per-term reduction.
//
// Connectivity (cache_strategy x = 1) is the sparse form of the reference's xsources cache
// (run_sqd, sqd.py:343-351): instead of a dense J x N int32 array with -1 for missing sources,
// only the pairs whose source exists are stored, row by row, in group order:
//   row_ptr[states_size + 1], cols[nnz] (source index), grps[nnz] (group index).
// Matrix elements (z = 2) are the composed diagonals C^(j)_i of the stored pairs
// (sqd.py:95-98), summed term by term in the reference's order (get_diagonal, sqd.py:603-628).
#include "internal.cuh"
#include "dispatch.cuh"
#include "sweep.cuh"

namespace sqd {
namespace {

// Groups that can connect, in three classes so that every row's stored pairs come in class
// order.  With the qubits split in a low half (mask mlo) and a high half (mhi):
//   class 0 (H): x acts on the high half only;
//   class 1 (L): x acts on the low half only;
//   class 2 (M): x acts on both halves.
// In an alpha x beta product subspace all rows with the same high string have the same class-0
// sources and all rows with the same low string the same class-1 sources, which the product
// layout of the matvec (product.cu) builds on.  Inside a class the group order is kept.
__global__ void k_gpre_flags(const uint64_t* group_x, int64_t J, int nsec, uint64_t m0,
                             uint64_t m1, uint64_t mlo, uint64_t mhi, int64_t* flags0,
                             int64_t* flags1, int64_t* flags2) {
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < J;
       j += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t x = group_x[j];
    bool ok = x != 0;
    if (nsec > 0) ok = ok && ((__popcll(x & m0) & 1) == 0);
    if (nsec > 1) ok = ok && ((__popcll(x & m1) & 1) == 0);
    const int cls = (x & mlo) == 0 ? 0 : (x & mhi) == 0 ? 1 : 2;
    flags0[j] = (ok && cls == 0) ? 1 : 0;
    flags1[j] = (ok && cls == 1) ? 1 : 0;
    flags2[j] = (ok && cls == 2) ? 1 : 0;
  }
}

__global__ void k_gpre_fill(const uint64_t* group_x, int64_t J, const int64_t* flags0,
                            const int64_t* pos0, const int64_t* flags1, const int64_t* pos1,
                            const int64_t* flags2, const int64_t* pos2, uint64_t m0, uint64_t m1,
                            GroupPre* out) {
  const int64_t n0 = pos0[J], n1 = pos1[J];
  for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < J;
       j += int64_t(gridDim.x) * blockDim.x) {
    if (!flags0[j] && !flags1[j] && !flags2[j]) continue;
    const uint64_t x = group_x[j];
    GroupPre g;
    g.x = x;
    g.group = static_cast<int32_t>(j);
    g.cx = (__popcll(x & m0) & 0xff) | ((__popcll(x & m1) & 0xff) << 8);
    out[flags0[j] ? pos0[j] : flags1[j] ? n0 + pos1[j] : n0 + n1 + pos2[j]] = g;
  }
}

__global__ void k_fill_counts(int64_t n_unique, int64_t size, int has_diag, int64_t* counts) {
  for (int64_t r = n_unique + blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < size;
       r += int64_t(gridDim.x) * blockDim.x)
    counts[r] = (has_diag && r == size - 1) ? 1 : 0;
}

__global__ void k_add_const(int64_t* counts, int64_t n, int64_t c) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x)
    counts[r] += c;
}

// Diagonal-group entries: real row r -> (r, 0); last fill-in slot -> (n_unique, 0).
__global__ void k_diag_entries(const int64_t* row_ptr, int64_t n_unique, int64_t size,
                               uint32_t* cols, uint32_t* grps) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n_unique;
       r += int64_t(gridDim.x) * blockDim.x) {
    cols[row_ptr[r]] = static_cast<uint32_t>(r);
    grps[row_ptr[r]] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && size > n_unique) {
    cols[row_ptr[size - 1]] = static_cast<uint32_t>(n_unique);
    grps[row_ptr[size - 1]] = 0;
  }
}

// Composed diagonal of group j at state s, term by term in the reference's order.
template <int NCA>
__device__ __forceinline__ Cx<double> diag_seq(const int64_t* gs, const int32_t* ge,
                                               const uint64_t* tz, const double* tc, int64_t j,
                                               uint64_t s) {
  const int64_t b = gs[j];
  const int32_t k = ge[j];
  double dr = 0.0, di = 0.0;
  for (int32_t t = 0; t < k; ++t) {
    const bool neg = parity64(s & __ldg(tz + b + t));
    const double cr = __ldg(tc + 2 * (b + t));
    dr = dr + (neg ? -cr : cr);
    if constexpr (NCA == 2) {
      const double ci = __ldg(tc + 2 * (b + t) + 1);
      di = di + (neg ? -ci : ci);
    }
  }
  return cx_make<double>(dr, di);
}

// One warp per row, lanes over the row's stored pairs: matrix element per pair.
// out_mode 0: values as NCA doubles per pair; 1: complex128 per pair (CSR export).
template <int NCA>
__global__ void k_values(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ grps,
                         const uint64_t* __restrict__ states, int64_t n_unique,
                         uint64_t fill_state, int64_t size, const int64_t* gs, const int32_t* ge,
                         const uint64_t* tz, const double* tc, double* out, int out_complex) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = w0; r < size; r += nw) {
    const uint64_t s = r < n_unique ? __ldg(states + r) : fill_state;
    const int64_t b = row_ptr[r], e = row_ptr[r + 1];
    for (int64_t i = b + lane; i < e; i += 32) {
      const Cx<double> d = diag_seq<NCA>(gs, ge, tz, tc, grps[i], s);
      if (out_complex) {
        out[2 * i] = d.re;
        out[2 * i + 1] = d.im;
      } else if constexpr (NCA == 2) {
        out[2 * i] = d.re;
        out[2 * i + 1] = d.im;
      } else {
        out[i] = d.re;
      }
    }
  }
}

__global__ void k_to_float(const double* in, float* out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}

template <int NCA>
__global__ void k_diagonal(const uint64_t* states, int64_t n_unique, uint64_t fill_state,
                           int64_t size, const int64_t* gs, const int32_t* ge,
                           const uint64_t* tz, const double* tc, int64_t j, double* out,
                           int out_complex) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < size;
       r += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t s = r < n_unique ? states[r] : fill_state;
    const Cx<double> d = diag_seq<NCA>(gs, ge, tz, tc, j, s);
    if (out_complex) {
      out[2 * r] = d.re;
      out[2 * r + 1] = d.im;
    } else {
      out[r] = d.re;
    }
  }
}

// Order-preserving map of a double onto unsigned integers; -0.0 maps like +0.0 (the two compare
// equal, and jnp.argmin at sqd.py:413 keeps the first of equal values).
__device__ __forceinline__ unsigned long long order_key(double v) {
  if (v == 0.0) v = 0.0;
  unsigned long long b = __double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Argmin of Re diag_0 over real rows; ties -> smallest index (jnp.argmin).
__global__ void k_argmin_partial(const uint64_t* states, int64_t n_unique, const int64_t* gs,
                                 const int32_t* ge, const uint64_t* tz, const double* tc,
                                 unsigned long long* best_key, long long* best_idx) {
  unsigned long long bk = ~0ull;
  long long bi = 0x7fffffffffffffffll;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n_unique;
       r += int64_t(gridDim.x) * blockDim.x) {
    const Cx<double> d = diag_seq<1>(gs, ge, tz, tc, 0, states[r]);
    const unsigned long long k = order_key(d.re);
    if (k < bk || (k == bk && r < bi)) {
      bk = k;
      bi = r;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ok = __shfl_xor_sync(kFullMask, bk, o);
    const long long oi = __shfl_xor_sync(kFullMask, bi, o);
    if (ok < bk || (ok == bk && oi < bi)) {
      bk = ok;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    const int64_t w = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    best_key[w] = bk;
    best_idx[w] = bi;
  }
}

__global__ void k_argmin_final(const unsigned long long* keys, const long long* idx, int64_t n,
                               long long* out) {
  unsigned long long bk = ~0ull;
  long long bi = 0x7fffffffffffffffll;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    if (keys[i] < bk || (keys[i] == bk && idx[i] < bi)) {
      bk = keys[i];
      bi = idx[i];
    }
  }
  __shared__ unsigned long long sk[32];
  __shared__ long long si[32];
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ok = __shfl_xor_sync(kFullMask, bk, o);
    const long long oi = __shfl_xor_sync(kFullMask, bi, o);
    if (ok < bk || (ok == bk && oi < bi)) {
      bk = ok;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    sk[threadIdx.x >> 5] = bk;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sk[w] < bk || (sk[w] == bk && si[w] < bi)) {
        bk = sk[w];
        bi = si[w];
      }
    *out = bi;
  }
}

__global__ void k_cols_to_i32(const uint32_t* cols, int32_t* out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = static_cast<int32_t>(cols[i]);
}

// ---------------------------------------------------------------------------------------------
// Hellmann-Feynman per-term reduction  g_t = Re sum_i conj(u_i) ph_t (-1)^{|s_i & z_t|} v_src.
// ---------------------------------------------------------------------------------------------
constexpr int GR_TILE = 1024;

// Diagonal group (x = 0, src = i): per block, w_i = conj(u_i) v_i for a tile of rows in shared
// memory, then one block-wide reduction per term and one atomicAdd per (block, term).
template <int NCV>
__global__ void k_grad_diag(const uint64_t* states, int64_t n_unique, const int64_t* gs,
                            const int32_t* ge, const uint64_t* tz, const double* tc,
                            const double* u, const double* v, double* g) {
  __shared__ uint64_t s_st[GR_TILE];
  __shared__ double s_wr[GR_TILE], s_wi[GR_TILE];
  __shared__ double red[32];
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * GR_TILE;
  for (int k = threadIdx.x; k < GR_TILE; k += blockDim.x) {
    const int64_t r = r0 + k;
    double wr = 0.0, wi = 0.0;
    uint64_t s = 0;
    if (r < n_unique) {
      s = states[r];
      const Cx<double> a = ld_elem<double, NCV>(u, r), b = ld_elem<double, NCV>(v, r);
      wr = a.re * b.re + a.im * b.im;
      wi = a.re * b.im - a.im * b.re;
    }
    s_st[k] = s;
    s_wr[k] = wr;
    s_wi[k] = wi;
  }
  __syncthreads();
  const int64_t b = gs[0];
  const int32_t K = ge[0];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // x = 0: the phase is 1 and Re((-1)^{|s & z|} w) = (-1)^{|s & z|} Re w.
  for (int32_t t = 0; t < K; ++t) {
    const uint64_t z = tz[b + t];
    double ar = 0.0;
    for (int k = threadIdx.x; k < GR_TILE; k += blockDim.x)
      ar += parity64(s_st[k] & z) ? -s_wr[k] : s_wr[k];
    ar = warp_sum(ar);
    if (lane == 0) red[warp] = ar;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sr = 0.0;
      for (int w = 0; w < nwarp; ++w) sr += red[w];
      atomicAdd(g + b + t, sr);
    }
    __syncthreads();
  }
}

// Off-diagonal stored pairs: per pair, loop over the group's terms and atomically add.
template <int NCV>
__global__ void k_grad_offdiag(const int64_t* row_ptr, const uint32_t* cols,
                               const uint32_t* grps, const uint64_t* states, int64_t n_unique,
                               int has_diag, const int64_t* gs, const int32_t* ge,
                               const uint64_t* gx, const uint64_t* tz, const double* u,
                               const double* v, double* g) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = w0; r < n_unique; r += nw) {
    const uint64_t s = states[r];
    const Cx<double> a = ld_elem<double, NCV>(u, r);
    const int64_t b = row_ptr[r] + has_diag, e = row_ptr[r + 1];
    for (int64_t i = b + lane; i < e; i += 32) {
      const int64_t j = grps[i];
      const Cx<double> x = ld_elem<double, NCV>(v, cols[i]);
      // w = conj(u_r) v_src
      const double wr = a.re * x.re + a.im * x.im;
      const double wi = a.re * x.im - a.im * x.re;
      const uint64_t xm = gx[j];
      const int64_t tb = gs[j];
      const int32_t K = ge[j];
      for (int32_t t = 0; t < K; ++t) {
        const uint64_t z = tz[tb + t];
        const int ph = __popcll(xm & z) & 3;
        // Re((-i)^ph * w)
        double val;
        switch (ph) {
          case 0: val = wr; break;
          case 1: val = wi; break;
          case 2: val = -wr; break;
          default: val = -wi; break;
        }
        if (parity64(s & z)) val = -val;
        atomicAdd(g + tb + t, val);
      }
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------------
void op_connect_sweep(sqd_op_s* op, cudaStream_t st);
void op_values_and_lanes(sqd_op_s* op, cudaStream_t st);

void op_build(sqd_op_s* op, cudaStream_t st) {
  sqd_paulis_s* p = op->p;
  sqd_space_s* sp = op->s;
  const int64_t J = p->num_groups;
  uint64_t x0 = 1;
  copy_to_host(&x0, p->group_x.ptr, 1, st);
  op->has_diag_group = (x0 == 0) ? 1 : 0;
  op->value_complex = p->is_complex;
  op->status.alloc(1, st);
  SQD_CUDA(cudaMemsetAsync(op->status.ptr, 0, sizeof(int), st));

  // Groups that can connect.
  {
    DevBuf<int64_t> flags[3], pos[3];
    for (int c = 0; c < 3; ++c) {
      flags[c].alloc(J, st);
      pos[c].alloc(J + 1, st);
    }
    const uint64_t mlo = half_mask_low(sp->num_qubits), mhi = sp->fill_state & ~mlo;
    const unsigned G = grid_for(J, 256, 4096);
    k_gpre_flags<<<G, 256, 0, st>>>(p->group_x.ptr, J, sp->num_sectors, sp->sector_mask[0],
                                   sp->sector_mask[1], mlo, mhi, flags[0].ptr, flags[1].ptr,
                                   flags[2].ptr);
    SQD_CHECK_LAUNCH();
    int64_t n_cls[3] = {0, 0, 0};
    for (int c = 0; c < 3; ++c) {
      exclusive_scan_i64(flags[c].ptr, pos[c].ptr, J, true, st);
      copy_to_host(&n_cls[c], pos[c].ptr + J, 1, st);
    }
    op->n_gpre = n_cls[0] + n_cls[1] + n_cls[2];
    for (int c = 0; c < 3; ++c) op->n_gpre_cls[c] = n_cls[c];
    op->gpre.alloc(op->n_gpre > 0 ? op->n_gpre : 1, st);
    k_gpre_fill<<<G, 256, 0, st>>>(p->group_x.ptr, J, flags[0].ptr, pos[0].ptr, flags[1].ptr,
                                  pos[1].ptr, flags[2].ptr, pos[2].ptr, sp->sector_mask[0],
                                  sp->sector_mask[1], op->gpre.ptr);
    SQD_CHECK_LAUNCH();
  }
  if (op->x_cache == 0) return;

  bool connected = false;
  if (op->lookup == SQD_LOOKUP_AUTO || op->lookup == SQD_LOOKUP_PRODUCT) {
    connected = op_connect_product(op, st);
    if (!connected && op->lookup == SQD_LOOKUP_PRODUCT)
      throw Error(SQD_ERR_UNSUPPORTED,
                  "SQD_LOOKUP_PRODUCT needs a product of high-half and low-half strings without "
                  "fill-in slots");
  }
  if (!connected) op_connect_sweep(op, st);
  op_values_and_lanes(op, st);
}

// Connectivity by the (row, group) sweep: any subspace, fill-in slots included.
void op_connect_sweep(sqd_op_s* op, cudaStream_t st) {
  sqd_space_s* sp = op->s;
  const int64_t size = sp->states_size;
  const int64_t nu = sp->n_unique;
  SweepParams P{};
  P.states = sp->states.ptr;
  P.n_unique = nu;
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
  const size_t dyn = P.bitmap ? (static_cast<size_t>(sp->num_sectors) << kBitmapLog2) / 8 : 0;
  const unsigned tiles = grid_for(nu, SW_TILE);

  DevBuf<int64_t> counts;
  counts.alloc(size, st);
  P.counts = counts.ptr;
  {
    auto kern = k_sweep<SWEEP_COUNT, double, 1, 1>;
    SQD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dyn)));
    kern<<<tiles, SW_THREADS, dyn, st>>>(P);
    SQD_CHECK_LAUNCH();
  }
  if (op->has_diag_group)
    k_add_const<<<grid_for(nu, 256, 8192), 256, 0, st>>>(counts.ptr, nu, 1);
  if (size > nu)
    k_fill_counts<<<grid_for(size - nu, 256, 1024), 256, 0, st>>>(nu, size, op->has_diag_group,
                                                                  counts.ptr);
  SQD_CHECK_LAUNCH();
  op->row_ptr.alloc(size + 1, st);
  exclusive_scan_i64(counts.ptr, op->row_ptr.ptr, size, true, st);
  copy_to_host(&op->nnz, op->row_ptr.ptr + size, 1, st);
  counts.release();

  op->cols.alloc(op->nnz > 0 ? op->nnz : 1, st);
  op->grps.alloc(op->nnz > 0 ? op->nnz : 1, st);
  if (op->has_diag_group) {
    k_diag_entries<<<grid_for(nu, 256, 8192), 256, 0, st>>>(op->row_ptr.ptr, nu, size,
                                                             op->cols.ptr, op->grps.ptr);
    SQD_CHECK_LAUNCH();
  }
  P.row_ptr = op->row_ptr.ptr;
  P.cols = op->cols.ptr;
  P.grps = op->grps.ptr;
  P.diag_first = op->has_diag_group;
  {
    auto kern = k_sweep<SWEEP_FILL, double, 1, 1>;
    SQD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(dyn)));
    kern<<<tiles, SW_THREADS, dyn, st>>>(P);
    SQD_CHECK_LAUNCH();
  }
}

// Matrix elements of the stored pairs (z = 2) and the initial lanes-per-row choice.
void op_values_and_lanes(sqd_op_s* op, cudaStream_t st) {
  sqd_paulis_s* p = op->p;
  sqd_space_s* sp = op->s;
  const int64_t size = sp->states_size;
  const int64_t nu = sp->n_unique;
  if (op->z_cache == 2) {
    const int nca = op->value_complex ? 2 : 1;
    op->values.alloc(static_cast<size_t>(op->nnz > 0 ? op->nnz : 1) * nca, st);
    const unsigned G = grid_for(size * 32, 256, 16384);
    if (nca == 2)
      k_values<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr, nu,
                                     sp->fill_state, size, p->group_start.ptr, p->group_eff.ptr,
                                     p->term_z.ptr, p->term_c.ptr, op->values.ptr, 0);
    else
      k_values<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr, nu,
                                     sp->fill_state, size, p->group_start.ptr, p->group_eff.ptr,
                                     p->term_z.ptr, p->term_c.ptr, op->values.ptr, 0);
    SQD_CHECK_LAUNCH();
  }
  // Lanes per row from the mean row length.
  const double avg = nu > 0 ? static_cast<double>(op->nnz) / static_cast<double>(nu) : 0.0;
  const int lpr = avg >= 96 ? 32 : avg >= 40 ? 16 : avg >= 16 ? 8 : avg >= 6 ? 4 : 2;
  op->lanes_per_row[0] = op->lanes_per_row[1] = lpr;
  SQD_CUDA(cudaStreamSynchronize(st));
}

void op_ensure_values32(sqd_op_s* op, cudaStream_t st) {
  if (op->z_cache != 2 || op->nnz == 0) return;
  if (!op->values32.ptr) {
    const size_t n = static_cast<size_t>(op->nnz) * (op->value_complex ? 2 : 1);
    op->values32.alloc(n, st);
    k_to_float<<<grid_for(n, 256, 16384), 256, 0, st>>>(op->values.ptr, op->values32.ptr, n);
    SQD_CHECK_LAUNCH();
  }
  // FP32 slab copies only when FP32 vectors use a product layout.
  if (op->layout[1] != SQD_LAYOUT_CSR) op_product_values32(op, st);
}

}  // namespace sqd

using namespace sqd;

extern "C" int sqd_op_create(sqd_paulis_t p, sqd_space_t s, int x_cache, int z_cache,
                             int lookup, void* stream, sqd_op_t* out) {
  return guarded([&] {
    SQD_REQUIRE(out != nullptr, "out handle is NULL");
    *out = nullptr;
    SQD_REQUIRE(p && s, "NULL Pauli or space handle");
    SQD_REQUIRE(p->num_qubits == s->num_qubits,
                "Pauli strings and states have different numbers of qubits");
    SQD_REQUIRE(x_cache == 0 || x_cache == 1, "x cache strategy must be 0 or 1");
    SQD_REQUIRE(z_cache >= 0 && z_cache <= 2, "z cache strategy must be 0, 1 or 2");
    SQD_REQUIRE(lookup >= SQD_LOOKUP_HASH && lookup <= SQD_LOOKUP_PRODUCT, "bad lookup method");
    auto op = std::make_unique<sqd_op_s>();
    op->p = p;
    op->s = s;
    op->x_cache = x_cache;
    op->z_cache = (x_cache == 1) ? z_cache : 0;
    op->lookup = lookup;
    op_build(op.get(), as_stream(stream));
    *out = op.release();
  });
}

extern "C" int sqd_op_info(sqd_op_t op, int64_t* nnz, int64_t* states_size, int* value_complex) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    if (nnz) *nnz = op->nnz;
    if (states_size) *states_size = op->s->states_size;
    if (value_complex) *value_complex = op->value_complex;
  });
}

extern "C" int sqd_op_set_lanes(sqd_op_t op, int precision, int lanes_per_row) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    dispatch_lpr(lanes_per_row, [](auto) {});
    op->lanes_per_row[precision] = lanes_per_row;
    ++op->schedule_version;
  });
}

extern "C" int sqd_op_set_chunk(sqd_op_t op, int precision, int64_t chunk_rows) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    SQD_REQUIRE(chunk_rows >= 0, "chunk_rows must be >= 0");
    op->chunk_rows[precision] = chunk_rows;
    ++op->schedule_version;
  });
}

extern "C" int sqd_op_get_lanes(sqd_op_t op, int precision, int* lanes_per_row) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && lanes_per_row != nullptr, "NULL argument");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    *lanes_per_row = op->lanes_per_row[precision];
  });
}

extern "C" int sqd_diagonal(sqd_op_t op, int64_t group, void* out, int dtype, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && out != nullptr, "NULL argument");
    SQD_REQUIRE(dtype == SQD_F64 || dtype == SQD_C128, "diagonal dtype must be F64 or C128");
    sqd_paulis_s* p = op->p;
    SQD_REQUIRE(group >= 0 && group < p->num_groups, "group index out of range");
    sqd_space_s* sp = op->s;
    cudaStream_t st = as_stream(stream);
    const unsigned G = grid_for(sp->states_size, 256, 8192);
    if (p->is_complex)
      k_diagonal<2><<<G, 256, 0, st>>>(sp->states.ptr, sp->n_unique, sp->fill_state,
                                       sp->states_size, p->group_start.ptr, p->group_eff.ptr,
                                       p->term_z.ptr, p->term_c.ptr, group,
                                       static_cast<double*>(out), dtype == SQD_C128);
    else
      k_diagonal<1><<<G, 256, 0, st>>>(sp->states.ptr, sp->n_unique, sp->fill_state,
                                       sp->states_size, p->group_start.ptr, p->group_eff.ptr,
                                       p->term_z.ptr, p->term_c.ptr, group,
                                       static_cast<double*>(out), dtype == SQD_C128);
    SQD_CHECK_LAUNCH();
  });
}

extern "C" int sqd_vinit(sqd_op_t op, int64_t* index_host, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && index_host != nullptr, "NULL argument");
    if (!op->has_diag_group) {
      *index_host = 0;
      return;
    }
    sqd_paulis_s* p = op->p;
    sqd_space_s* sp = op->s;
    cudaStream_t st = as_stream(stream);
    const unsigned G = grid_for(sp->n_unique, 256, 1184);
    const int64_t nw = static_cast<int64_t>(G) * 8;
    DevBuf<unsigned long long> keys;
    DevBuf<long long> idx, res;
    keys.alloc(nw, st);
    idx.alloc(nw, st);
    res.alloc(1, st);
    k_argmin_partial<<<G, 256, 0, st>>>(sp->states.ptr, sp->n_unique, p->group_start.ptr,
                                        p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr,
                                        keys.ptr, idx.ptr);
    SQD_CHECK_LAUNCH();
    k_argmin_final<<<1, 1024, 0, st>>>(keys.ptr, idx.ptr, nw, res.ptr);
    SQD_CHECK_LAUNCH();
    long long h = 0;
    copy_to_host(&h, res.ptr, 1, st);
    *index_host = h;
  });
}

extern "C" int sqd_op_csr(sqd_op_t op, int64_t* indptr, int32_t* indices, double* data,
                          void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(op->x_cache == 1, "CSR export needs cache_strategy x = 1");
    SQD_REQUIRE(op->nnz == 0 || op->grps.ptr != nullptr,
                "the operator released its group indices; create a new operator");
    sqd_paulis_s* p = op->p;
    sqd_space_s* sp = op->s;
    cudaStream_t st = as_stream(stream);
    const int64_t size = sp->states_size;
    if (indptr)
      SQD_CUDA(cudaMemcpyAsync(indptr, op->row_ptr.ptr, (size + 1) * sizeof(int64_t),
                               cudaMemcpyDeviceToDevice, st));
    if (indices && op->nnz > 0) {
      k_cols_to_i32<<<grid_for(op->nnz, 256, 8192), 256, 0, st>>>(op->cols.ptr, indices,
                                                                   op->nnz);
      SQD_CHECK_LAUNCH();
    }
    if (data && op->nnz > 0) {
      const unsigned G = grid_for(size * 32, 256, 16384);
      if (p->is_complex)
        k_values<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr,
                                       sp->n_unique, sp->fill_state, size, p->group_start.ptr,
                                       p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr, data, 1);
      else
        k_values<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr,
                                       sp->n_unique, sp->fill_state, size, p->group_start.ptr,
                                       p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr, data, 1);
      SQD_CHECK_LAUNCH();
    }
  });
}

extern "C" int sqd_op_cache_values(sqd_op_t op, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(op->x_cache == 1, "caching elements needs cached sources (cache_strategy (1, *))");
    if (op->z_cache == 2) return;
    op->z_cache = 2;
    try {
      op_values_and_lanes(op, as_stream(stream));
    } catch (...) {
      op->values.release();
      op->z_cache = 0;
      throw;
    }
    ++op->schedule_version;
  });
}

extern "C" int sqd_op_release_groups(sqd_op_t op) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(op->x_cache == 1 && op->z_cache == 2,
                "only operators with cached matrix elements can release their group indices");
    op->grps.release();
  });
}

extern "C" int sqd_op_refresh(sqd_op_t op, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr, "NULL operator");
    SQD_REQUIRE(op->z_cache != 2 || op->nnz == 0 || op->grps.ptr != nullptr,
                "the operator released its group indices; create a new operator");
    sqd_paulis_s* p = op->p;
    sqd_space_s* sp = op->s;
    SQD_REQUIRE(p->is_complex == op->value_complex,
                "the Pauli sum changed between real and complex; create a new operator");
    if (op->z_cache != 2 || op->nnz == 0) return;
    cudaStream_t st = as_stream(stream);
    const int64_t size = sp->states_size;
    const unsigned G = grid_for(size * 32, 256, 16384);
    if (op->value_complex)
      k_values<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr,
                                     sp->n_unique, sp->fill_state, size, p->group_start.ptr,
                                     p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr,
                                     op->values.ptr, 0);
    else
      k_values<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->grps.ptr, sp->states.ptr,
                                     sp->n_unique, sp->fill_state, size, p->group_start.ptr,
                                     p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr,
                                     op->values.ptr, 0);
    SQD_CHECK_LAUNCH();
    if (op->values32.ptr) {
      const size_t n = static_cast<size_t>(op->nnz) * (op->value_complex ? 2 : 1);
      k_to_float<<<grid_for(n, 256, 16384), 256, 0, st>>>(op->values.ptr, op->values32.ptr, n);
      SQD_CHECK_LAUNCH();
    }
    op_product_values(op, st);
    ++op->schedule_version;
  });
}

extern "C" int sqd_grad_terms(sqd_op_t op, const void* u, const void* v, int dtype,
                              double* out_terms, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && u && v && out_terms, "NULL argument");
    SQD_REQUIRE(op->x_cache == 1, "the coefficient gradient needs cache_strategy x = 1");
    SQD_REQUIRE(op->nnz == 0 || op->grps.ptr != nullptr,
                "the operator released its group indices; create a new operator");
    SQD_REQUIRE(dtype == SQD_F64 || dtype == SQD_C128, "gradient dtype must be F64 or C128");
    SQD_REQUIRE(dtype == SQD_C128 || !op->value_complex, "complex Hamiltonian needs C128");
    sqd_paulis_s* p = op->p;
    sqd_space_s* sp = op->s;
    cudaStream_t st = as_stream(stream);
    SQD_CUDA(cudaMemsetAsync(out_terms, 0, p->num_terms * sizeof(double), st));
    const double* ud = static_cast<const double*>(u);
    const double* vd = static_cast<const double*>(v);
    if (op->has_diag_group && sp->n_unique > 0) {
      const unsigned G = grid_for(sp->n_unique, GR_TILE);
      if (dtype == SQD_C128)
        k_grad_diag<2><<<G, 256, 0, st>>>(sp->states.ptr, sp->n_unique, p->group_start.ptr,
                                          p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr, ud, vd,
                                          out_terms);
      else
        k_grad_diag<1><<<G, 256, 0, st>>>(sp->states.ptr, sp->n_unique, p->group_start.ptr,
                                          p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr, ud, vd,
                                          out_terms);
      SQD_CHECK_LAUNCH();
    }
    const unsigned G = grid_for(sp->n_unique * 32, 256, 16384);
    if (dtype == SQD_C128)
      k_grad_offdiag<2><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->grps.ptr,
                                           sp->states.ptr, sp->n_unique, op->has_diag_group,
                                           p->group_start.ptr, p->group_eff.ptr, p->group_x.ptr,
                                           p->term_z.ptr, ud, vd, out_terms);
    else
      k_grad_offdiag<1><<<G, 256, 0, st>>>(op->row_ptr.ptr, op->cols.ptr, op->grps.ptr,
                                           sp->states.ptr, sp->n_unique, op->has_diag_group,
                                           p->group_start.ptr, p->group_eff.ptr, p->group_x.ptr,
                                           p->term_z.ptr, ud, vd, out_terms);
    SQD_CHECK_LAUNCH();
  });
}

extern "C" void sqd_op_destroy(sqd_op_t op) { delete op; }
