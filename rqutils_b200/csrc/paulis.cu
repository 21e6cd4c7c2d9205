// Device-side Pauli-sum preprocessing: PauliSumXZ.from_paulisum (paulis/symplectic.py:50-124).
//
// Pipeline (all on the device, stream-ordered):
//   1. drop zero coefficients (symplectic.py:67-69);
//   2. stable radix sort of the terms by the 2-word key (x, z) — the order np.unique gives the
//      reference's Pauli strings: 'I' < 'X' < 'Y' < 'Z' per character, character 0 = highest
//      qubit, which is ascending (x, z) as integers;
//   3. merge equal (x, z) runs by summing their coefficients in input order (:70-72);
//   4. optional force_real (:92-95);
//   5. group by x (:98-101), multiply each coefficient by (-i)^{popcount(x & z) mod 4}
//      (:109-111), detect whether any imaginary part survives (:113-114);
//   6. per group, the number of terms before the first zero coefficient — get_diagonal stops
//      there (sqd.py:611-613), and the matvec mirrors that.
#include "internal.cuh"

namespace sqd {
namespace {

__global__ void k_keep_flags(const double* re, const double* im, int64_t n, int64_t* flags) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    flags[i] = (re[i] != 0.0 || (im != nullptr && im[i] != 0.0)) ? 1 : 0;
}

__global__ void k_compact_terms(const uint64_t* x, const uint64_t* z, const int64_t* flags,
                                const int64_t* pos, int64_t n, uint64_t* xo, uint64_t* zo,
                                uint32_t* idx) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    if (flags[i]) {
      const int64_t p = pos[i];
      xo[p] = x[i];
      zo[p] = z[i];
      idx[p] = static_cast<uint32_t>(i);
    }
  }
}

__global__ void k_run_flags(const uint64_t* x, const uint64_t* z, int64_t n, int64_t* new_term) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    new_term[i] = (i == 0 || x[i] != x[i - 1] || z[i] != z[i - 1]) ? 1 : 0;
}

// item -> term id (inclusive position), term start positions.
__global__ void k_term_starts(const int64_t* new_term, const int64_t* term_pos, int64_t n,
                              int64_t* term_item_start) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    if (new_term[i]) term_item_start[term_pos[i]] = i;
}

// One thread per merged term: sequential sum of its items' coefficients in input order.
__global__ void k_merge_terms(const uint64_t* xs, const uint64_t* zs, const uint32_t* idx,
                              const int64_t* term_item_start, int64_t n_items, int64_t m,
                              const double* re, const double* im, int force_real,
                              uint64_t* term_x, uint64_t* term_z, double* term_c,
                              int32_t* raw_to_term, int* imag_dropped) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < m;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = term_item_start[t];
    const int64_t e = (t + 1 < m) ? term_item_start[t + 1] : n_items;
    double sr = 0.0, si = 0.0;
    for (int64_t i = b; i < e; ++i) {
      const uint32_t r = idx[i];
      sr += re[r];
      if (im) si += im[r];
      raw_to_term[r] = static_cast<int32_t>(t);
    }
    if (force_real) {
      if (si != 0.0) atomicExch(imag_dropped, 1);
      si = 0.0;
    }
    const uint64_t x = xs[b], z = zs[b];
    // (-i)^ph: 0 -> (a, b); 1 -> (b, -a); 2 -> (-a, -b); 3 -> (-b, a)
    const int ph = __popcll(x & z) & 3;
    double cr, ci;
    switch (ph) {
      case 0: cr = sr; ci = si; break;
      case 1: cr = si; ci = -sr; break;
      case 2: cr = -sr; ci = -si; break;
      default: cr = -si; ci = sr; break;
    }
    term_x[t] = x;
    term_z[t] = z;
    term_c[2 * t] = cr;
    term_c[2 * t + 1] = ci;
  }
}

__global__ void k_group_flags(const uint64_t* term_x, const double* term_c, int64_t m,
                              int64_t* new_group, int* any_imag) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < m;
       t += int64_t(gridDim.x) * blockDim.x) {
    new_group[t] = (t == 0 || term_x[t] != term_x[t - 1]) ? 1 : 0;
    if (term_c[2 * t + 1] != 0.0) atomicExch(any_imag, 1);
  }
}

__global__ void k_group_starts(const int64_t* new_group, const int64_t* gpos,
                               const uint64_t* term_x, int64_t m, int64_t* group_start,
                               uint64_t* group_x, int32_t* term_group) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < m;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int64_t g = gpos[t] + new_group[t] - 1;
    term_group[t] = static_cast<int32_t>(g);
    if (new_group[t]) {
      group_start[g] = t;
      group_x[g] = term_x[t];
    }
  }
}

__global__ void k_group_eff(const int64_t* group_start, const double* term_c, int64_t j_count,
                            int32_t* group_eff, unsigned long long* max_k) {
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < j_count;
       g += int64_t(gridDim.x) * blockDim.x) {
    const int64_t b = group_start[g], e = group_start[g + 1];
    int64_t eff = e - b;
    for (int64_t t = b; t < e; ++t) {
      if (term_c[2 * t] == 0.0 && term_c[2 * t + 1] == 0.0) {
        eff = t - b;
        break;
      }
    }
    group_eff[g] = static_cast<int32_t>(eff);
    atomicMax(max_k, static_cast<unsigned long long>(e - b));
  }
}

}  // namespace
}  // namespace sqd

using namespace sqd;

extern "C" int sqd_paulis_create(const uint64_t* x, const uint64_t* z, const double* coef_re,
                                 const double* coef_im, int64_t num_raw, int num_qubits,
                                 uint32_t flags, void* stream, sqd_paulis_t* out,
                                 int* imag_dropped_host) {
  return guarded([&] {
    SQD_REQUIRE(out != nullptr, "out handle is NULL");
    *out = nullptr;
    SQD_REQUIRE(num_raw > 0, "empty Pauli sum");
    SQD_REQUIRE(num_raw < (int64_t(1) << 31), "too many Pauli terms");
    SQD_REQUIRE(num_qubits >= 1 && num_qubits <= 63, "num_qubits must be in [1, 63]");
    SQD_REQUIRE(x && z && coef_re, "NULL input array");
    cudaStream_t st = as_stream(stream);
    const int B = 256;
    const unsigned G = grid_for(num_raw, B, 4096);

    auto p = std::make_unique<sqd_paulis_s>();
    p->num_qubits = num_qubits;
    p->num_raw = num_raw;

    DevBuf<int64_t> flags_keep, pos;
    flags_keep.alloc(num_raw, st);
    pos.alloc(num_raw + 1, st);
    k_keep_flags<<<G, B, 0, st>>>(coef_re, coef_im, num_raw, flags_keep.ptr);
    SQD_CHECK_LAUNCH();
    exclusive_scan_i64(flags_keep.ptr, pos.ptr, num_raw, true, st);
    int64_t n_kept = 0;
    copy_to_host(&n_kept, pos.ptr + num_raw, 1, st);
    SQD_REQUIRE(n_kept > 0, "all Pauli coefficients are zero");

    DevBuf<uint64_t> xs, zs;
    DevBuf<uint32_t> idx;
    xs.alloc(n_kept, st);
    zs.alloc(n_kept, st);
    idx.alloc(n_kept, st);
    k_compact_terms<<<G, B, 0, st>>>(x, z, flags_keep.ptr, pos.ptr, num_raw, xs.ptr, zs.ptr,
                                     idx.ptr);
    SQD_CHECK_LAUNCH();
    radix_sort_pair(xs.ptr, zs.ptr, idx.ptr, n_kept, num_qubits, num_qubits, st);

    DevBuf<int64_t> new_term, term_pos;
    new_term.alloc(n_kept, st);
    term_pos.alloc(n_kept + 1, st);
    const unsigned Gk = grid_for(n_kept, B, 4096);
    k_run_flags<<<Gk, B, 0, st>>>(xs.ptr, zs.ptr, n_kept, new_term.ptr);
    SQD_CHECK_LAUNCH();
    exclusive_scan_i64(new_term.ptr, term_pos.ptr, n_kept, true, st);
    int64_t m = 0;
    copy_to_host(&m, term_pos.ptr + n_kept, 1, st);
    p->num_terms = m;

    DevBuf<int64_t>& term_item_start = p->term_raw_start;
    term_item_start.alloc(m + 1, st);
    k_term_starts<<<Gk, B, 0, st>>>(new_term.ptr, term_pos.ptr, n_kept, term_item_start.ptr);
    SQD_CHECK_LAUNCH();
    SQD_CUDA(cudaMemcpyAsync(term_item_start.ptr + m, &n_kept, sizeof(int64_t),
                             cudaMemcpyHostToDevice, st));
    p->num_kept = n_kept;
    p->flags = flags;

    DevBuf<uint64_t>& term_x = p->term_x;
    DevBuf<int> flags_dev;
    term_x.alloc(m, st);
    p->term_z.alloc(m, st);
    p->term_c.alloc(2 * m, st);
    p->raw_to_term.alloc(num_raw, st);
    flags_dev.alloc(2, st);
    SQD_CUDA(cudaMemsetAsync(flags_dev.ptr, 0, 2 * sizeof(int), st));
    SQD_CUDA(cudaMemsetAsync(p->raw_to_term.ptr, 0xff, num_raw * sizeof(int32_t), st));
    const unsigned Gm = grid_for(m, B, 4096);
    k_merge_terms<<<Gm, B, 0, st>>>(xs.ptr, zs.ptr, idx.ptr, term_item_start.ptr, n_kept, m,
                                    coef_re, coef_im, (flags & SQD_PAULIS_FORCE_REAL) ? 1 : 0,
                                    term_x.ptr, p->term_z.ptr, p->term_c.ptr,
                                    p->raw_to_term.ptr, flags_dev.ptr);
    SQD_CHECK_LAUNCH();

    DevBuf<int64_t> new_group, gpos;
    new_group.alloc(m, st);
    gpos.alloc(m + 1, st);
    k_group_flags<<<Gm, B, 0, st>>>(term_x.ptr, p->term_c.ptr, m, new_group.ptr,
                                    flags_dev.ptr + 1);
    SQD_CHECK_LAUNCH();
    exclusive_scan_i64(new_group.ptr, gpos.ptr, m, true, st);
    int64_t jn = 0;
    copy_to_host(&jn, gpos.ptr + m, 1, st);
    p->num_groups = jn;
    p->group_start.alloc(jn + 1, st);
    p->group_x.alloc(jn, st);
    p->group_eff.alloc(jn, st);
    p->term_group.alloc(m, st);
    k_group_starts<<<Gm, B, 0, st>>>(new_group.ptr, gpos.ptr, term_x.ptr, m, p->group_start.ptr,
                                     p->group_x.ptr, p->term_group.ptr);
    SQD_CHECK_LAUNCH();
    SQD_CUDA(cudaMemcpyAsync(p->group_start.ptr + jn, &m, sizeof(int64_t),
                             cudaMemcpyHostToDevice, st));
    DevBuf<unsigned long long> maxk;
    maxk.alloc(1, st);
    SQD_CUDA(cudaMemsetAsync(maxk.ptr, 0, sizeof(unsigned long long), st));
    k_group_eff<<<grid_for(jn, B, 4096), B, 0, st>>>(p->group_start.ptr, p->term_c.ptr, jn,
                                                     p->group_eff.ptr, maxk.ptr);
    SQD_CHECK_LAUNCH();
    int hflags[2];
    unsigned long long hmax = 0;
    SQD_CUDA(cudaMemcpyAsync(hflags, flags_dev.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    SQD_CUDA(cudaMemcpyAsync(&hmax, maxk.ptr, sizeof(hmax), cudaMemcpyDeviceToHost, st));
    SQD_CUDA(cudaStreamSynchronize(st));
    p->is_complex = hflags[1];
    p->max_k = static_cast<int64_t>(hmax);
    if (imag_dropped_host) *imag_dropped_host = hflags[0];
    p->term_raw.swap(idx);
    *out = p.release();
  });
}

namespace sqd {
namespace {

// New coefficients for the same terms: merged sums in input order, phase, as at creation.
__global__ void k_set_coeffs(const int64_t* trs, const uint32_t* tr, int64_t m,
                             const uint64_t* term_x, const uint64_t* term_z, const double* re,
                             const double* im, int force_real, double* term_c, int* flags) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < m;
       t += int64_t(gridDim.x) * blockDim.x) {
    double sr = 0.0, si = 0.0;
    for (int64_t i = trs[t]; i < trs[t + 1]; ++i) {
      sr += re[tr[i]];
      if (im) si += im[tr[i]];
    }
    if (force_real) {
      if (si != 0.0) atomicExch(flags, 1);
      si = 0.0;
    }
    const int ph = __popcll(term_x[t] & term_z[t]) & 3;
    double cr, ci;
    switch (ph) {
      case 0: cr = sr; ci = si; break;
      case 1: cr = si; ci = -sr; break;
      case 2: cr = -sr; ci = -si; break;
      default: cr = -si; ci = sr; break;
    }
    term_c[2 * t] = cr;
    term_c[2 * t + 1] = ci;
    if (ci != 0.0) atomicExch(flags + 1, 1);
  }
}

// A raw term dropped at creation (zero coefficient) must stay zero: the table has no slot.
__global__ void k_check_dropped(const int32_t* raw_to_term, const double* re, const double* im,
                                int64_t n, int* flag) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n;
       r += int64_t(gridDim.x) * blockDim.x)
    if (raw_to_term[r] < 0 && (re[r] != 0.0 || (im != nullptr && im[r] != 0.0)))
      atomicExch(flag, 1);
}

}  // namespace
}  // namespace sqd

extern "C" int sqd_paulis_set_coeffs(sqd_paulis_t p, const double* coef_re,
                                     const double* coef_im, void* stream,
                                     int* imag_dropped_host) {
  return guarded([&] {
    SQD_REQUIRE(p != nullptr && coef_re != nullptr, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const int B = 256;
    DevBuf<int> flags;
    flags.alloc(3, st);
    SQD_CUDA(cudaMemsetAsync(flags.ptr, 0, 3 * sizeof(int), st));
    k_check_dropped<<<grid_for(p->num_raw, B, 4096), B, 0, st>>>(
        p->raw_to_term.ptr, coef_re, coef_im, p->num_raw, flags.ptr + 2);
    SQD_CHECK_LAUNCH();
    int h[3];
    copy_to_host(h, flags.ptr, 3, st);
    SQD_REQUIRE(h[2] == 0,
                "a term whose coefficient was zero when the Pauli sum was created became nonzero; "
                "create a new Pauli sum");
    DevBuf<double> newc;
    newc.alloc(2 * p->num_terms, st);
    k_set_coeffs<<<grid_for(p->num_terms, B, 4096), B, 0, st>>>(
        p->term_raw_start.ptr, p->term_raw.ptr, p->num_terms, p->term_x.ptr, p->term_z.ptr,
        coef_re, coef_im, (p->flags & SQD_PAULIS_FORCE_REAL) ? 1 : 0, newc.ptr, flags.ptr);
    SQD_CHECK_LAUNCH();
    copy_to_host(h, flags.ptr, 2, st);
    SQD_REQUIRE(h[1] == 0 || p->is_complex,
                "new coefficients make a real Hamiltonian complex; create a new Pauli sum");
    SQD_CUDA(cudaMemcpyAsync(p->term_c.ptr, newc.ptr, newc.bytes(), cudaMemcpyDeviceToDevice, st));
    DevBuf<unsigned long long> maxk;
    maxk.alloc(1, st);
    SQD_CUDA(cudaMemsetAsync(maxk.ptr, 0, sizeof(unsigned long long), st));
    k_group_eff<<<grid_for(p->num_groups, B, 4096), B, 0, st>>>(
        p->group_start.ptr, p->term_c.ptr, p->num_groups, p->group_eff.ptr, maxk.ptr);
    SQD_CHECK_LAUNCH();
    SQD_CUDA(cudaStreamSynchronize(st));
    if (imag_dropped_host) *imag_dropped_host = h[0];
  });
}

extern "C" int sqd_paulis_info(sqd_paulis_t p, int64_t* num_groups, int64_t* num_terms,
                               int64_t* max_k, int* is_complex, int* num_qubits) {
  return guarded([&] {
    SQD_REQUIRE(p != nullptr, "NULL Pauli handle");
    if (num_groups) *num_groups = p->num_groups;
    if (num_terms) *num_terms = p->num_terms;
    if (max_k) *max_k = p->max_k;
    if (is_complex) *is_complex = p->is_complex;
    if (num_qubits) *num_qubits = p->num_qubits;
  });
}

extern "C" int sqd_paulis_export(sqd_paulis_t p, uint64_t* group_x, int64_t* group_start,
                                 uint64_t* term_z, double* term_c, int32_t* raw_to_term,
                                 void* stream) {
  return guarded([&] {
    SQD_REQUIRE(p != nullptr, "NULL Pauli handle");
    cudaStream_t st = as_stream(stream);
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) SQD_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st));
    };
    cp(group_x, p->group_x.ptr, p->group_x.bytes());
    cp(group_start, p->group_start.ptr, p->group_start.bytes());
    cp(term_z, p->term_z.ptr, p->term_z.bytes());
    cp(term_c, p->term_c.ptr, p->term_c.bytes());
    cp(raw_to_term, p->raw_to_term.ptr, p->raw_to_term.bytes());
  });
}

extern "C" void sqd_paulis_destroy(sqd_paulis_t p) { delete p; }
