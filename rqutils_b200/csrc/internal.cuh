// Internal handle layouts shared by the library's translation units.
#pragma once

#include "common.cuh"

// Grouped Pauli table (device CSR).  Mirrors PauliSumXZ (paulis/symplectic.py:41-48): groups
// ascending in x, terms ascending in z inside a group, coefficients already multiplied by
// (-i)^{popcount(x & z)}.
struct sqd_paulis_s {
  int num_qubits = 0;
  int64_t num_raw = 0;
  int64_t num_terms = 0;   // M (merged)
  int64_t num_groups = 0;  // J
  int64_t max_k = 0;       // largest group
  int is_complex = 0;      // any phased coefficient with a nonzero imaginary part
  sqd::DevBuf<uint64_t> group_x;      // [J]
  sqd::DevBuf<int64_t> group_start;   // [J+1]
  sqd::DevBuf<int32_t> group_eff;     // [J] terms used by the diagonal (stop at first zero)
  sqd::DevBuf<uint64_t> term_z;       // [M]
  sqd::DevBuf<double> term_c;         // [2M] interleaved (re, im)
  sqd::DevBuf<int32_t> term_group;    // [M]
  sqd::DevBuf<int32_t> raw_to_term;   // [num_raw]
  // term -> raw terms merged into it, in input order (for coefficient updates)
  int64_t num_kept = 0;
  uint32_t flags = 0;
  sqd::DevBuf<int64_t> term_raw_start;  // [M + 1] into term_raw
  sqd::DevBuf<uint32_t> term_raw;       // [num_kept] raw indices
  sqd::DevBuf<uint64_t> term_x;         // [M]
};

// Sorted unique subspace plus lookup structures.
struct sqd_space_s {
  int num_qubits = 0;
  int64_t n_unique = 0;
  int64_t states_size = 0;
  uint64_t fill_state = 0;            // all-ones over the qubit bits (the 255 rows' diagonal)
  sqd::DevBuf<uint64_t> states;       // [n_unique]
  // Open-addressing hash table (linear probing, load <= 1/2): key -> row index.
  sqd::DevBuf<uint64_t> hkeys;
  sqd::DevBuf<uint32_t> hvals;
  uint64_t hmask = 0;
  // Conserved-weight sectors: popcount(s & sector_mask[l]) == sector_weight[l] for every state.
  int num_sectors = 0;
  uint64_t sector_mask[2] = {0, 0};
  int sector_weight[2] = {0, 0};
  // Per-sector membership bitmaps over the sector projection (exact when the sector is at most
  // kBitmapBits wide, hashed otherwise).  Used as a no-false-negative prefilter.
  sqd::DevBuf<uint32_t> bitmap;       // [num_sectors << kBitmapLog2 / 32]
};

constexpr int kBitmapLog2 = 17;

namespace sqd {
// Low half of the qubits (bits 0 .. n/2 - 1): the low sector of the conserved-weight sectors and
// of the product layout.
inline uint64_t half_mask_low(int num_qubits) {
  const int h = num_qubits / 2;
  return h == 0 ? 0ull : ((1ull << h) - 1ull);
}
}  // namespace sqd

// Per-group data for the connectivity sweep.
struct GroupPre {
  uint64_t x;
  int32_t group;     // group index j
  int32_t cx;        // popcount(x & sector_mask[l]) packed as bytes (l = 0, 1)
};

// Product-subspace layout of the cached matvec (product.cu).  Rows r = h * nl + l.  H entries
// of slab h: k in [ho[h], ho[h+1]), source offset hsrc[k] = h' * nl, elements vh at
// panel-major ((l / 32) * th + k) * 32 + l % 32; L entries of low string l: e in
// [lo[l], lo[l+1]), source offset lsrc[e] = l' * nh (into the transposed vector), elements vl
// at ((h / 32) * tl + e) * 32 + h % 32.  The rest of a row (M pairs) stays in the CSR arrays
// after the first (ho[h+1] - ho[h]) + (lo[l+1] - lo[l]) pairs.
struct ProductLayout {
  int built = 0;
  int64_t nh = 0, nl = 0;
  int64_t th = 0, tl = 0;            // H and L entries over all slabs
  int64_t pairs_h = 0, pairs_l = 0, pairs_m = 0;
  sqd::DevBuf<int64_t> ho, lo;       // [nh + 1], [nl + 1]
  sqd::DevBuf<uint32_t> hsrc, lsrc;  // [th], [tl]
  sqd::DevBuf<double> vh, vl;        // FP64 elements (x2 interleaved when complex)
  sqd::DevBuf<float> vh32, vl32;     // FP32 copies (64-wide panels when wide32)
  int wide32 = 0;                    // both halves even: FP32 slabs read two positions per lane
  sqd::DevBuf<double> vt, tt, t;     // per-matvec scratch: transposed input, L and M partials
  // Compact copies of the row tails (the M pairs of each row, contiguous: mptr, mval) with the
  // sources in one or both of two forms.  Shared memory (tail_slots > 0), when every slab's M
  // source slabs fit there together: indices into the block's staged slabs (msidx = slot * nl +
  // l'), and each slab's source slabs are listed (slist).  Short tails (compact_tail): rows
  // (mcol), read by the CSR tail kernel.
  int tail_slots = 0;                // largest number of M source slabs of one slab
  int compact_tail = 0;
  sqd::DevBuf<int64_t> mptr;         // [n + 1]
  sqd::DevBuf<uint16_t> msidx;       // [pairs_m] (shared-memory form)
  sqd::DevBuf<uint32_t> mcol;        // [pairs_m] (short-tail form)
  sqd::DevBuf<double> mval;          // [pairs_m] (x2 interleaved when complex)
  sqd::DevBuf<float> mval32;
  sqd::DevBuf<int64_t> soff;         // [nh + 1]
  sqd::DevBuf<uint32_t> slist;       // [soff[nh]] ascending source slabs
};

// Solver objects an operator keeps between LOCG solves (locg.cu): work vectors and the
// instantiated CUDA graphs of the iteration, rebuilt when the matvec schedule changes.
struct LocgCacheBase {
  virtual ~LocgCacheBase() = default;
};

struct sqd_op_s {
  sqd_paulis_s* p = nullptr;   // borrowed: must outlive the operator
  sqd_space_s* s = nullptr;    // borrowed
  int x_cache = 1, z_cache = 0, lookup = SQD_LOOKUP_HASH;
  int has_diag_group = 0;      // group 0 has x == 0
  int value_complex = 0;
  int64_t nnz = 0;
  int lanes_per_row[2] = {32, 32};  // [0]: FP64 vectors, [1]: FP32 vectors
  int64_t chunk_rows[2] = {0, 0};   // rows a block owns at a time (0 = interleaved rows)
  sqd::DevBuf<int64_t> row_ptr;   // [states_size + 1]
  sqd::DevBuf<uint32_t> cols;     // [nnz] source index of each stored pair
  sqd::DevBuf<uint32_t> grps;     // [nnz] group index of each stored pair
  sqd::DevBuf<double> values;     // [nnz] or [2 nnz]: composed diagonal per stored pair
  sqd::DevBuf<float> values32;    // FP32 copy for the mixed-precision matvec
  sqd::DevBuf<GroupPre> gpre;     // groups that can connect (x != 0, even sector counts)
  int64_t n_gpre = 0;
  int64_t n_gpre_cls[3] = {0, 0, 0};  // gpre entries per class (H, L, M), in that order
  int product_built = 0;          // connectivity assembled from the two halves' lists
  sqd::DevBuf<int> status;        // device status word
  int layout[2] = {0, 0};         // SQD_LAYOUT_* per precision
  ProductLayout prod;
  // Bumped whenever the kernels or buffers a matvec launches may change (lanes, chunk,
  // layout, coefficient refresh): cached solver graphs captured before are then stale.
  uint64_t schedule_version = 0;
  std::unique_ptr<LocgCacheBase> locg_cache;
};

namespace sqd {

// Lookup of key in the space: index or -1.
__device__ __forceinline__ int64_t hash_lookup(const uint64_t* __restrict__ keys,
                                               const uint32_t* __restrict__ vals, uint64_t mask,
                                               uint64_t key) {
  uint64_t slot = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const uint64_t k = __ldg(keys + slot);
    if (k == key) return static_cast<int64_t>(__ldg(vals + slot));
    if (k == kEmptyKey) return -1;
    slot = (slot + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ int64_t bsearch_lookup(const uint64_t* __restrict__ states, int64_t n,
                                                  uint64_t key) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(states + mid) < key) lo = mid + 1; else hi = mid;
  }
  return (lo < n && __ldg(states + lo) == key) ? lo : -1;
}

__device__ __forceinline__ uint32_t sector_bitmap_index(uint64_t proj, int shift, bool exact) {
  const uint64_t v = exact ? (proj >> shift) : mix64(proj);
  return static_cast<uint32_t>(v & ((1ull << kBitmapLog2) - 1));
}

// Build helpers implemented in matvec.cu / connect.cu.
void op_build(sqd_op_s* op, cudaStream_t st);
void op_matvec(sqd_op_s* op, const void* v, void* out, int dtype, cudaStream_t st);
void op_ensure_values32(sqd_op_s* op, cudaStream_t st);
// Product layout (product.cu).
bool op_product_detect(sqd_op_s* op, cudaStream_t st, int64_t* nh, int64_t* nl);
void op_product_build(sqd_op_s* op, cudaStream_t st);
void op_product_values(sqd_op_s* op, cudaStream_t st);
void op_product_values32(sqd_op_s* op, cudaStream_t st);
void op_product_matvec(sqd_op_s* op, const void* v, void* out, int dtype, cudaStream_t st);
// Connectivity (row_ptr, cols, grps, nnz) of a product subspace from per-half partner lists;
// false when the subspace is not such a product.
bool op_connect_product(sqd_op_s* op, cudaStream_t st);

}  // namespace sqd
