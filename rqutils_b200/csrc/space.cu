// Subspace construction and the b XOR x lookup.
//
//  * sqd_pack_states: the uint64 form of np.packbits(np.pad(states, (1, 0))) (sqd.py:255).
//    Ascending uint64 order equals the reference's lexicographic order of padded big-endian
//    byte rows, because the pad bit is 0 for every real state.
//  * sqd_space_create: uniquify_states (sqd.py:445-482) — radix sort + unique; the fill-in
//    slots are kept implicit (states_size > n_unique), then lookup structures are built:
//    an open-addressing hash table, conserved-weight sectors and sector bitmaps.
//  * sqd_xsource: get_xsource (sqd.py:485-548) for one X mask, bit-exact including the values
//    the reference's sort-based algorithm produces for fill-in slots.
//  * sqd_space_lookup: sorted index of arbitrary keys, for the unsorted-input branch of
//    get_xsource (sqd.py:515-516, 542-545) and the indices of uniquify_states (sqd.py:478-481).
#include "internal.cuh"

namespace sqd {
namespace {

__global__ void k_pack(const uint8_t* __restrict__ bits, int64_t n_rows, int nq,
                       uint64_t* __restrict__ out) {
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < n_rows;
       r += int64_t(gridDim.x) * blockDim.x) {
    const uint8_t* row = bits + r * nq;
    uint64_t v = 0;
    for (int c = 0; c < nq; ++c) v |= static_cast<uint64_t>(row[c] & 1u) << (nq - 1 - c);
    out[r] = v;
  }
}

__global__ void k_unique_flags(const uint64_t* s, int64_t n, int64_t* flags) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    flags[i] = (i == 0 || s[i] != s[i - 1]) ? 1 : 0;
}

__global__ void k_unique_scatter(const uint64_t* s, const int64_t* flags, const int64_t* pos,
                                 int64_t n, uint64_t* out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    if (flags[i]) out[pos[i]] = s[i];
}

__global__ void k_hash_insert(const uint64_t* __restrict__ s, int64_t n, uint64_t* keys,
                              uint32_t* vals, uint64_t mask, int* status) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t key = s[i];
    uint64_t slot = mix64(key) & mask;
    bool done = false;
    for (uint64_t probe = 0; probe <= mask; ++probe) {
      const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(keys + slot),
                                                static_cast<unsigned long long>(kEmptyKey),
                                                static_cast<unsigned long long>(key));
      if (prev == kEmptyKey || prev == key) {
        vals[slot] = static_cast<uint32_t>(i);
        done = true;
        break;
      }
      slot = (slot + 1) & mask;
    }
    if (!done) atomicExch(status, 1);
  }
}

// min/max of popcount(s & m) for m in {all bits, low half, high half}.
__global__ void k_sector_stats(const uint64_t* __restrict__ s, int64_t n, uint64_t m_all,
                               uint64_t m_lo, uint64_t m_hi, int* stats /* [6] min,max x3 */) {
  int mn[3] = {64, 64, 64}, mx[3] = {0, 0, 0};
  const uint64_t m[3] = {m_all, m_lo, m_hi};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t v = s[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int c = __popcll(v & m[k]);
      mn[k] = min(mn[k], c);
      mx[k] = max(mx[k], c);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    atomicMin(stats + 2 * k, mn[k]);
    atomicMax(stats + 2 * k + 1, mx[k]);
  }
}

__global__ void k_bitmap_build(const uint64_t* __restrict__ s, int64_t n, int nsec, uint64_t m0,
                               uint64_t m1, int sh0, int sh1, int ex0, int ex1,
                               uint32_t* bitmap) {
  constexpr uint32_t words = (1u << kBitmapLog2) / 32;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t v = s[i];
    uint32_t b = sector_bitmap_index(v & m0, sh0, ex0);
    atomicOr(bitmap + (b >> 5), 1u << (b & 31));
    if (nsec > 1) {
      b = sector_bitmap_index(v & m1, sh1, ex1);
      atomicOr(bitmap + words + (b >> 5), 1u << (b & 31));
    }
  }
}

__global__ void k_popc_sum(const uint32_t* w, int64_t n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    acc += __popc(w[i]);
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// get_xsource for one x.  Real rows: index of s^x or -1.  Fill-in slots f_1..f_m (all equal
// to the 255 row): the stable sort of [S; S^x] puts them consecutively, so the reference
// yields f_{i+1} - size for i < m, and for the last one f_1 when x == 0 (its equal successor
// is its own copy in the second half) or -1 otherwise.
__global__ void k_xsource(const uint64_t* __restrict__ states, int64_t n_unique,
                          int64_t states_size, uint64_t x, const uint64_t* __restrict__ hkeys,
                          const uint32_t* __restrict__ hvals, uint64_t hmask, int lookup,
                          int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < states_size;
       i += int64_t(gridDim.x) * blockDim.x) {
    int64_t r;
    if (i < n_unique) {
      const uint64_t key = __ldg(states + i) ^ x;
      r = (lookup == SQD_LOOKUP_BSEARCH) ? bsearch_lookup(states, n_unique, key)
                                         : hash_lookup(hkeys, hvals, hmask, key);
    } else if (i + 1 < states_size) {
      r = (i + 1) - states_size;
    } else {
      r = (x == 0) ? n_unique : -1;
    }
    out[i] = static_cast<int32_t>(r);
  }
}

// Row index of arbitrary keys: -1 when absent or when a key has bits above num_qubits.
__global__ void k_lookup_keys(const uint64_t* __restrict__ q, int64_t n, uint64_t valid,
                              const uint64_t* __restrict__ states, int64_t n_unique,
                              const uint64_t* __restrict__ hkeys,
                              const uint32_t* __restrict__ hvals, uint64_t hmask, int lookup,
                              int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint64_t key = __ldg(q + i);
    int64_t r = -1;
    if ((key & ~valid) == 0)
      r = (lookup == SQD_LOOKUP_BSEARCH) ? bsearch_lookup(states, n_unique, key)
                                         : hash_lookup(hkeys, hvals, hmask, key);
    out[i] = static_cast<int32_t>(r);
  }
}

}  // namespace
}  // namespace sqd

using namespace sqd;

extern "C" int sqd_pack_states(const uint8_t* bits, int64_t n_rows, int num_qubits,
                               uint64_t* out, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(num_qubits >= 1 && num_qubits <= 63, "num_qubits must be in [1, 63]");
    SQD_REQUIRE(n_rows >= 0, "negative row count");
    if (n_rows == 0) return;
    SQD_REQUIRE(bits && out, "NULL array");
    cudaStream_t st = as_stream(stream);
    k_pack<<<grid_for(n_rows, 256, 8192), 256, 0, st>>>(bits, n_rows, num_qubits, out);
    SQD_CHECK_LAUNCH();
  });
}

extern "C" int sqd_space_create(const uint64_t* states, int64_t n_in, int num_qubits,
                                int64_t states_size, void* stream, sqd_space_t* out) {
  return guarded([&] {
    SQD_REQUIRE(out != nullptr, "out handle is NULL");
    *out = nullptr;
    SQD_REQUIRE(num_qubits >= 1 && num_qubits <= 63, "num_qubits must be in [1, 63]");
    SQD_REQUIRE(n_in >= 1, "empty subspace");
    SQD_REQUIRE(n_in < (int64_t(1) << 31), "subspace limited to 2^31 - 1 states");
    SQD_REQUIRE(states != nullptr, "NULL states");
    cudaStream_t st = as_stream(stream);
    auto sp = std::make_unique<sqd_space_s>();
    sp->num_qubits = num_qubits;
    sp->fill_state = (num_qubits == 64) ? ~0ull : ((1ull << num_qubits) - 1ull);

    DevBuf<uint64_t> work;
    work.alloc(n_in, st);
    SQD_CUDA(cudaMemcpyAsync(work.ptr, states, n_in * sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                             st));
    // Reject states with bits above num_qubits: they have no meaning in the padded layout.
    {
      DevBuf<int> stats;
      stats.alloc(6, st);
      int init[6] = {64, 0, 64, 0, 64, 0};
      SQD_CUDA(cudaMemcpyAsync(stats.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
      const uint64_t hi_bits = ~sp->fill_state;
      k_sector_stats<<<grid_for(n_in, 256, 2048), 256, 0, st>>>(work.ptr, n_in, hi_bits, 0, 0,
                                                               stats.ptr);
      SQD_CHECK_LAUNCH();
      int h[6];
      copy_to_host(h, stats.ptr, 6, st);
      SQD_REQUIRE(h[1] == 0, "a state has bits set above num_qubits");
    }
    radix_sort_u64(work.ptr, nullptr, n_in, num_qubits, st);

    DevBuf<int64_t> flags, pos;
    flags.alloc(n_in, st);
    pos.alloc(n_in + 1, st);
    const unsigned G = grid_for(n_in, 256, 8192);
    k_unique_flags<<<G, 256, 0, st>>>(work.ptr, n_in, flags.ptr);
    SQD_CHECK_LAUNCH();
    exclusive_scan_i64(flags.ptr, pos.ptr, n_in, true, st);
    int64_t nu = 0;
    copy_to_host(&nu, pos.ptr + n_in, 1, st);
    SQD_REQUIRE(states_size >= nu, "states_size smaller than the number of unique states");
    sp->n_unique = nu;
    sp->states_size = states_size;
    sp->states.alloc(nu, st);
    k_unique_scatter<<<G, 256, 0, st>>>(work.ptr, flags.ptr, pos.ptr, n_in, sp->states.ptr);
    SQD_CHECK_LAUNCH();

    // Hash table, load factor <= 1/2.
    uint64_t cap = 1024;
    while (cap < 2 * static_cast<uint64_t>(nu)) cap <<= 1;
    sp->hmask = cap - 1;
    sp->hkeys.alloc(cap, st);
    sp->hvals.alloc(cap, st);
    SQD_CUDA(cudaMemsetAsync(sp->hkeys.ptr, 0xff, cap * sizeof(uint64_t), st));
    DevBuf<int> status;
    status.alloc(1, st);
    SQD_CUDA(cudaMemsetAsync(status.ptr, 0, sizeof(int), st));
    k_hash_insert<<<grid_for(nu, 256, 8192), 256, 0, st>>>(sp->states.ptr, nu, sp->hkeys.ptr,
                                                           sp->hvals.ptr, sp->hmask, status.ptr);
    SQD_CHECK_LAUNCH();

    // Conserved-weight sectors.
    const int h = num_qubits / 2;
    const uint64_t m_all = sp->fill_state;
    const uint64_t m_lo = half_mask_low(num_qubits);
    const uint64_t m_hi = m_all & ~m_lo;
    DevBuf<int> stats;
    stats.alloc(6, st);
    int init[6] = {64, 0, 64, 0, 64, 0};
    SQD_CUDA(cudaMemcpyAsync(stats.ptr, init, sizeof(init), cudaMemcpyHostToDevice, st));
    k_sector_stats<<<grid_for(nu, 256, 2048), 256, 0, st>>>(sp->states.ptr, nu, m_all, m_lo, m_hi,
                                                           stats.ptr);
    SQD_CHECK_LAUNCH();
    int hs[6];
    copy_to_host(hs, stats.ptr, 6, st);
    int hstatus = 0;
    copy_to_host(&hstatus, status.ptr, 1, st);
    if (hstatus) throw Error(SQD_ERR_DEVICE, "hash table insertion failed");
    if (h > 0 && hs[2] == hs[3] && hs[4] == hs[5]) {
      sp->num_sectors = 2;
      sp->sector_mask[0] = m_lo;
      sp->sector_mask[1] = m_hi;
      sp->sector_weight[0] = hs[2];
      sp->sector_weight[1] = hs[4];
    } else if (hs[0] == hs[1]) {
      sp->num_sectors = 1;
      sp->sector_mask[0] = m_all;
      sp->sector_weight[0] = hs[0];
    }
    // Sector bitmaps (kept only if at most half full).
    if (sp->num_sectors > 0) {
      const size_t words = (static_cast<size_t>(sp->num_sectors) << kBitmapLog2) / 32;
      sp->bitmap.alloc(words, st);
      SQD_CUDA(cudaMemsetAsync(sp->bitmap.ptr, 0, words * sizeof(uint32_t), st));
      const int sh0 = __builtin_ctzll(sp->sector_mask[0]);
      const int sh1 = sp->num_sectors > 1 ? __builtin_ctzll(sp->sector_mask[1]) : 0;
      const int ex0 = __builtin_popcountll(sp->sector_mask[0]) <= kBitmapLog2;
      const int ex1 = sp->num_sectors > 1 && __builtin_popcountll(sp->sector_mask[1]) <= kBitmapLog2;
      k_bitmap_build<<<grid_for(nu, 256, 4096), 256, 0, st>>>(
          sp->states.ptr, nu, sp->num_sectors, sp->sector_mask[0], sp->sector_mask[1], sh0, sh1,
          ex0, ex1, sp->bitmap.ptr);
      SQD_CHECK_LAUNCH();
      DevBuf<unsigned long long> cnt;
      cnt.alloc(1, st);
      SQD_CUDA(cudaMemsetAsync(cnt.ptr, 0, sizeof(unsigned long long), st));
      k_popc_sum<<<64, 256, 0, st>>>(sp->bitmap.ptr, static_cast<int64_t>(words), cnt.ptr);
      SQD_CHECK_LAUNCH();
      unsigned long long set = 0;
      copy_to_host(&set, cnt.ptr, 1, st);
      if (set > static_cast<unsigned long long>(sp->num_sectors) << (kBitmapLog2 - 1))
        sp->bitmap.release();
    }
    SQD_CUDA(cudaStreamSynchronize(st));
    *out = sp.release();
  });
}

extern "C" int sqd_space_info(sqd_space_t s, int64_t* n_unique, int64_t* states_size,
                              int* num_sectors, uint64_t* sector_masks_host) {
  return guarded([&] {
    SQD_REQUIRE(s != nullptr, "NULL space handle");
    if (n_unique) *n_unique = s->n_unique;
    if (states_size) *states_size = s->states_size;
    if (num_sectors) *num_sectors = s->num_sectors;
    if (sector_masks_host) {
      sector_masks_host[0] = s->sector_mask[0];
      sector_masks_host[1] = s->sector_mask[1];
    }
  });
}

extern "C" int sqd_space_states(sqd_space_t s, uint64_t* out, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(s != nullptr && out != nullptr, "NULL argument");
    SQD_CUDA(cudaMemcpyAsync(out, s->states.ptr, s->states.bytes(), cudaMemcpyDeviceToDevice,
                             as_stream(stream)));
  });
}

extern "C" int sqd_xsource(sqd_space_t s, uint64_t x, int lookup, int32_t* out, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(s != nullptr && out != nullptr, "NULL argument");
    SQD_REQUIRE(lookup == SQD_LOOKUP_HASH || lookup == SQD_LOOKUP_BSEARCH ||
                    lookup == SQD_LOOKUP_AUTO,
                "sqd_xsource takes SQD_LOOKUP_HASH, SQD_LOOKUP_BSEARCH or SQD_LOOKUP_AUTO");
    SQD_REQUIRE((x & ~s->fill_state) == 0, "x has bits above num_qubits");
    cudaStream_t st = as_stream(stream);
    k_xsource<<<grid_for(s->states_size, 256, 8192), 256, 0, st>>>(
        s->states.ptr, s->n_unique, s->states_size, x, s->hkeys.ptr, s->hvals.ptr, s->hmask,
        lookup == SQD_LOOKUP_BSEARCH ? SQD_LOOKUP_BSEARCH : SQD_LOOKUP_HASH, out);
    SQD_CHECK_LAUNCH();
  });
}

extern "C" int sqd_space_lookup(sqd_space_t s, const uint64_t* keys, int64_t n, int lookup,
                                int32_t* out, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(s != nullptr, "NULL space handle");
    SQD_REQUIRE(n >= 0, "negative key count");
    SQD_REQUIRE(n == 0 || (keys != nullptr && out != nullptr), "NULL argument");
    SQD_REQUIRE(lookup == SQD_LOOKUP_HASH || lookup == SQD_LOOKUP_BSEARCH ||
                    lookup == SQD_LOOKUP_AUTO,
                "sqd_space_lookup takes SQD_LOOKUP_HASH, SQD_LOOKUP_BSEARCH or SQD_LOOKUP_AUTO");
    if (n == 0) return;
    cudaStream_t st = as_stream(stream);
    k_lookup_keys<<<grid_for(n, 256, 8192), 256, 0, st>>>(
        keys, n, s->fill_state, s->states.ptr, s->n_unique, s->hkeys.ptr, s->hvals.ptr, s->hmask,
        lookup == SQD_LOOKUP_BSEARCH ? SQD_LOOKUP_BSEARCH : SQD_LOOKUP_HASH, out);
    SQD_CHECK_LAUNCH();
  });
}

extern "C" void sqd_space_destroy(sqd_space_t s) { delete s; }
