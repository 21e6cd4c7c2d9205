// The (row, X-group) sweep: for every real row s and every group x that can connect, test
// whether s ^ x is in the subspace.  This is get_xsource (sqd.py:485-548) for all groups at
// once, restricted to the pairs whose source can exist:
//   1. sector filter: a state of the subspace has popcount(s & m_l) == w_l in every conserved
//      sector l, so s ^ x can only be a state if 2 * popcount(s & x & m_l) == popcount(x & m_l);
//   2. sector bitmaps in shared memory: the projection (s ^ x) & m_l must be the projection of
//      some state (no false negatives);
//   3. exact lookup (hash table or binary search) of s ^ x.
// Candidates surviving 1-2 are pushed into a per-warp FIFO in shared memory and looked up 32 at
// a time, so the expensive step runs on full warps.  Candidates of one row enter the FIFO in
// the order of the group list, so COUNT and FILL agree and every row's pairs follow that order
// (the high-sector-only groups first, see k_gpre_flags).
//
// Modes: COUNT (pairs per row), FILL (write (col, group) at the row's CSR slots), APPLY
// (accumulate diag_j(s) * v[src] per row: the uncached matvec, cache_strategy (0, *)).
#pragma once
#include "internal.cuh"

namespace sqd {

constexpr int SW_THREADS = 256;
constexpr int SW_WARPS = SW_THREADS / 32;
constexpr int SW_RPT = 4;
constexpr int SW_TILE = SW_THREADS * SW_RPT;
constexpr int SW_CHUNK = 256;
constexpr int SW_QCAP = 64;

enum SweepMode { SWEEP_COUNT = 0, SWEEP_FILL = 1, SWEEP_APPLY = 2 };

struct SweepParams {
  const uint64_t* states;
  int64_t n_unique;
  const GroupPre* gpre;
  int64_t n_gpre;
  const uint64_t* hkeys;
  const uint32_t* hvals;
  uint64_t hmask;
  int lookup;
  int nsec;
  uint64_t m0, m1;
  int sh0, sh1, ex0, ex1;
  const uint32_t* bitmap;  // NULL = no bitmap filter
  // COUNT
  int64_t* counts;
  // FILL
  const int64_t* row_ptr;
  uint32_t* cols;
  uint32_t* grps;
  int diag_first;
  // APPLY
  const int64_t* group_start;
  const int32_t* group_eff;
  const uint64_t* term_z;
  const double* term_c;
  const void* vin;
  void* vout;
  int has_diag;
};

struct QEntry {
  uint64_t key;
  uint32_t group;
  uint32_t lrow;
};

template <typename R, int NCA>
__device__ __forceinline__ Cx<R> group_diag(const SweepParams& P, int64_t j, uint64_t s) {
  const int64_t b = P.group_start[j];
  const int32_t k = P.group_eff[j];
  R dr = 0, di = 0;
  for (int32_t t = 0; t < k; ++t) {
    const uint64_t z = __ldg(P.term_z + b + t);
    const R sg = parity64(s & z) ? R(-1) : R(1);
    dr += R(__ldg(P.term_c + 2 * (b + t))) * sg;
    if constexpr (NCA == 2) di += R(__ldg(P.term_c + 2 * (b + t) + 1)) * sg;
  }
  return cx_make<R>(dr, di);
}

template <int MODE, typename R, int NCV, int NCA>
__global__ void __launch_bounds__(SW_THREADS)
k_sweep(SweepParams P) {
  extern __shared__ uint32_t sm_bitmap[];
  __shared__ GroupPre sm_groups[SW_CHUNK];
  __shared__ QEntry sm_queue[SW_WARPS][SW_QCAP];
  __shared__ int32_t sm_cnt[SW_TILE];
  __shared__ Cx<R> sm_acc[MODE == SWEEP_APPLY ? SW_TILE : 1];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t tile_base = static_cast<int64_t>(blockIdx.x) * SW_TILE;
  const bool use_bitmap = P.bitmap != nullptr;
  constexpr uint32_t bm_words = (1u << kBitmapLog2) / 32;

  if (use_bitmap) {
    const int words = P.nsec * bm_words;
    for (int w = tid; w < words; w += SW_THREADS) sm_bitmap[w] = P.bitmap[w];
  }

  uint64_t srow[SW_RPT];
  bool valid[SW_RPT];
#pragma unroll
  for (int k = 0; k < SW_RPT; ++k) {
    const int lr = k * SW_THREADS + tid;
    const int64_t r = tile_base + lr;
    valid[k] = r < P.n_unique;
    srow[k] = valid[k] ? __ldg(P.states + r) : 0ull;
    sm_cnt[lr] = 0;
    if constexpr (MODE == SWEEP_APPLY) {
      Cx<R> a = cx_make<R>(0, 0);
      if (valid[k] && P.has_diag) {
        const Cx<R> d = group_diag<R, NCA>(P, 0, srow[k]);
        const Cx<R> x = ld_elem<R, NCV>(static_cast<const R*>(P.vin), r);
        a.re = d.re * x.re - d.im * x.im;
        a.im = d.re * x.im + d.im * x.re;
      }
      sm_acc[lr] = a;
    }
  }

  int head = 0, tail = 0;  // warp-uniform FIFO cursors

  auto process = [&](int count) {
    QEntry e;
    int64_t found = -1;
    if (lane < count) {
      e = sm_queue[warp][(head + lane) & (SW_QCAP - 1)];
      found = (P.lookup == SQD_LOOKUP_BSEARCH) ? bsearch_lookup(P.states, P.n_unique, e.key)
                                               : hash_lookup(P.hkeys, P.hvals, P.hmask, e.key);
    }
    const bool hit = found >= 0;
    if constexpr (MODE == SWEEP_COUNT) {
      if (hit) atomicAdd(&sm_cnt[e.lrow], 1);
    } else if constexpr (MODE == SWEEP_FILL) {
      const unsigned key = hit ? e.lrow : (0x10000u + lane);
      const unsigned peers = __match_any_sync(kFullMask, key);
      const int rank = __popc(peers & lt_mask);
      int base = 0;
      if (hit) base = sm_cnt[e.lrow];
      __syncwarp();
      if (hit) {
        const int64_t row = tile_base + e.lrow;
        const int64_t slot = P.row_ptr[row] + P.diag_first + base + rank;
        P.cols[slot] = static_cast<uint32_t>(found);
        P.grps[slot] = e.group;
        if (rank == __popc(peers) - 1) sm_cnt[e.lrow] = base + __popc(peers);
      }
      __syncwarp();
    } else {
      // APPLY: contributions added to the row accumulator in FIFO (= group) order.
      Cx<R> c = cx_make<R>(0, 0);
      if (hit) {
        const int64_t row = tile_base + e.lrow;
        const uint64_t srow_state = __ldg(P.states + row);
        const Cx<R> d = group_diag<R, NCA>(P, e.group, srow_state);
        const Cx<R> x = ld_elem<R, NCV>(static_cast<const R*>(P.vin), found);
        c.re = d.re * x.re - d.im * x.im;
        c.im = d.re * x.im + d.im * x.re;
      }
      unsigned hits = __ballot_sync(kFullMask, hit);
      while (hits) {
        const int src = __ffs(hits) - 1;
        hits &= hits - 1;
        const unsigned lr = __shfl_sync(kFullMask, e.lrow, src);
        const R cr = __shfl_sync(kFullMask, c.re, src);
        const R ci = __shfl_sync(kFullMask, c.im, src);
        if (lane == 0) {
          sm_acc[lr].re += cr;
          sm_acc[lr].im += ci;
        }
        __syncwarp();
      }
    }
  };

  for (int64_t c0 = 0; c0 < P.n_gpre; c0 += SW_CHUNK) {
    const int64_t left = P.n_gpre - c0;
    const int clen = left < SW_CHUNK ? static_cast<int>(left) : SW_CHUNK;
    __syncthreads();
    for (int g = tid; g < clen; g += SW_THREADS) sm_groups[g] = P.gpre[c0 + g];
    __syncthreads();
    for (int g = 0; g < clen; ++g) {
      const GroupPre gp = sm_groups[g];
      const int cx0 = gp.cx & 0xff, cx1 = (gp.cx >> 8) & 0xff;
#pragma unroll
      for (int k = 0; k < SW_RPT; ++k) {
        const uint64_t cand = srow[k] ^ gp.x;
        bool pass = valid[k];
        if (P.nsec > 0) {
          pass = pass && (2 * __popcll(srow[k] & gp.x & P.m0) == cx0);
          if (P.nsec > 1) pass = pass && (2 * __popcll(srow[k] & gp.x & P.m1) == cx1);
        }
        if (pass && use_bitmap) {
          uint32_t b = sector_bitmap_index(cand & P.m0, P.sh0, P.ex0);
          pass = (sm_bitmap[b >> 5] >> (b & 31)) & 1u;
          if (pass && P.nsec > 1) {
            b = sector_bitmap_index(cand & P.m1, P.sh1, P.ex1);
            pass = (sm_bitmap[bm_words + (b >> 5)] >> (b & 31)) & 1u;
          }
        }
        const unsigned ballot = __ballot_sync(kFullMask, pass);
        if (ballot) {
          if (pass) {
            QEntry q;
            q.key = cand;
            q.group = static_cast<uint32_t>(gp.group);
            q.lrow = static_cast<uint32_t>(k * SW_THREADS + tid);
            sm_queue[warp][(tail + __popc(ballot & lt_mask)) & (SW_QCAP - 1)] = q;
          }
          tail += __popc(ballot);
          __syncwarp();
          if (tail - head >= 32) {
            process(32);
            head += 32;
          }
        }
      }
    }
  }
  while (tail - head > 0) {
    const int cnt = min(32, tail - head);
    __syncwarp();
    process(cnt);
    head += cnt;
  }
  __syncwarp();
  __syncthreads();
#pragma unroll
  for (int k = 0; k < SW_RPT; ++k) {
    const int lr = k * SW_THREADS + tid;
    const int64_t r = tile_base + lr;
    if (!valid[k]) continue;
    if constexpr (MODE == SWEEP_COUNT) {
      P.counts[r] = sm_cnt[lr];
    } else if constexpr (MODE == SWEEP_APPLY) {
      st_elem<R, NCV>(static_cast<R*>(P.vout), r, sm_acc[lr]);
    }
  }
}

}  // namespace sqd
