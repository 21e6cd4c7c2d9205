// sqd_vinit_noalloc: the start-index search of sqd_vinit (argmin of the real group-0 diagonal
// over the real rows) without any device allocation.
//
// Why it exists: sqd_vinit allocates its per-warp partial results with cudaMallocAsync on
// every call.  Some callers cannot allocate device memory at that point — a process whose
// device memory is fully reserved by its own caching allocator or arena (a new allocation
// fails there), or one that must not take the allocator's slow paths inside a latency-bound
// loop.  This entry point keeps its partial results in a file-scope __device__ array of fixed
// size instead.
//
// Contract:
//  * Scratch: one static array of kNaMaxBlocks (key, index) pairs plus the result slot,
//    256 KiB + 8 bytes, present in every GPU context that loads this library until the process
//    exits.  Each call writes every slot it later reads, so nothing needs clearing, but the
//    array keeps the last call's contents.
//  * Limit: at most kNaMaxRows = 67,108,864 real rows (one slot per 4096 rows); larger
//    subspaces are rejected with SQD_ERR_INVALID and a message naming the limit.
//  * All calls on a device share the array: calls whose GPU work overlaps (different streams,
//    or several host threads) race and must be serialised by the caller.
//  * Set-up: the first call on each device resolves the array's device address with
//    cudaGetSymbolAddress (with that device current) and keeps it for the process; make that
//    first call before any stream capture begins.  After cudaDeviceReset the kept address
//    belongs to the destroyed context, so the function must not be used on that device again.
//  * No cudaMalloc / cudaFree / allocating library call; every call synchronises `stream` and
//    returns the index to the host.
#include <mutex>

#include "internal.cuh"

namespace sqd {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaRowsPerThread = 16;
constexpr int64_t kNaRowsPerBlock = int64_t(kNaThreads) * kNaRowsPerThread;  // 4096
constexpr int kNaMaxBlocks = 16384;
constexpr int64_t kNaMaxRows = kNaRowsPerBlock * kNaMaxBlocks;              // 67,108,864
constexpr int kNaMaxDevices = 64;

struct NaScratch {
  unsigned long long key[kNaMaxBlocks];
  long long idx[kNaMaxBlocks];
  long long result;
};

static __device__ __align__(256) NaScratch g_vinit_scratch;

// Group-0 diagonal at state s, real part, term by term in the reference's order
// (get_diagonal, sqd.py:603-628).
__device__ __forceinline__ double na_diag0(const int64_t* gs, const int32_t* ge,
                                           const uint64_t* tz, const double* tc, uint64_t s) {
  const int64_t b = gs[0];
  const int32_t k = ge[0];
  double d = 0.0;
  for (int32_t t = 0; t < k; ++t) {
    const double c = tc[2 * (b + t)];
    d = d + (parity64(s & tz[b + t]) ? -c : c);
  }
  return d;
}

// Order-preserving map of a double onto unsigned integers; -0.0 maps like +0.0, so the two
// tie and the smaller row index wins, as in jnp.argmin (sqd.py:413).
__device__ __forceinline__ unsigned long long na_key(double v) {
  if (v == 0.0) v = 0.0;
  const unsigned long long b = __double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ void na_pick(unsigned long long& bk, long long& bi,
                                        unsigned long long k, long long i) {
  if (k < bk || (k == bk && i < bi)) {
    bk = k;
    bi = i;
  }
}

__global__ void __launch_bounds__(kNaThreads)
k_na_partial(const uint64_t* __restrict__ states, int64_t n, const int64_t* gs,
             const int32_t* ge, const uint64_t* tz, const double* tc, NaScratch* scr) {
  __shared__ unsigned long long sk[kNaThreads / 32];
  __shared__ long long si[kNaThreads / 32];
  unsigned long long bk = ~0ull;
  long long bi = 0x7fffffffffffffffll;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * kNaRowsPerBlock;
  for (int k = 0; k < kNaRowsPerThread; ++k) {
    const int64_t r = base + static_cast<int64_t>(k) * kNaThreads + threadIdx.x;
    if (r < n) na_pick(bk, bi, na_key(na_diag0(gs, ge, tz, tc, states[r])), r);
  }
  for (int o = 16; o > 0; o >>= 1)
    na_pick(bk, bi, __shfl_xor_sync(kFullMask, bk, o), __shfl_xor_sync(kFullMask, bi, o));
  if ((threadIdx.x & 31) == 0) {
    sk[threadIdx.x >> 5] = bk;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kNaThreads / 32; ++w) na_pick(bk, bi, sk[w], si[w]);
    scr->key[blockIdx.x] = bk;
    scr->idx[blockIdx.x] = bi;
  }
}

__global__ void __launch_bounds__(1024) k_na_final(NaScratch* scr, int nblocks) {
  __shared__ unsigned long long sk[32];
  __shared__ long long si[32];
  unsigned long long bk = ~0ull;
  long long bi = 0x7fffffffffffffffll;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) na_pick(bk, bi, scr->key[b], scr->idx[b]);
  for (int o = 16; o > 0; o >>= 1)
    na_pick(bk, bi, __shfl_xor_sync(kFullMask, bk, o), __shfl_xor_sync(kFullMask, bi, o));
  if ((threadIdx.x & 31) == 0) {
    sk[threadIdx.x >> 5] = bk;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) na_pick(bk, bi, sk[w], si[w]);
    scr->result = bi;
  }
}

// Device address of g_vinit_scratch for the current device (resolved once per device).
NaScratch* na_scratch_address() {
  static std::mutex mu;
  static NaScratch* addr[kNaMaxDevices] = {};
  int dev = 0;
  SQD_CUDA(cudaGetDevice(&dev));
  SQD_REQUIRE(dev >= 0 && dev < kNaMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (addr[dev] == nullptr) {
    void* p = nullptr;
    SQD_CUDA(cudaGetSymbolAddress(&p, g_vinit_scratch));
    addr[dev] = static_cast<NaScratch*>(p);
  }
  return addr[dev];
}

}  // namespace
}  // namespace sqd

using namespace sqd;

extern "C" int sqd_vinit_noalloc(sqd_op_t op, int64_t* index_host, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(op != nullptr && index_host != nullptr, "NULL argument");
    if (!op->has_diag_group) {
      *index_host = 0;
      return;
    }
    const sqd_paulis_s* p = op->p;
    const sqd_space_s* sp = op->s;
    const int64_t n = sp->n_unique;
    if (n > kNaMaxRows)
      throw Error(SQD_ERR_INVALID,
                  "sqd_vinit_noalloc: the subspace has " + std::to_string(n) +
                      " states, above its limit of 67108864 (fixed scratch of 16384 slots); "
                      "use sqd_vinit");
    NaScratch* scr = na_scratch_address();
    cudaStream_t st = as_stream(stream);
    const int nblocks = static_cast<int>((n + kNaRowsPerBlock - 1) / kNaRowsPerBlock);
    k_na_partial<<<nblocks, kNaThreads, 0, st>>>(sp->states.ptr, n, p->group_start.ptr,
                                                 p->group_eff.ptr, p->term_z.ptr, p->term_c.ptr,
                                                 scr);
    SQD_CHECK_LAUNCH();
    k_na_final<<<1, 1024, 0, st>>>(scr, nblocks);
    SQD_CHECK_LAUNCH();
    long long h = 0;
    SQD_CUDA(cudaMemcpyAsync(&h, &scr->result, sizeof(h), cudaMemcpyDeviceToHost, st));
    SQD_CUDA(cudaStreamSynchronize(st));
    *index_host = h;
  });
}
