// Device-wide primitives used during setup: exclusive scans and a stable LSD radix sort.
//
// Radix sort: one 8-bit digit per pass, three kernels per pass (tile histogram, scan of the
// digit-major histogram, stable scatter).  The scatter ranks equal digits inside a tile with
// __match_any_sync per warp plus per-warp digit counts in shared memory, so the order of equal
// keys is preserved across passes (LSD correctness).
#include "common.cuh"

namespace sqd {

namespace {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_IPT = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_IPT;

template <typename T>
__device__ T block_exclusive_scan(T v, T* total) {
  __shared__ T warp_tot[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(kFullMask, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < SCAN_THREADS / 32 ? warp_tot[lane] : T(0);
    T winc = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(kFullMask, winc, o);
      if (lane >= o) winc += y;
    }
    if (lane < SCAN_THREADS / 32) warp_tot[lane] = winc - w;
    if (lane == SCAN_THREADS / 32 - 1) *total = winc;
  }
  __syncthreads();
  T res = inc - v + warp_tot[warp];
  __syncthreads();
  return res;
}

template <typename T>
__global__ void scan_tile_sums(const T* in, int64_t n, T* sums) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * SCAN_TILE;
  T acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    int64_t idx = base + static_cast<int64_t>(threadIdx.x) * SCAN_IPT + i;
    if (idx < n) acc += in[idx];
  }
  __shared__ T tot;
  block_exclusive_scan<T>(acc, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <typename T>
__global__ void scan_tiles(const T* in, T* out, int64_t n, const T* tile_offsets) {
  const int64_t base = static_cast<int64_t>(blockIdx.x) * SCAN_TILE;
  T vals[SCAN_IPT];
  T acc = 0;
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    int64_t idx = base + static_cast<int64_t>(threadIdx.x) * SCAN_IPT + i;
    vals[i] = idx < n ? in[idx] : T(0);
    acc += vals[i];
  }
  __shared__ T tot;
  T pre = block_exclusive_scan<T>(acc, &tot);
  pre += tile_offsets ? tile_offsets[blockIdx.x] : T(0);
#pragma unroll
  for (int i = 0; i < SCAN_IPT; ++i) {
    int64_t idx = base + static_cast<int64_t>(threadIdx.x) * SCAN_IPT + i;
    if (idx < n) out[idx] = pre;
    pre += vals[i];
  }
}

template <typename T>
__global__ void write_total(const T* in_last, const T* out_last, T* dst) {
  *dst = *in_last + *out_last;
}

template <typename T>
void exclusive_scan(const T* in, T* out, int64_t n, bool total, cudaStream_t s) {
  if (n <= 0) {
    if (total) SQD_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
    return;
  }
  // The last input is needed for the total; save it before an in-place scan overwrites it.
  DevBuf<T> last;
  if (total) {
    last.alloc(1, s);
    SQD_CUDA(cudaMemcpyAsync(last.ptr, in + n - 1, sizeof(T), cudaMemcpyDeviceToDevice, s));
  }
  const int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (tiles == 1) {
    scan_tiles<T><<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr);
    SQD_CHECK_LAUNCH();
  } else {
    DevBuf<T> sums;
    sums.alloc(tiles, s);
    scan_tile_sums<T><<<static_cast<unsigned>(tiles), SCAN_THREADS, 0, s>>>(in, n, sums.ptr);
    SQD_CHECK_LAUNCH();
    exclusive_scan<T>(sums.ptr, sums.ptr, tiles, false, s);
    scan_tiles<T><<<static_cast<unsigned>(tiles), SCAN_THREADS, 0, s>>>(in, out, n, sums.ptr);
    SQD_CHECK_LAUNCH();
  }
  if (total) {
    write_total<T><<<1, 1, 0, s>>>(last.ptr, out + n - 1, out + n);
    SQD_CHECK_LAUNCH();
  }
}

// ---------------------------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_IPT = 8;
constexpr int RS_TILE = RS_THREADS * RS_IPT;
constexpr int RS_WARPS = RS_THREADS / 32;

__global__ void rs_hist(const uint64_t* __restrict__ dkey, int64_t n, int shift,
                        int32_t* __restrict__ hist, int num_tiles) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = static_cast<int64_t>(blockIdx.x) * RS_TILE;
#pragma unroll
  for (int i = 0; i < RS_IPT; ++i) {
    int64_t idx = base + i * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&h[(dkey[idx] >> shift) & 255], 1);
  }
  __syncthreads();
  hist[static_cast<int64_t>(threadIdx.x) * num_tiles + blockIdx.x] = h[threadIdx.x];
}

template <bool TWO, bool VALS>
__global__ void rs_scatter(const uint64_t* __restrict__ dkey, const uint64_t* __restrict__ a_in,
                           const uint64_t* __restrict__ b_in, const uint32_t* __restrict__ v_in,
                           uint64_t* __restrict__ a_out, uint64_t* __restrict__ b_out,
                           uint32_t* __restrict__ v_out, int64_t n, int shift,
                           const int32_t* __restrict__ offs, int num_tiles) {
  __shared__ int running[256];
  __shared__ int cnt[RS_WARPS][257];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  running[tid] = offs[static_cast<int64_t>(tid) * num_tiles + blockIdx.x];
  const unsigned lt_mask = (1u << lane) - 1u;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * RS_TILE;
  for (int r = 0; r < RS_IPT; ++r) {
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) cnt[w][tid] = 0;
    __syncthreads();
    const int64_t idx = base + r * RS_THREADS + tid;
    const bool valid = idx < n;
    const int d = valid ? static_cast<int>((dkey[idx] >> shift) & 255) : 256;
    const unsigned peers = __match_any_sync(kFullMask, d);
    const int rank = __popc(peers & lt_mask);
    if (rank == 0) cnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pos = running[d] + rank;
      for (int w = 0; w < warp; ++w) pos += cnt[w][d];
      a_out[pos] = a_in[idx];
      if constexpr (TWO) b_out[pos] = b_in[idx];
      if constexpr (VALS) v_out[pos] = v_in[idx];
    }
    __syncthreads();
    int add = 0;
#pragma unroll
    for (int w = 0; w < RS_WARPS; ++w) add += cnt[w][tid];
    running[tid] += add;
    __syncthreads();
  }
}

// One pass: digit from `dkey` (either a or b) at `shift`.
template <bool TWO, bool VALS>
void rs_pass(const uint64_t* dkey, const uint64_t* a_in, const uint64_t* b_in,
             const uint32_t* v_in, uint64_t* a_out, uint64_t* b_out, uint32_t* v_out, int64_t n,
             int shift, int32_t* hist, int num_tiles, cudaStream_t s) {
  rs_hist<<<num_tiles, RS_THREADS, 0, s>>>(dkey, n, shift, hist, num_tiles);
  SQD_CHECK_LAUNCH();
  exclusive_scan<int32_t>(hist, hist, static_cast<int64_t>(num_tiles) * 256, false, s);
  rs_scatter<TWO, VALS><<<num_tiles, RS_THREADS, 0, s>>>(dkey, a_in, b_in, v_in, a_out, b_out,
                                                         v_out, n, shift, hist, num_tiles);
  SQD_CHECK_LAUNCH();
}

}  // namespace

void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, bool write_total,
                        cudaStream_t s) {
  exclusive_scan<int64_t>(in, out, n, write_total, s);
}

void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, bool write_total,
                        cudaStream_t s) {
  exclusive_scan<int32_t>(in, out, n, write_total, s);
}

void radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s) {
  if (n <= 1 || key_bits <= 0) return;
  SQD_REQUIRE(n < (int64_t(1) << 31), "radix sort supports fewer than 2^31 items");
  const int num_tiles = static_cast<int>((n + RS_TILE - 1) / RS_TILE);
  const int passes = (key_bits + 7) / 8;
  DevBuf<uint64_t> ka;
  DevBuf<uint32_t> va;
  DevBuf<int32_t> hist;
  ka.alloc(n, s);
  if (vals) va.alloc(n, s);
  hist.alloc(static_cast<size_t>(num_tiles) * 256, s);
  uint64_t *kin = keys, *kout = ka.ptr;
  uint32_t *vin = vals, *vout = va.ptr;
  for (int p = 0; p < passes; ++p) {
    if (vals)
      rs_pass<false, true>(kin, kin, nullptr, vin, kout, nullptr, vout, n, 8 * p, hist.ptr,
                           num_tiles, s);
    else
      rs_pass<false, false>(kin, kin, nullptr, nullptr, kout, nullptr, nullptr, n, 8 * p,
                            hist.ptr, num_tiles, s);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {
    SQD_CUDA(cudaMemcpyAsync(keys, kin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    if (vals)
      SQD_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
}

void radix_sort_pair(uint64_t* hi, uint64_t* lo, uint32_t* vals, int64_t n, int hi_bits,
                     int lo_bits, cudaStream_t s) {
  if (n <= 1) return;
  SQD_REQUIRE(vals != nullptr, "radix_sort_pair needs a payload");
  SQD_REQUIRE(n < (int64_t(1) << 31), "radix sort supports fewer than 2^31 items");
  const int num_tiles = static_cast<int>((n + RS_TILE - 1) / RS_TILE);
  DevBuf<uint64_t> ha, la;
  DevBuf<uint32_t> va;
  DevBuf<int32_t> hist;
  ha.alloc(n, s);
  la.alloc(n, s);
  va.alloc(n, s);
  hist.alloc(static_cast<size_t>(num_tiles) * 256, s);
  uint64_t *hin = hi, *hout = ha.ptr, *lin = lo, *lout = la.ptr;
  uint32_t *vin = vals, *vout = va.ptr;
  const int lo_passes = (lo_bits + 7) / 8, hi_passes = (hi_bits + 7) / 8;
  for (int p = 0; p < lo_passes + hi_passes; ++p) {
    const bool on_lo = p < lo_passes;
    const int shift = 8 * (on_lo ? p : p - lo_passes);
    rs_pass<true, true>(on_lo ? lin : hin, hin, lin, vin, hout, lout, vout, n, shift, hist.ptr,
                        num_tiles, s);
    std::swap(hin, hout);
    std::swap(lin, lout);
    std::swap(vin, vout);
  }
  if (hin != hi) {
    SQD_CUDA(cudaMemcpyAsync(hi, hin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    SQD_CUDA(cudaMemcpyAsync(lo, lin, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    SQD_CUDA(cudaMemcpyAsync(vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
}

}  // namespace sqd
