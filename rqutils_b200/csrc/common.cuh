// Shared helpers for the SQD sm_100a library: status handling, stream-ordered allocation,
// complex arithmetic on interleaved (re, im) pairs, warp reductions and popcount parity.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <memory>
#include <string>
#include <vector>
#include <stdexcept>

#include "../../include/sqd_b200.h"

namespace sqd {

// ------------------------------------------------------------------------------------------
// Errors.  Internal code throws sqd::Error; every extern "C" entry point catches and converts
// it to a status code plus a thread-local message.
// ------------------------------------------------------------------------------------------
struct Error : public std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);

#define SQD_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t err__ = (call);                                                         \
    if (err__ != cudaSuccess)                                                           \
      throw ::sqd::Error(SQD_ERR_CUDA, std::string(#call) + ": " +                      \
                                           cudaGetErrorString(err__) + " (" __FILE__ ")"); \
  } while (0)

#define SQD_CHECK_LAUNCH() SQD_CUDA(cudaGetLastError())

#define SQD_REQUIRE(cond, msg)                                        \
  do {                                                                \
    if (!(cond)) throw ::sqd::Error(SQD_ERR_INVALID, (msg));          \
  } while (0)

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SQD_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return SQD_ERR_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SQD_ERR_INVALID;
  }
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ------------------------------------------------------------------------------------------
// Stream-ordered device buffers, allocated from a library-owned memory pool per device that
// keeps freed memory for reuse (release threshold = unlimited); sqd_trim_memory returns it.
// ------------------------------------------------------------------------------------------
cudaMemPool_t library_pool();

template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  cudaStream_t stream = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { swap(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    swap(o);
    return *this;
  }
  ~DevBuf() { release(); }
  void swap(DevBuf& o) {
    std::swap(ptr, o.ptr);
    std::swap(count, o.count);
    std::swap(stream, o.stream);
  }
  void alloc(size_t n, cudaStream_t s) {
    release();
    stream = s;
    count = n;
    if (n == 0) return;
    cudaError_t err =
        cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ptr), n * sizeof(T), library_pool(), s);
    if (err != cudaSuccess) {
      ptr = nullptr;
      count = 0;
      throw Error(SQD_ERR_MEMORY, std::string("device allocation of ") +
                                      std::to_string(n * sizeof(T)) + " bytes failed: " +
                                      cudaGetErrorString(err));
    }
  }
  void release() {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    count = 0;
  }
  size_t bytes() const { return count * sizeof(T); }
};

// ------------------------------------------------------------------------------------------
// Device helpers.
// ------------------------------------------------------------------------------------------
constexpr uint64_t kEmptyKey = ~0ull;
constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ int parity64(uint64_t v) {
  return __popc(static_cast<unsigned>(v) ^ static_cast<unsigned>(v >> 32)) & 1;
}

// MurmurHash3 64-bit finalizer (Austin Appleby, public domain).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

template <typename R>
struct Cx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ Cx<R> cx_make(R a, R b) {
  Cx<R> c;
  c.re = a;
  c.im = b;
  return c;
}

// Vector element load/store: NC = 1 (real) or 2 (interleaved complex).
template <typename R, int NC>
__device__ __forceinline__ Cx<R> ld_elem(const R* p, int64_t i) {
  if constexpr (NC == 2) {
    if constexpr (sizeof(R) == 8) {
      double2 v = __ldg(reinterpret_cast<const double2*>(p) + i);
      return cx_make<R>(v.x, v.y);
    } else {
      float2 v = __ldg(reinterpret_cast<const float2*>(p) + i);
      return cx_make<R>(v.x, v.y);
    }
  } else {
    return cx_make<R>(__ldg(p + i), R(0));
  }
}

// Plain (coherent) load, for buffers written earlier in the same kernel sequence on-device.
// Load through L2 only (ld.global.cg): for data written earlier in the same kernel launch by
// other thread blocks, which a non-coherent L1 copy could shadow.
template <typename R, int NC>
__device__ __forceinline__ Cx<R> ld_elem_cg(const R* p, int64_t i) {
  if constexpr (NC == 2) {
    if constexpr (sizeof(R) == 8) {
      const double2 v = __ldcg(reinterpret_cast<const double2*>(p) + i);
      return cx_make<R>(v.x, v.y);
    } else {
      const float2 v = __ldcg(reinterpret_cast<const float2*>(p) + i);
      return cx_make<R>(v.x, v.y);
    }
  } else {
    return cx_make<R>(__ldcg(p + i), R(0));
  }
}

template <typename R, int NC>
__device__ __forceinline__ Cx<R> ld_elem_rw(const R* p, int64_t i) {
  if constexpr (NC == 2) {
    if constexpr (sizeof(R) == 8) {
      double2 v = reinterpret_cast<const double2*>(p)[i];
      return cx_make<R>(v.x, v.y);
    } else {
      float2 v = reinterpret_cast<const float2*>(p)[i];
      return cx_make<R>(v.x, v.y);
    }
  } else {
    return cx_make<R>(p[i], R(0));
  }
}

template <typename R, int NC>
__device__ __forceinline__ void st_elem(R* p, int64_t i, Cx<R> v) {
  if constexpr (NC == 2) {
    if constexpr (sizeof(R) == 8) {
      reinterpret_cast<double2*>(p)[i] = make_double2(v.re, v.im);
    } else {
      reinterpret_cast<float2*>(p)[i] = make_float2(v.re, v.im);
    }
  } else {
    p[i] = v.re;
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFullMask, v, o);
  return v;
}

inline int dtype_is_complex(int dtype) { return dtype == SQD_C128 || dtype == SQD_C64; }
inline int dtype_is_double(int dtype) { return dtype == SQD_F64 || dtype == SQD_C128; }
inline size_t dtype_size(int dtype) {
  switch (dtype) {
    case SQD_F64: return 8;
    case SQD_C128: return 16;
    case SQD_F32: return 4;
    case SQD_C64: return 8;
  }
  throw Error(SQD_ERR_INVALID, "unknown dtype");
}

inline int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    SQD_CUDA(cudaGetDevice(&dev));
    SQD_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

inline unsigned grid_for(int64_t n, int block, int64_t cap = 0) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (cap > 0 && g > cap) g = cap;
  return static_cast<unsigned>(g);
}

// ------------------------------------------------------------------------------------------
// Primitives implemented in primitives.cu.
// ------------------------------------------------------------------------------------------
// Exclusive scan of n int64 values (in may alias out); returns nothing, total at out[n] if
// out has n+1 slots and write_total is set.
void exclusive_scan_i64(const int64_t* in, int64_t* out, int64_t n, bool write_total,
                        cudaStream_t s);
void exclusive_scan_i32(const int32_t* in, int32_t* out, int64_t n, bool write_total,
                        cudaStream_t s);

// Stable LSD radix sort of uint64 keys on bits [0, key_bits), with an optional uint32 payload.
// keys/vals are sorted in place (temporary double buffers are allocated on s).
void radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s);
// Stable sort by the 2-word key (hi, lo) with payload; bits give the significant widths.
void radix_sort_pair(uint64_t* hi, uint64_t* lo, uint32_t* vals, int64_t n, int hi_bits,
                     int lo_bits, cudaStream_t s);

template <typename T>
inline void copy_to_host(T* dst, const T* src, size_t count, cudaStream_t s) {
  if (count == 0) return;
  SQD_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToHost, s));
  SQD_CUDA(cudaStreamSynchronize(s));
}

}  // namespace sqd
