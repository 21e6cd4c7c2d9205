// Library-level C ABI: version string, the per-thread last error message, and the library's
// device memory pools.
#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace sqd {
namespace {
thread_local std::string g_last_error;
constexpr int kMaxDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pools[kMaxDevices] = {};
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }

cudaMemPool_t library_pool() {
  int dev = 0;
  SQD_CUDA(cudaGetDevice(&dev));
  SQD_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    SQD_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t threshold = UINT64_MAX;
    SQD_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    g_pools[dev] = pool;
  }
  return g_pools[dev];
}
}  // namespace sqd

extern "C" int sqd_trim_memory(uint64_t keep_bytes) {
  return sqd::guarded([&] {
    SQD_CUDA(cudaDeviceSynchronize());
    SQD_CUDA(cudaMemPoolTrimTo(sqd::library_pool(), static_cast<size_t>(keep_bytes)));
  });
}

extern "C" int sqd_memory_stats(uint64_t* reserved_host, uint64_t* used_host,
                                uint64_t* used_high_host, int reset_high) {
  return sqd::guarded([&] {
    cudaMemPool_t pool = sqd::library_pool();
    uint64_t v = 0;
    if (reset_high) {
      uint64_t zero = 0;      // resets the high-water mark to the current usage
      SQD_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero));
    }
    if (reserved_host) {
      SQD_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
      *reserved_host = v;
    }
    if (used_host) {
      SQD_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &v));
      *used_host = v;
    }
    if (used_high_host) {
      SQD_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &v));
      *used_high_host = v;
    }
  });
}

extern "C" const char* sqd_version(void) { return "sqd_b200 0.1.0 (sm_100a)"; }

extern "C" const char* sqd_last_error(void) { return sqd::g_last_error.c_str(); }
