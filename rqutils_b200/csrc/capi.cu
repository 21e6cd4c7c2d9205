// Library-level C ABI: version string and the per-thread last error message.
#include "common.cuh"

namespace sqd {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace sqd

extern "C" const char* sqd_version(void) { return "sqd_b200 0.1.0 (sm_100a)"; }

extern "C" const char* sqd_last_error(void) { return sqd::g_last_error.c_str(); }
