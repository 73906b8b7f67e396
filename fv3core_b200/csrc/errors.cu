// Last-error bookkeeping for the C ABI (thread-local, no allocation) and
// the launch counter.
#include <stdio.h>
#include <string.h>

#include <atomic>

#include "common.cuh"

namespace {
thread_local char g_last_error[512] = "";
std::atomic<long long> g_launches{0};
}

namespace fv3b {
void set_last_error(const char* where, cudaError_t e) {
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s)", where, cudaGetErrorName(e),
           cudaGetErrorString(e));
}
void set_last_error_msg(const char* msg) { snprintf(g_last_error, sizeof(g_last_error), "%s", msg); }
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace fv3b

extern "C" const char* fv3b_last_error(void) { return g_last_error; }
// Kernel launches issued by this library since it was loaded.
extern "C" long long fv3b_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" const char* fv3b_version(void) { return "fv3core_b200 0.1.0 sm_100a"; }
