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

int& tile_slots() {
  thread_local int slots = 6;
  return slots;
}

namespace {
LaunchShape g_shape;
}
const LaunchShape& launch_shape() { return g_shape; }
LaunchShape& launch_shape_mut() { return g_shape; }
}  // namespace fv3b

extern "C" const char* fv3b_last_error(void) { return g_last_error; }
// Thread-block shapes of the box kernels (box_x * box_y threads, box_x a
// multiple of 32) and of the column kernels (col threads, a multiple of 32).
// Process-wide; set it between calls, not while kernels of this library are
// being enqueued from another thread.
extern "C" int fv3b_set_launch_shape(int box_x, int box_y, int col) {
  FV3B_REQUIRE(box_x >= 32 && box_x % 32 == 0 && box_y >= 1 && box_x * box_y <= 1024,
               "fv3b_set_launch_shape: box_x must be a multiple of 32 and box_x*box_y <= 1024");
  FV3B_REQUIRE(col >= 32 && col % 32 == 0 && col <= 1024, "fv3b_set_launch_shape: col must be 32..1024, multiple of 32");
  fv3b::LaunchShape& ls = fv3b::launch_shape_mut();
  ls.box_x = box_x;
  ls.box_y = box_y;
  ls.col = col;
  return FV3B_OK;
}

extern "C" void fv3b_get_launch_shape(int* box_x, int* box_y, int* col) {
  const fv3b::LaunchShape& ls = fv3b::launch_shape();
  if (box_x) *box_x = ls.box_x;
  if (box_y) *box_y = ls.box_y;
  if (col) *col = ls.col;
}

// Kernel launches issued by this library since it was loaded.
extern "C" long long fv3b_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" const char* fv3b_version(void) { return "fv3core_b200 0.1.0 sm_100a"; }
