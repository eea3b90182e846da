// Error reporting, version and launch accounting for the C ABI.
#include <cstdarg>
#include <cstdio>
#include <atomic>

#include "common.cuh"

namespace vx {

static thread_local char g_err[1024] = "";
static std::atomic<unsigned long long> g_launches{0};

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return VX_OK;
}

void count_launches(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

}  // namespace vx

extern "C" {

const char* vx_last_error(void) { return vx::g_err; }

const char* vx_version(void) { return "voxneus_b200 1.0 sm_100a"; }

uint64_t vx_launch_count(void) { return (uint64_t)vx::g_launches.load(std::memory_order_relaxed); }

}
