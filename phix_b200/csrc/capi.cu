// capi.cu -- library-level C ABI: version, per-thread error text, launch
// counter, CUDA status translation.
#include <atomic>
#include <cstdarg>
#include <cstdio>

#include "phix/detail/common.cuh"

namespace phix {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
    set_error("CUDA error in %s: %s", where, cudaGetErrorString(e));
    return PHIX_ERR_CUDA;
}

static thread_local int t_count_paused = 0;

void count_launch(int n) {
    if (!t_count_paused) g_launches.fetch_add(n, std::memory_order_relaxed);
}
LaunchCountPause::LaunchCountPause() { ++t_count_paused; }
LaunchCountPause::~LaunchCountPause() { --t_count_paused; }

}  // namespace phix

extern "C" {

int phix_abi_version(void) { return PHIX_ABI_VERSION; }

const char* phix_last_error(void) { return phix::g_err; }

long long phix_launch_count(void) { return phix::g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
