// Error reporting and device queries shared by every entry point.
#include <atomic>
#include <cstdarg>
#include <cstring>
#include "common.cuh"

namespace petch {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    return PETCH_E_CUDA;
}

static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

}  // namespace petch

extern "C" int petch_abi_version(void) { return 3; }

extern "C" int petch_launch_count(long long* n) {
    if (!n) {
        petch::set_error("petch_launch_count: null pointer");
        return PETCH_E_INVALID;
    }
    *n = petch::g_launches.load(std::memory_order_relaxed);
    return PETCH_OK;
}

extern "C" int petch_last_error(char* buf, int n) {
    int len = (int)strlen(petch::g_last_error);
    if (buf && n > 0) {
        int m = len < n - 1 ? len : n - 1;
        memcpy(buf, petch::g_last_error, (size_t)m);
        buf[m] = '\0';
    }
    return len;
}
