// Shared helpers for the petch-b200 CUDA library: error reporting, launch checks, grid indexing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include "petch_b200.h"

namespace petch {

// Records a formatted message for petch_last_error() (thread-local, host side).
void set_error(const char* fmt, ...);

// Maps a CUDA error to PETCH_E_CUDA and records "<what>: <cuda message>".
int cuda_fail(cudaError_t e, const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Number of SMs on the current device (cached per device).
int sm_count();

// Kernel launches enqueued by this library since load (read with petch_launch_count).
void count_launch();

// Blocks for a grid-stride kernel: a multiple of the SM count, capped by the work.
inline int grid_for(long long n, int block, int per_sm = 8) {
    long long want = (n + block - 1) / block;
    long long cap = (long long)sm_count() * per_sm;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return (int)want;
}

// The single-instance ion and neutral-pair traces (petch_trace_ions, petch_trace_neutral_pair)
// with the seed read on the device: seed_add + (*step + seed_off) * seed_mul, so that a captured
// etch step takes its seeds from a device step counter (trace.cu).
int trace_ions_stepped(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                       const petch_ion_params* p, const int* step, uint32_t seed_mul,
                       uint32_t seed_off, uint32_t seed_add, int n_ion, float* tally4, float* ang,
                       int* work, void* stream);
int trace_neutral_pair_stepped(const void* mesh, int max_tris, int max_verts,
                               const petch_domain* dom, const float* bare, float beta_a,
                               float beta_b, const int* step, uint32_t seed_mul, uint32_t seed_off,
                               uint32_t seed_add_a, uint32_t seed_add_b, uint32_t stream_id,
                               int n_neu, float* flux_a, float* flux_b, int* work, void* stream);

}  // namespace petch

#define PETCH_LAUNCH_CHECK(what)                                   \
    do {                                                           \
        petch::count_launch();                                     \
        cudaError_t _e = cudaGetLastError();                       \
        if (_e != cudaSuccess) return petch::cuda_fail(_e, what);  \
    } while (0)

#define PETCH_CUDA(call, what)                                     \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return petch::cuda_fail(_e, what);  \
    } while (0)

#define PETCH_REQUIRE(cond, ...)                                   \
    do {                                                           \
        if (!(cond)) {                                             \
            petch::set_error(__VA_ARGS__);                         \
            return PETCH_E_INVALID;                                \
        }                                                          \
    } while (0)
