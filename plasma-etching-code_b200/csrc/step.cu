// The fused etch step: one C call per step of run_etch_3d's coverage-coupled Monte-Carlo loop
// (petch/threed.py:1671-1792 with mc_flux_3d_coupled, threed.py:740-905), on a workspace the
// library allocates once (petch_plan) and frees (petch_destroy).
//
// A step issues only stream-ordered work: no host synchronisation, no allocation, no host
// reads.  Everything that varies from step to step lives on the device -- the Philox seeds come
// from a device step counter, the CFL substep count from the device's max surface velocity (the
// advection runs a fixed sequence of 160 substep launches, each gated on the device count), error
// bits accumulate in device words -- so a caller may capture steps into a CUDA graph and replay
// them.  The warm-started coverage alternates between two mesh / coverage buffers (the previous
// step's mesh is the warm start's source), so one captured graph covers two consecutive steps,
// and the first (cold) step, with its four coverage rounds, is a separate capture.
//
// The stages are the library's own entry points, called in the order run_etch_3d calls them
// (forms that read the seed or the substep count from the device where those vary by step), so
// a plan's steps equal run_etch_3d's bit for bit with deterministic tallies.
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <nvtx3/nvToolsExt.h>
#include "common.cuh"
#include "mesh.cuh"

namespace petch {
namespace {

// Plan workspaces come from a memory pool of the library's own, one per device, that keeps up to
// kPoolKeep bytes of freed workspace for the next plan: a caller that plans once per run (as
// run_etch_3d does) then pays cudaMalloc's and cudaFree's device-wide synchronisation once, not
// per run.  Freed memory above the threshold goes back to the driver at the next
// synchronisation.
constexpr unsigned long long kPoolKeep = 8ULL << 30;

int plan_pool(cudaMemPool_t* out) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    PETCH_CUDA(cudaGetDevice(&dev), "petch_plan: cudaGetDevice");
    PETCH_REQUIRE(dev >= 0 && dev < 64, "petch_plan: device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        PETCH_CUDA(cudaMemPoolCreate(&pool, &props), "petch_plan: cudaMemPoolCreate");
        unsigned long long keep = kPoolKeep;
        PETCH_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep),
                   "petch_plan: pool release threshold");
        pools[dev] = pool;
    }
    *out = pools[dev];
    return PETCH_OK;
}

// Device words of a plan (int32): [0..5] the tracers' work words (ray counter, error bits,
// uint64 queries, uint64 visits), [6..7] surface-rate stats (non-finite count, max V bits),
// [8] band cells listed for the advection, [9..10] CFL substeps and dt bits, [11] step counter,
// [12] tracer error bits OR-ed over steps, [13] mesh error bits OR-ed over steps, [14]
// non-finite velocities summed over steps, [15] largest face count seen, [16..17] uint64
// BVH queries summed over steps, [18] the last step's face count, [19] the last step's substeps,
// [20] held: this step's mesh outgrew the capacity, so the level set stays as it was, [21] the
// largest substep count seen.
constexpr int W_WORK = 0, W_STATS = 6, W_NACTIVE = 8, W_SUB = 9, W_STEP = 11, W_TERR = 12,
              W_MERR = 13, W_NONFINITE = 14, W_FMAX = 15, W_QUERIES = 16, W_F = 18, W_NSUB = 19,
              W_HOLD = 20, W_NSUBMAX = 21, W_COUNT = 22;
constexpr int kPerStepWords = 11;   // [0, 11) are reset at the start of each step

__global__ void k_fill(float* a, int n, float v) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// The mask cells of the domain (their order does not matter: each is pinned on its own).
__global__ void k_mask_list(const uint8_t* mask, long long n, int* idx, int* count) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x)
        if (mask[c]) idx[atomicAdd(count, 1)] = (int)c;
}

// A mesh that outgrew its buffers (face / vertex overflow, hash table full) holds the step: the
// advection and reinit leave the level set unchanged and the step counter stays, so the host can
// plan again with more capacity and repeat the step.
__global__ void k_hold(int* w, const int* hdr) {
    if (threadIdx.x == 0 && blockIdx.x == 0) w[W_HOLD] = (hdr[HDR_ERR] & 7) != 0;
}

// Fold one step's status into the plan's accumulated words and advance the step counter.
__global__ void k_accumulate(int* w, const int* hdr) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (!w[W_HOLD]) w[W_STEP] += 1;
    w[W_TERR] |= w[W_WORK + 1];
    w[W_MERR] |= hdr[HDR_ERR];
    w[W_NONFINITE] += w[W_STATS];
    w[W_FMAX] = max(w[W_FMAX], hdr[HDR_F]);
    w[W_F] = hdr[HDR_F];
    w[W_NSUB] = w[W_SUB];
    w[W_NSUBMAX] = max(w[W_NSUBMAX], w[W_SUB]);
    unsigned long long* q = reinterpret_cast<unsigned long long*>(w + W_QUERIES);
    *q += *reinterpret_cast<const unsigned long long*>(w + W_WORK + 2);
}

// Records a timing event on st: a plain record, or an external event node when st is being
// captured into a graph (so that every replay records it).
cudaError_t record_timing_event(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    return cs == cudaStreamCaptureStatusActive
               ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
               : cudaEventRecord(ev, st);
}

}  // namespace
}  // namespace petch

using namespace petch;

struct petch_plan_s {
    petch_step_config cfg;
    int MT, MV;
    long long ncell;
    float* phi;                     // caller-owned level set (in / out)
    void* mesh[2];
    float* bare[2];
    void* mesh_scratch;
    long long mesh_scratch_bytes;
    float *tal4, *ang, *flux_a, *flux_b, *m_i, *m_F, *m_O, *cos_i, *y, *V, *tmp5;
    float *tmp, *ua, *ub, *F, *mask_phi;
    uint8_t* mask;
    int* mask_idx;
    int n_mask;
    int* active;
    int* words;
    int cur;
    long long steps_done;
    void* arena;                    // one allocation holds every buffer above
    cudaEvent_t trace_ev[2];        // petch_plan_timing: recorded around the neutral-pair traces
};

namespace {

// Carve the plan's buffers out of one allocation (256-byte aligned pieces); returns the bytes
// needed when base is NULL.
long long carve(petch_plan_s* p, char* base) {
    long long off = 0;
    auto take = [&](long long bytes) -> char* {
        char* r = base ? base + off : nullptr;
        off += (bytes + 255) / 256 * 256;
        return r;
    };
    long long mesh_bytes = 0;
    {
        long long offs[PETCH_MESH_SEGMENTS];
        petch_mesh_layout(p->MT, p->MV, offs, PETCH_MESH_SEGMENTS, &mesh_bytes);
    }
    const long long MT = p->MT, n = p->ncell;
    p->mesh[0] = take(mesh_bytes);
    p->mesh[1] = take(mesh_bytes);
    p->bare[0] = (float*)take(4 * MT);
    p->bare[1] = (float*)take(4 * MT);
    p->mesh_scratch = take(p->mesh_scratch_bytes);
    p->tal4 = (float*)take(16 * MT);
    p->ang = (float*)take(4 * MT);
    p->flux_a = (float*)take(4 * MT);
    p->flux_b = (float*)take(4 * MT);
    p->m_i = (float*)take(4 * MT);
    p->m_F = (float*)take(4 * MT);
    p->m_O = (float*)take(4 * MT);
    p->cos_i = (float*)take(4 * MT);
    p->y = (float*)take(12 * MT);
    p->V = (float*)take(4 * MT);
    p->tmp5 = (float*)take(20 * MT);
    p->tmp = (float*)take(4 * n);
    p->ua = (float*)take(4 * n);
    p->ub = (float*)take(4 * n);
    p->F = (float*)take(4 * n);
    p->mask_phi = (float*)take(4 * n);
    p->mask = (uint8_t*)take(n);
    p->mask_idx = (int*)take(4 * n);
    p->active = (int*)take(4 * n);
    p->words = (int*)take(4 * W_COUNT);
    return off;
}

petch_batch_grid grid_of(const petch_plan_s* p) {
    petch_batch_grid g;
    std::memset(&g, 0, sizeof(g));
    g.phi = p->phi;
    g.tmp = p->tmp;
    g.ua = p->ua;
    g.ub = p->ub;
    g.F = p->F;
    g.mask_phi = p->mask_phi;
    g.mask_idx = p->mask_idx;
    g.n_mask = p->n_mask;
    g.active = p->active;
    g.n_active = p->words + W_NACTIVE;
    g.max_active = (int)p->ncell;
    g.nx = p->cfg.nx;
    g.ny = p->cfg.ny;
    g.nz = p->cfg.nz;
    g.dx = p->cfg.dx;
    g.dt = p->cfg.dt;
    g.stats = p->words + W_STATS;
    g.hdr = reinterpret_cast<const int*>(p->mesh[p->cur]);   // the header is segment 0
    g.sub = p->words + W_SUB;
    g.hold = p->words + W_HOLD;
    return g;
}

#define PETCH_TRY(call)          \
    do {                         \
        int _rc = (call);        \
        if (_rc) return _rc;     \
    } while (0)

// NVTX ranges of petch_step: one over the step and one per stage (next() closes the previous
// stage's), all closed on every exit path.  They mark the host calls that enqueue the work (a
// profiler's timeline shows them beside the kernels launched); a captured graph's replays make
// no host calls and carry none.
struct NvtxStages {
    bool open = false;
    NvtxStages() { nvtxRangePushA("petch_step"); }
    void next(const char* name) {
        if (open) nvtxRangePop();
        nvtxRangePushA(name);
        open = true;
    }
    ~NvtxStages() {
        if (open) nvtxRangePop();
        nvtxRangePop();
    }
    NvtxStages(const NvtxStages&) = delete;
    NvtxStages& operator=(const NvtxStages&) = delete;
};

}  // namespace

extern "C" int petch_plan(const petch_step_config* cfg, float* phi, int seed_field,
                          petch_plan_t** out, void* stream) {
    PETCH_REQUIRE(cfg && phi && out, "petch_plan: null pointer");
    *out = nullptr;
    const petch_step_config& c = *cfg;
    PETCH_REQUIRE(c.nx > 1 && c.ny > 1 && c.nz > 1 && c.dx > 0.0 && c.dt >= 0.0,
                  "petch_plan: bad grid (%d %d %d, dx %g, dt %g)", c.nx, c.ny, c.nz, c.dx, c.dt);
    PETCH_REQUIRE((long long)c.nx * c.ny * c.nz < (1LL << 31), "petch_plan: grid too large");
    PETCH_REQUIRE(c.n_ion >= 0 && c.n_neu >= 0 && c.n_neu < (1 << 29),
                  "petch_plan: ray counts out of range");
    PETCH_REQUIRE(c.max_tris > 0 && c.max_tris < (1 << 28), "petch_plan: bad max_tris %d",
                  c.max_tris);
    PETCH_REQUIRE(c.n_fp >= 0 && c.n_fp <= 64 && c.n_smooth >= 0,
                  "petch_plan: bad coverage rounds / smoothing passes");
    cudaStream_t st = as_stream(stream);
    petch_plan_s* p = new (std::nothrow) petch_plan_s;
    PETCH_REQUIRE(p, "petch_plan: out of host memory");
    std::memset(p, 0, sizeof(*p));
    p->cfg = c;
    p->MT = c.max_tris;
    p->MV = c.max_tris;
    p->ncell = (long long)c.nx * c.ny * c.nz;
    p->phi = phi;
    int rc = petch_mesh_scratch_bytes(c.nx, c.ny, c.nz, p->MT, &p->mesh_scratch_bytes);
    if (rc) {
        delete p;
        return rc;
    }
    const long long bytes = carve(p, nullptr);
    cudaMemPool_t pool = nullptr;
    rc = plan_pool(&pool);
    if (rc) {
        delete p;
        return rc;
    }
    cudaError_t e = cudaMallocFromPoolAsync(&p->arena, (size_t)bytes, pool, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // usable from any stream from here on
    if (e != cudaSuccess) {
        delete p;
        return cuda_fail(e, "petch_plan: workspace allocation");
    }
    carve(p, (char*)p->arena);
    auto fail = [&](int code) {
        cudaStreamSynchronize(st);
        cudaFreeAsync(p->arena, st);
        delete p;
        return code;
    };
    if (cudaMemsetAsync(p->words, 0, 4 * W_COUNT, st) != cudaSuccess ||
        cudaMemsetAsync(p->mesh[0], 0, 64, st) != cudaSuccess ||
        cudaMemsetAsync(p->mesh[1], 0, 64, st) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "petch_plan: clearing the workspace"));
    // make_trench_3d (threed.py:32-59): the CSG field and mask; with seed_field the field is
    // redistanced into phi (24 cells, zero nodes frozen), otherwise phi keeps the caller's level
    // set and only the mask is taken from the geometry.
    float* csg = seed_field ? p->tmp : p->ub;
    rc = petch_seed_level_set(csg, p->mask, c.nx, c.ny, c.nz, c.dx, c.Lx, c.Ly, c.sub_top,
                              c.mask_th, c.trench_width, c.hole, stream);
    if (rc) return fail(rc);
    if (seed_field) {
        const double band = 24.0 * c.dx;
        rc = petch_reinit_eik(csg, phi, p->ua, p->ub, c.nx, c.ny, c.nz, c.dx,
                              (float)(band + 4.0 * c.dx), (float)(band + c.dx), 28, 1, stream);
        if (rc) return fail(rc);
    }
    if (cudaMemcpyAsync(p->mask_phi, phi, 4 * p->ncell, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "petch_plan: mask_phi"));
    k_mask_list<<<grid_for(p->ncell, 256), 256, 0, st>>>(p->mask, p->ncell, p->mask_idx,
                                                           p->words + W_NACTIVE);
    if (cudaGetLastError() != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "k_mask_list"));
    count_launch();
    int n_mask = 0;
    if (cudaMemcpyAsync(&n_mask, p->words + W_NACTIVE, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "petch_plan: mask count"));
    p->n_mask = n_mask;
    if (cudaMemsetAsync(p->words, 0, 4 * W_COUNT, st) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "petch_plan: clearing the words"));
    rc = petch_prepare_device();
    if (rc) return fail(rc);
    *out = p;
    return PETCH_OK;
}

extern "C" int petch_step(petch_plan_s* p, void* stream) {
    PETCH_REQUIRE(p, "petch_step: null plan");
    const petch_step_config& c = p->cfg;
    cudaStream_t st = as_stream(stream);
    const int MT = p->MT, MV = p->MV;
    const bool cold = p->steps_done == 0 || !c.warm_start;
    const int cur = p->cur, prev = 1 - cur;
    int* w = p->words;
    NvtxStages stage;
    PETCH_CUDA(cudaMemsetAsync(w, 0, 4 * kPerStepWords, st), "petch_step: step words");
    // mesh: marching cubes, geometry, adjacency, BVH
    stage.next("mesh");
    PETCH_TRY(petch_mesh_build(p->phi, c.nx, c.ny, c.nz, c.dx, c.Lx, c.Ly, c.sub_top, c.mask_th,
                               c.trench_width, c.hole, p->mesh[cur], MT, MV, p->mesh_scratch,
                               p->mesh_scratch_bytes, stream));
    // coverage: warm start from the previous mesh, or cold at 1
    stage.next("flux");
    if (!cold) {
        PETCH_TRY(petch_warmstart(p->mesh[prev], MT, MV, p->bare[prev], p->mesh[cur], MT, MV,
                                  p->bare[cur], w + W_WORK, stream));
    } else {
        k_fill<<<grid_for(MT, 256), 256, 0, st>>>(p->bare[cur], MT, 1.0f);
        PETCH_LAUNCH_CHECK("k_fill");
    }
    // ions (seed (step + seed_offset) * 9 + 1, step from the device counter) and their
    // post-processing
    const uint32_t off = (uint32_t)c.seed_offset;
    PETCH_TRY(trace_ions_stepped(p->mesh[cur], MT, MV, &c.dom, &c.ion, w + W_STEP, 9, off, 1,
                                 c.n_ion, p->tal4, p->ang, w + W_WORK, stream));
    const double A_src = c.Lx * c.Ly;
    float* y_sp = p->y;
    float* y_ie = p->y + MT;
    float* y_ip = p->y + 2LL * MT;
    PETCH_TRY(petch_ion_post(p->mesh[cur], MT, MV, p->tal4, p->ang,
                             c.n_ion > 0 ? (float)(A_src / c.n_ion) : 0.0f, c.n_smooth,
                             c.smooth_alpha, y_sp, y_ie, y_ip, p->m_i, p->cos_i, p->tmp5, stream));
    // coverage fixed point: both neutral species of a round in one launch (F: betaE, seed
    // * 9 + 2 + 2 it; O: betaO, seed * 9 + 3 + 2 it), normalised + smoothed, Belen coverages
    const int n_fp = c.n_fp > 0 ? c.n_fp : (cold ? 4 : 1);
    const float norm_neu = c.n_neu > 0 ? (float)(A_src / c.n_neu) : 0.0f;
    for (int it = 0; it < n_fp; ++it) {
        if (it == 0 && p->trace_ev[0])
            PETCH_CUDA(record_timing_event(p->trace_ev[0], st), "petch_step: timing event");
        PETCH_TRY(trace_neutral_pair_stepped(p->mesh[cur], MT, MV, &c.dom, p->bare[cur], c.betaE,
                                             c.betaO, w + W_STEP, 9, off, 2 + 2 * it, 3 + 2 * it,
                                             0, c.n_neu, p->flux_a, p->flux_b, w + W_WORK, stream));
        if (it == n_fp - 1 && p->trace_ev[1])
            PETCH_CUDA(record_timing_event(p->trace_ev[1], st), "petch_step: timing event");
        PETCH_TRY(petch_norm_smooth(p->mesh[cur], MT, MV, p->flux_a, norm_neu, 0.0f, 8.0f, 1,
                                    c.n_smooth, c.smooth_alpha, p->m_F, p->tmp5, p->tmp5 + MT,
                                    stream));
        PETCH_TRY(petch_norm_smooth(p->mesh[cur], MT, MV, p->flux_b, norm_neu, 0.0f, 8.0f, 1,
                                    c.n_smooth, c.smooth_alpha, p->m_O, p->tmp5, p->tmp5 + MT,
                                    stream));
        PETCH_TRY(petch_belen_bare(p->mesh[cur], MT, MV, &c.chem, p->m_i, p->m_F, p->m_O,
                                   p->cos_i, y_ie, y_ip, p->bare[cur], stream));
    }
    // surface rate, then the velocity into the band (mask cells folded to -1, band list)
    stage.next("rate + extend");
    PETCH_TRY(petch_surface_rate(p->mesh[cur], MT, MV, &c.chem, p->m_i, p->m_F, p->m_O, p->cos_i,
                                 y_sp, y_ie, y_ip, p->V, w + W_STATS, stream));
    PETCH_TRY(petch_extend_velocity(p->mesh[cur], MT, MV, p->phi, p->mask, c.nx, c.ny, c.nz, c.dx,
                                    4.0 * c.dx, p->V, p->F, 1, p->active, w + W_NACTIVE,
                                    (int)p->ncell, w + W_WORK, stream));
    // CFL substeps on the device, narrow-band advection, Eikonal reinit (band 4dx + 2dx); all
    // skipped when the mesh overflowed
    stage.next("advect + reinit");
    k_hold<<<1, 32, 0, st>>>(w, reinterpret_cast<const int*>(p->mesh[cur]));
    PETCH_LAUNCH_CHECK("k_hold");
    const petch_batch_grid g = grid_of(p);
    PETCH_TRY(petch_batch_advect(&g, 1, stream));
    PETCH_TRY(petch_batch_reinit(&g, 1, 4.0 * c.dx + 2.0 * c.dx, stream));
    k_accumulate<<<1, 32, 0, st>>>(w, reinterpret_cast<const int*>(p->mesh[cur]));
    PETCH_LAUNCH_CHECK("k_accumulate");
    if (c.warm_start) p->cur = prev;
    p->steps_done += 1;
    return PETCH_OK;
}

extern "C" int petch_plan_seek(petch_plan_t* p, long long step) {
    PETCH_REQUIRE(p && step >= 0, "petch_plan_seek: null plan or negative step");
    p->steps_done = step;
    p->cur = p->cfg.warm_start ? (int)(step & 1) : 0;
    return PETCH_OK;
}

extern "C" int petch_plan_status(petch_plan_s* p, petch_step_status* s, void* stream) {
    PETCH_REQUIRE(p && s, "petch_plan_status: null pointer");
    int h[W_COUNT];
    cudaStream_t st = as_stream(stream);
    PETCH_CUDA(cudaMemcpyAsync(h, p->words, sizeof(h), cudaMemcpyDeviceToHost, st),
               "petch_plan_status: read");
    PETCH_CUDA(cudaStreamSynchronize(st), "petch_plan_status: sync");
    std::memset(s, 0, sizeof(*s));
    s->steps = h[W_STEP];
    s->faces = h[W_F];
    s->max_faces = h[W_FMAX];
    s->trace_errors = h[W_TERR];
    s->mesh_errors = h[W_MERR];
    s->nonfinite = h[W_NONFINITE];
    s->nsub = h[W_NSUB];
    s->nsub_max = h[W_NSUBMAX];
    std::memcpy(&s->queries, h + W_QUERIES, sizeof(long long));
    std::memcpy(&s->vmax, h + W_STATS + 1, sizeof(float));
    if (h[W_MERR] & (1 | 2 | 4)) {
        set_error("petch_step: mesh capacity %d exceeded (error bits %d, largest mesh %d faces); "
                  "that step and the ones after it left the level set unchanged -- plan again "
                  "with a larger max_tris and repeat them from step %d",
                  p->MT, h[W_MERR], h[W_FMAX], h[W_STEP]);
        return PETCH_E_OVERFLOW;
    }
    if (h[W_TERR]) {
        set_error("petch_step: device traversal limit hit (error bits %d)", h[W_TERR]);
        return PETCH_E_LIMIT;
    }
    return PETCH_OK;
}

extern "C" int petch_plan_timing(petch_plan_s* p, int on) {
    PETCH_REQUIRE(p, "petch_plan_timing: null plan");
    for (int i = 0; i < 2; ++i) {
        if (on && !p->trace_ev[i])
            PETCH_CUDA(cudaEventCreate(&p->trace_ev[i]), "petch_plan_timing: event");
        if (!on && p->trace_ev[i]) {
            PETCH_CUDA(cudaEventDestroy(p->trace_ev[i]), "petch_plan_timing: event");
            p->trace_ev[i] = nullptr;
        }
    }
    return PETCH_OK;
}

extern "C" int petch_plan_trace_ms(petch_plan_s* p, float* ms) {
    PETCH_REQUIRE(p && ms, "petch_plan_trace_ms: null pointer");
    PETCH_REQUIRE(p->trace_ev[0] && p->trace_ev[1], "petch_plan_trace_ms: timing is off");
    PETCH_CUDA(cudaEventSynchronize(p->trace_ev[1]), "petch_plan_trace_ms: sync");
    PETCH_CUDA(cudaEventElapsedTime(ms, p->trace_ev[0], p->trace_ev[1]),
               "petch_plan_trace_ms: elapsed time");
    return PETCH_OK;
}

extern "C" int petch_plan_mask(petch_plan_s* p, unsigned char* host_mask, void* stream) {
    PETCH_REQUIRE(p && host_mask, "petch_plan_mask: null pointer");
    cudaStream_t st = as_stream(stream);
    PETCH_CUDA(cudaMemcpyAsync(host_mask, p->mask, (size_t)p->ncell, cudaMemcpyDeviceToHost, st),
               "petch_plan_mask: copy");
    PETCH_CUDA(cudaStreamSynchronize(st), "petch_plan_mask: sync");
    return PETCH_OK;
}

extern "C" int petch_destroy(petch_plan_s* p) {
    if (!p) return PETCH_OK;
    petch_plan_timing(p, 0);
    // as cudaFree would: no work of the plan may still be running when its workspace returns to
    // the pool (work on any stream, hence the device-wide wait)
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaFreeAsync(p->arena, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    delete p;
    if (e != cudaSuccess) return cuda_fail(e, "petch_destroy");
    return PETCH_OK;
}
