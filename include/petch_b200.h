/*
 * petch-b200 C ABI: the per-step 3D etch loop of petch (level set -> marching-cubes surface ->
 * Monte-Carlo ion / neutral flux -> SF6/O2 coverage fixed point -> upwind advection -> Eikonal
 * reinit) as sm_100a CUDA kernels behind plain C entry points.
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller; the library never allocates,
 *     frees or keeps them (scratch buffers are passed in too) -- except the fused step's plan
 *     (petch_plan), which allocates its workspace once and frees it in petch_destroy;
 *   - grids are (nx, ny, nz) C-order, z fastest: cell (i, j, k) is at (i * ny + j) * nz + k, node
 *     coordinates x = i * dx, y = j * dx, z = k * dx (as petch's make_trench_3d);
 *   - `stream` is a cudaStream_t (NULL = legacy default stream); work is enqueued, not waited on;
 *   - the return value is a PETCH_* status; on failure petch_last_error() gives a message.
 *
 * Each declaration names the petch function it replaces as `petch/<file>:<line>` (paths within
 * the reference project's src/ tree).
 */
#ifndef PETCH_B200_H
#define PETCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PETCH_OK = 0,
    PETCH_E_INVALID = 1,   /* bad argument (null pointer, non-positive size, ...) */
    PETCH_E_CUDA = 2,      /* a CUDA runtime call or kernel launch failed */
    PETCH_E_OVERFLOW = 3,  /* a caller-sized device buffer was too small (output truncated) */
    PETCH_E_NONFINITE = 4, /* non-finite values met where the reference raises */
    PETCH_E_LIMIT = 5      /* a bounded device loop hit its iteration limit */
};

/* ABI version (bumped on any signature change). */
int petch_abi_version(void);

/* Number of kernel launches this library has enqueued since it was loaded (all threads). */
int petch_launch_count(long long* n);

/* Copies the last error message of the calling host thread into buf (NUL-terminated, <= n bytes).
 * Returns the message length. */
int petch_last_error(char* buf, int n);

/* ------------------------------------------------------------------------------------------ */
/* Level set                                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* Replaces make_trench_3d (petch/threed.py:32-59): writes the analytic CSG field
 * max(sub_top - z, min(min(z - sub_top, sub_top + mask_th - z), r - width/2)) with
 * r = hypot(x - Lx/2, y - Ly/2) (hole) or |x - Lx/2| (trench), and the mask flag
 * (z in [sub_top, sub_top + mask_th) and outside the opening), evaluated in double.
 * The reference then calls skfmm.distance; callers redistance with petch_reinit_eik. */
int petch_seed_level_set(float* phi, uint8_t* mask, int nx, int ny, int nz, double dx,
                         double Lx, double Ly, double sub_top, double mask_th, double width,
                         int hole, void* stream);

/* Replaces advect_3d_gpu + _advect_iter (petch/threed.py:1262-1307): `nsub` first-order
 * Godunov upwind substeps phi <- phi - dt_sub * F * sqrt(g), with a zero one-sided difference at
 * the domain faces; cells with mask != 0 are re-pinned to mask_phi every substep.
 * phi (in/out) and tmp are ping-pong buffers of nx*ny*nz floats; the result lands in phi.
 * If mask is NULL, cells with F < 0 are treated as mask cells (the engine's folded encoding).
 * inv_dx and dt_sub are the float32 values the reference passes (1/dx and dt/nsub). */
int petch_advect(float* phi, float* tmp, const float* F, const uint8_t* mask,
                 const float* mask_phi, int nx, int ny, int nz, float inv_dx, float dt_sub,
                 int nsub, void* stream);

/* Block shape of the row-mapped level-set stencils (knob of the tuner, petch_b200.tune): bz
 * threads along z (a multiple of 32) by br grid rows, bz * br <= 256; default 128 x 2.  Applies
 * to later reinit calls (single grid, batched, allocation-free).  Results do not depend on it. */
int petch_stencil_config(int bz, int br);

/* Replaces reinit_fsm + _eik_init + _eik_jacobi + _eik_solve (petch/threed.py:1421-1537):
 * Russo-Smereka frozen interface distance, n_iter Jacobi Godunov-Eikonal sweeps, then
 * phi_out = sign(phi_in) * min(U, cap) with sign(0) = +1.  big = band + 4 dx and
 * cap = band + dx as the reference computes them (float64, rounded to float32); dx is taken in
 * double so that 1/dx is rounded once, as the reference's host does; n_iter >= 1.
 * phi_in may alias phi_out.  u_a, u_b: scratch of nx*ny*nz floats each.
 * mode 0 is reinit_fsm exactly.  mode 1 is the stand-in for skfmm.distance on the initial field
 * (make_trench_3d, petch/threed.py:56): nodes where phi_in == 0 are frozen at distance 0 and stay
 * 0, as fast marching keeps them on the front. */
int petch_reinit_eik(const float* phi_in, float* phi_out, float* u_a, float* u_b, int nx,
                     int ny, int nz, double dx, float big, float cap, int n_iter, int mode,
                     void* stream);


/* petch_reinit_eik without caller scratch, for callers that cannot allocate device memory at
 * all (a host framework that owns the whole device heap and forbids driver allocations, or a
 * fixed-budget loop that cannot afford an allocation's latency and implicit synchronisation).
 * No counterpart in the reference (its reinit_fsm allocates Warp arrays on every call).
 * The two Eikonal scratch grids live in a fixed device array of the library (16 MiB held by
 * every GPU that loads it, until exit), so the grid may have at most 2,097,152 cells; larger
 * grids are rejected with PETCH_E_INVALID.  Allocates nothing.  The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress); make it before any stream capture.  The
 * address is kept for the life of the process: do not call it again after cudaDeviceReset (or
 * any destruction of the device's primary context), which may move the array.
 * Calls share the array: calls whose kernels overlap on the GPU race.  Same arguments and
 * results as petch_reinit_eik otherwise. */
int petch_reinit_eik_noalloc(const float* phi_in, float* phi_out, int nx, int ny, int nz,
                             double dx, float big, float cap, int n_iter, int mode, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Surface mesh + BVH (one caller-allocated device buffer, rebuilt each step)                  */
/* ------------------------------------------------------------------------------------------ */

/* Segments of a mesh buffer, in order (offsets from petch_mesh_layout):
 *   0 hdr int32[16]: [0] faces F, [1] vertices V, [2] BVH leaves, [3] error bits
 *     (1 face overflow, 2 vertex overflow, 4 hash full, 8 non-manifold edge), [8..13] root box
 *   1 vnode f32[3*MV] vertex position / dx     2 verts f32[3*MV] vertex position (um)
 *   3 faces i32[3*MT] (winding normal points into the gas)    4 tri f32[12*MT] tracer copy
 *   5 area f32[MT] max(area, 1e-9)   6 normal f32[3*MT]   7 centroid f32[3*MT]
 *   8 fmask u8[MT] faces_in_mask     9 nbr i32[3*MT] edge neighbours (-1 none)
 *  10 nbrw f32[3*MT] max(0, n_i.n_j) 11..15 BVH (leaf codes, leaf starts, nodes, links, flags) */
#define PETCH_MESH_SEGMENTS 16

/* Byte offsets of the segments and the total size of a mesh buffer for the given capacities
 * (0 < max_tris < 2^28). */
int petch_mesh_layout(int max_tris, int max_verts, long long* offsets, int n_offsets,
                      long long* total_bytes);

/* Scratch bytes petch_mesh_build needs for an (nx, ny, nz) grid. */
int petch_mesh_scratch_bytes(int nx, int ny, int nz, int max_tris, long long* bytes);

/* Replaces extract_mesh_3d_gpu + faces_in_mask + _edge_adjacency + _smooth_prep_dev + wp.Mesh
 * (petch/threed.py:62-125, 228-257, 1608-1616, 1674-1675): marching cubes at phi = 0 (phi > 0
 * solid) emitting faces in Morton order of their cubes, float64 areas / centroids, winding normals,
 * faces_in_mask(Lx, Ly, sub_top, mask_th, width, hole), edge neighbours with smoothing weights,
 * and a linear BVH over the surface cubes.  Counts stay on the device (hdr). */
int petch_mesh_build(const float* phi, int nx, int ny, int nz, double dx, double Lx, double Ly,
                     double sub_top, double mask_th, double width, int hole, void* mesh,
                     int max_tris, int max_verts, void* scratch, long long scratch_bytes,
                     void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Monte-Carlo flux (Philox4x32-10 streams keyed by (seed, species), counted by ray id)        */
/* ------------------------------------------------------------------------------------------ */

typedef struct petch_domain {
    float lx, ly, lz;   /* source plane extent and open top (Lx, Ly, Lz) */
    float z_src;        /* source plane height, Lz - dx */
    int periodic;       /* 1: periodic x/y wrap for rays that miss (par['periodic_y']); a ray
                           above the surface takes its wraps down to the mesh's top in one step
                           (the same re-entry points, wrap count and 256-wrap limit) */
} petch_domain;

typedef struct petch_ion_params {  /* the float32 arguments of _trace3d_ion_yield */
    float meanE, sigmaE;
    float A_sp, Eth_sp, B_sp, A_ie, Eth_ie, A_p, Eth_p;
    float inflect, minang, n_l, A_en, minE, thrmin, thrmax;
    float sigma;        /* ion angular spread of the source (par['ion_ang_sigma']) */
} petch_ion_params;

/* Tracer configuration for this process (knobs of the tuner, petch_b200.tune): bvh_width 2
 * (binary LBVH, default) or 8 (quantised 8-wide BVH, built only by mesh builds made while it is
 * configured); each warp runs traversal steps for all its lanes with an open query, at most
 * steps_per_round (default 32) and only while more than keep_lanes lanes (0..31, default 16)
 * still have one, between shading / refill rounds; once the ray pool is empty a warp steps until
 * its last query ends.  Applies to later trace / raycast calls. */
int petch_tracer_config(int bvh_width, int steps_per_round, int keep_lanes);

/* Warp-aggregated deposits for later trace calls (on = 1; default 0): lanes of a warp that
 * deposit into the same tally entry in the same hit combine their values first and one lane
 * issues the atomic (the reference deposits with one wp.atomic_add per tally per hit, threed.py:575,
 * 648-652).  Results are the same estimator (bit-equal with deterministic tallies); the choice is
 * a speed knob of the tuner. */
int petch_tally_aggregation(int on);

/* Leaf grouping of the traversal (binary and 8-wide) for later trace calls (knob of the tuner):
 * 0 off, or g in 2..8 -- each warp iteration then runs the triangle tests of the lanes at a leaf
 * when they are at least 1/g of the lanes with an open query, otherwise the box tests of the
 * lanes at an internal node, instead of both paths in every iteration.  Default 2.  Results do
 * not depend on it (each lane's traversal order is unchanged). */
int petch_tracer_grouping(int group);

/* The tracer settings in force: out[0] BVH width, [1] steps per round, [2] keep lanes, [3]
 * warp-aggregated deposits (0 / 1), [4] leaf grouping. */
int petch_tracer_settings(int* out);

/* Replaces _gen_source + _trace3d_ion_yield (petch/threed.py:441-458, 599-712): n_ion ions
 * generated and traced on the device.  tally4 (16-byte aligned float4[max_tris]) receives per
 * face (sputter, ion-enhanced, passivation, arrival) and ang the cos-weighted arrival; both are
 * zeroed first.  work: int[6] device words, 8-byte aligned: [0] ray counter (reset by every trace
 * call), [1] error bits OR-ed by every kernel (1 = traversal bound hit, 2 = active list full,
 * 4 = tracer round bound hit, 8 = BVH width 8 configured but the mesh was built without the
 * 8-wide tree)
 * until the caller clears them, [2..3] uint64 BVH queries and [4..5] uint64 node + leaf visits,
 * accumulated by every trace call until the caller clears them. */
int petch_trace_ions(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                     const petch_ion_params* p, uint32_t seed, int n_ion, float* tally4,
                     float* ang, int* work, void* stream);

/* Replaces _gen_source + _trace3d_cov_rr (petch/threed.py:441-458, 549-596): n_neu
 * Russian-roulette neutrals with sticking bare[f] * beta (bare NULL = 1); flux (float[max_tris],
 * zeroed first) receives the arriving weight.  stream_id separates species / fixed-point
 * iterations that share a seed. */
int petch_trace_neutrals(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                         const float* bare, float beta, uint32_t seed, uint32_t stream_id,
                         int n_neu, float* flux, int* work, void* stream);

/* Replaces the two _trace3d_cov_rr launches of one coverage round (petch/threed.py:898-902: the F
 * species with betaE, the O species with betaO, on the same coverage) with ONE launch: rays
 * [0, n_neu) follow petch_trace_neutrals with (beta_a, seed_a), rays [n_neu, 2 n_neu) with
 * (beta_b, seed_b), both with stream_id; ray r of each species draws the same Philox stream as in
 * the single-species call, so each flux equals that call's up to the order of float atomic
 * additions (exactly, with deterministic tallies).  flux_a, flux_b: float[max_tris], distinct,
 * zeroed first; n_neu < 2^30. */
int petch_trace_neutral_pair(const void* mesh, int max_tris, int max_verts,
                             const petch_domain* dom, const float* bare, float beta_a,
                             float beta_b, uint32_t seed_a, uint32_t seed_b, uint32_t stream_id,
                             int n_neu, float* flux_a, float* flux_b, int* work, void* stream);

/* Replaces _trace3d (petch/threed.py:352-406), the legacy species of mc_flux_3d and the
 * non-faithful ion of mc_flux_3d_coupled: first-hit / specular ions (ion = 1, source tilt sigma)
 * or neutrals with fixed sticking and n_reemit diffuse re-emissions; no lateral wrap. */
int petch_trace_legacy(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                       int ion, float sigma, float sticking, int n_reemit, int specular,
                       float cos_thr, float eta, uint32_t seed, int n, float* flux, float* angacc,
                       int* work, void* stream);

/* Replaces the electron trace of mc_flux_3d_coupled's surface-charging block
 * (petch/threed.py:852-856: _src('ion', ..., e_ang_sigma) + _trace3d_cov_rr with bare = 1,
 * beta = 1): n electrons from the Gaussian-angle source (tilt sigma), each depositing weight 1
 * on the face it first reaches; lateral wrap as the domain says.  flux float[max_tris], zeroed
 * first. */
int petch_trace_electrons(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                          float sigma, uint32_t seed, int n, float* flux, int* work, void* stream);

/* Replaces extend_velocity_gpu + _extend_kernel (petch/threed.py:1324-1346): Fs = V[nearest face]
 * on cells with |phi| < band, else 0.  fold_mask = 1: mask cells get -1 (petch_advect's pinned
 * marker, mask may not be NULL) and band cells with Fs > 0 are appended to active (if not NULL;
 * count in *n_active, overflow past max_active sets work[1] bit 2). */
int petch_extend_velocity(const void* mesh, int max_tris, int max_verts, const float* phi,
                          const uint8_t* mask, int nx, int ny, int nz, double dx, double band,
                          const float* V, float* Fs, int fold_mask, int* active, int* n_active,
                          int max_active, int* work, void* stream);

/* Replaces extend_velocity_3d (petch/threed.py:1310-1321, run_etch_3d's extend != "gpu"): as
 * petch_extend_velocity but each band cell takes V of the face with the nearest CENTROID (the
 * reference's cKDTree over centroids); exact ties go to the lower face index. */
int petch_extend_velocity_centroid(const void* mesh, int max_tris, int max_verts, const float* phi,
                                   const uint8_t* mask, int nx, int ny, int nz, double dx,
                                   double band, const float* V, float* Fs, int fold_mask,
                                   int* active, int* n_active, int max_active, int* work,
                                   void* stream);

/* Replaces gpu_warmstart_bare + _nearest_face_cov (petch/threed.py:1619-1639): bare[f] =
 * clip(prev_bare[nearest face of the previous mesh to centroid f], 0, 1), 1 if none. */
int petch_warmstart(const void* prev_mesh, int prev_max_tris, int prev_max_verts,
                    const float* prev_bare, const void* mesh, int max_tris, int max_verts,
                    float* bare, int* work, void* stream);

/* Replaces wp.mesh_query_ray (used by every petch trace kernel): closest hit of each ray
 * (o, d: float[3n]) with 0 <= t < tmax; face = -1 on a miss. */
int petch_raycast(const void* mesh, int max_tris, int max_verts, const float* o, const float* d,
                  int n, float tmax, int* face, float* t, int* work, void* stream);

/* Replaces wp.mesh_query_point_no_sign (petch/threed.py:1328, 1626): nearest face of each point
 * (float[3n]) within max_dist, ties to the lower face index; -1 if none. */
int petch_nearest_face(const void* mesh, int max_tris, int max_verts, const float* p, int n,
                       float max_dist, int* face, int* work, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Per-face post-processing and surface chemistry (float64 arithmetic, float32 arrays)         */
/* ------------------------------------------------------------------------------------------ */

typedef struct petch_chem_params {
    double ionFlux, Fflux, Oflux;      /* PAR['ionFlux'], ['Fflux'], ['Oflux'] */
    double k_sigma, beta_sigma;        /* Belen couplings */
    double rho, rate_scale;            /* density factor, rate calibration */
    double fnorm_E, fnorm_O;           /* surface_rate_belen's flux normalisation (default 1) */
    double s_F, s_O;                   /* Langmuir sticking (surface_rate_langmuir) */
    double Yie, Ysp, Yp;               /* IED-integrated yields (chemistry._yields) */
    double B_sp;                       /* sputter angular coefficient */
    int yield_angular;                 /* 0 = "cosine", 1 = "viennaps" */
    int chemistry;                     /* 0 = "langmuir", 1 = "belen" */
} petch_chem_params;

/* Replaces _norm_clip + smooth_flux_dev (petch/threed.py:165-214, _finish :783-790):
 * out = clamp((fl / area) * scale, lo, hi) (no clamp if clip == 0), then n_smooth passes of
 * the 1-neighbour smoothing, each blended with its own input by alpha.  tmp_a, tmp_b: float[MT]. */
int petch_norm_smooth(const void* mesh, int max_tris, int max_verts, const float* fl, float scale,
                      float lo, float hi, int clip, int n_smooth, float alpha, float* out,
                      float* tmp_a, float* tmp_b, void* stream);

/* Replaces the faithful-ion post-processing of mc_flux_3d_coupled (petch/threed.py:814-823):
 * from petch_trace_ions' tallies, y_sp/y_ie/y_ip = smoothed (tally / area) * norm (the ion
 * yields, no clip), m_i = smoothed (arrival / area) * norm, cos_i = ang / max(arrival, 1e-9)
 * where arrival > 0 (unsmoothed).  smooth_flux_gpu semantics: n_smooth passes, one final blend
 * by alpha.  tmp: float[5 * max_tris]. */
int petch_ion_post(const void* mesh, int max_tris, int max_verts, const float* tally4,
                   const float* ang, float norm, int n_smooth, float alpha, float* y_sp, float* y_ie,
                   float* y_ip, float* m_i, float* cos_i, float* tmp, void* stream);

/* Replaces _cos_k (petch/threed.py:179-185): out = ang / fl where fl > 0, else 0. */
int petch_cos_ratio(const void* mesh, int max_tris, int max_verts, const float* fl,
                    const float* ang, float* out, void* stream);

/* Replaces _belen_coverages + the bare update of the fixed point (petch/threed.py:715-737,
 * 903-904): bare = clip(1 - thetaF - thetaO, 0, 1).  y_ie / y_ip: the faithful-ion yields, or
 * both NULL for the analytic yields (Yie, Yp with the angular factor of cos_i). */
int petch_belen_bare(const void* mesh, int max_tris, int max_verts, const petch_chem_params* p,
                     const float* m_i, const float* m_F, const float* m_O, const float* cos_i,
                     const float* y_ie, const float* y_ip, float* bare, void* stream);

/* Replaces surface_rate (chemistry.py:83-92 -> belen.py:26-63 / chemistry.py:96-114) and
 * run_etch_3d's guard (petch/threed.py:1721-1728): V per face, 0 on faces_in_mask faces,
 * non-finite values zeroed.  stats: int[2] device, [0] = non-finite count, [1] = float bits of
 * max(V) (for the CFL substep count).  Yields: all three or NULL (analytic). */
int petch_surface_rate(const void* mesh, int max_tris, int max_verts, const petch_chem_params* p,
                       const float* m_i, const float* m_F, const float* m_O, const float* cos_i,
                       const float* y_sp, const float* y_ie, const float* y_ip, float* V,
                       int* stats, void* stream);

/* petch_advect restricted to a narrow band, with identical results: cells listed in `active`
 * (F > 0, not mask, from petch_extend_velocity) are updated each substep; mask cells (mask_idx)
 * are re-pinned to mask_phi after the first substep; every other cell keeps its value.
 * tmp: nx*ny*nz floats of scratch. */
int petch_advect_sparse(float* phi, float* tmp, const float* F, const float* mask_phi,
                        const int* mask_idx, int n_mask, const int* active, int n_active, int nx,
                        int ny, int nz, float inv_dx, float dt_sub, int nsub, void* stream);

/* Replaces reinit_gpu + _reinit_iter (petch/threed.py:1349-1418, reinit_method="gpu"): n_iter
 * forward-Euler sweeps (step 0.3 dx) of phi_tau + sgn(phi0)(|grad phi| - 1) = 0 with the
 * Russo-Smereka sub-cell target phi0 / max(|grad phi0|, 0.5) clipped to +-1.8 dx at interface
 * cells (sign change with a face neighbour).  phi0, tmp: scratch grids; phi_out may equal phi_in. */
int petch_reinit_pde(const float* phi_in, float* phi_out, float* phi0, float* tmp, int nx, int ny,
                     int nz, double dx, int n_iter, void* stream);

/* Replaces run_etch_3d's surf_smooth step (petch/threed.py:1779-1782):
 * phi = scipy.ndimage.gaussian_filter(phi, sigma) (axes 0, 1, 2 in turn; weights
 * exp(-t^2 / (2 sigma^2)) normalised over |t| <= int(truncate * sigma + 0.5) <= 64; 'reflect'
 * boundaries; double accumulation), then phi[mask] = mask_phi[mask] when mask is not NULL.
 * tmp_a, tmp_b: scratch grids. */
int petch_gaussian_smooth(float* phi, float* tmp_a, float* tmp_b, const uint8_t* mask,
                          const float* mask_phi, int nx, int ny, int nz, double sigma,
                          double truncate, void* stream);

/* The column scan of the depth metrics (_depth3d / max_depth_3d, petch/threed.py:1798-1869):
 * for each column cols[2c], cols[2c+1] (= i, j; device ints) of phi (nx, ny, nz; z fastest),
 * k_out[c] = the index of the lowest cell of the gas run (phi < 0) that reaches the top cell, -1
 * when the top cell is not gas, -2 when (i, j) lies outside the grid.  The caller takes zs[k]
 * and the median / percentile. */
int petch_column_floors(const float* phi, int nx, int ny, int nz, const int* cols, int n_cols,
                        int* k_out, void* stream);

/* Deterministic tallies (no reference counterpart).  With a scratch registered, every tracing
 * entry point accumulates its per-face tallies as 64-bit fixed-point integers (units of 2^-32,
 * carved from the scratch, converted to the float outputs at the end of the call): integer sums
 * do not depend on the order in which rays deposit, so with the Philox streams fixed a run is
 * reproducible bit for bit.  Deposits are rounded to 2^-32 (far below the 1e-6 weight floor of
 * the Russian roulette).  The scratch must hold 8 bytes per tally entry of the largest call
 * (ions: 5 * max_tris, 8 * max_tris with tangents; batches: per instance) plus 256-byte
 * alignment per array; calls fail with PETCH_E_INVALID otherwise.  NULL switches back to float
 * atomics.  Process-wide state: calls on several streams at once share the scratch and race. */
int petch_set_deterministic(void* scratch, long long scratch_bytes);

/* ---- batched tracing (many independent instances in one launch) ---- */

/* Caches the host-side device queries the launchers use (SM count, resident blocks of the
 * persistent tracers) for the current device, so that calls made while a stream is being
 * captured into a CUDA graph issue no driver queries.  Call once per device before capturing. */
int petch_prepare_device(void);

/* One instance of a batched trace: its mesh buffer (laid out by petch_mesh_layout with the
 * batch's max_tris / max_verts), domain, ion parameters (kind 0), coverage (kind 1; NULL = 1),
 * outputs and ray count.  out: kind 0 the tally4 of petch_trace_ions (float4[max_tris], 16-byte
 * aligned), kind 1 the flux of petch_trace_neutrals (float[max_tris]); ang: kind 0 only. */
typedef struct petch_batch_item {
    const void* mesh;
    petch_domain dom;
    petch_ion_params ion;
    const float* bare;
    float* out;
    float* ang;
    int n_rays;
    uint32_t seed;       /* added to *step before the seed multiplier */
} petch_batch_item;

/* No single reference counterpart: runs petch_trace_ions (kind 0) or petch_trace_neutrals
 * (kind 1, coverage-weighted with beta) for up to 64 instances in ONE persistent launch with one
 * global ray queue, zeroing each instance's outputs first.  Ray r of instance b uses the Philox
 * stream of ray r in the single-instance call with seed (*step + items[b].seed) * seed_mul +
 * seed_add (step: device int, NULL = 0), so the result equals the per-instance calls up to the
 * order of float atomic additions.  The seed is read on the device: the call can be captured in
 * a CUDA graph and replayed step after step.  items: host array (copied into the launch).
 * work: as petch_trace_ions, shared by the batch. */
int petch_trace_batch(int kind, const petch_batch_item* items, int B, int max_tris, int max_verts,
                      float beta, const int* step, uint32_t seed_mul, uint32_t seed_add,
                      int* work, void* stream);

/* petch_trace_batch for both neutral species of a coverage round in ONE launch (the batched
 * counterpart of petch_trace_neutral_pair): item b's rays [0, n_rays) follow kind 1 with beta_a
 * and seed_add_a into items[b].out, rays [n_rays, 2 n_rays) with beta_b and seed_add_b into
 * items[b].ang (the second flux, float[max_tris], distinct from out); each species' ray r draws
 * the Philox stream of ray r of its own kind-1 launch.  n_rays <= 2^29 per item. */
int petch_trace_batch_pair(const petch_batch_item* items, int B, int max_tris, int max_verts,
                           float beta_a, float beta_b, const int* step, uint32_t seed_mul,
                           uint32_t seed_add_a, uint32_t seed_add_b, int* work, void* stream);

/* Tangent outputs of one instance for petch_trace_batch_tangent: dout = d(sputter, ion-enhanced,
 * passivation tallies) / d(mean ion energy) [3][max_tris] (kind 0) or d(flux) [3][max_tris] along
 * the three recipe directions (kind 1); dbare = the coverage tangents [3][max_tris] (kind 1; NULL
 * = 0). */
typedef struct petch_batch_tangent {
    float* dout;
    const float* dbare;
} petch_batch_tangent;

/* petch_trace_batch carrying tangents: the batched form of petch_trace_ions_tangent (kind 0) and
 * petch_trace_neutrals_tangent (kind 1); tans: host array parallel to items. */
int petch_trace_batch_tangent(int kind, const petch_batch_item* items,
                              const petch_batch_tangent* tans, int B, int max_tris, int max_verts,
                              float beta, const int* step, uint32_t seed_mul, uint32_t seed_add,
                              int* work, void* stream);

/* petch_trace_batch_pair with the weight tangents of petch_trace_batch_tangent kind 1: item b's
 * rays [0, n_rays) (beta_a, seed_add_a) deposit into items[b].out and tans_a[b].dout, rays
 * [n_rays, 2 n_rays) (beta_b, seed_add_b) into items[b].ang and tans_b[b].dout; tans_a[b].dbare
 * is the coverage tangent both species read (tans_b[b].dbare is not read). */
int petch_trace_batch_pair_tangent(const petch_batch_item* items,
                                   const petch_batch_tangent* tans_a,
                                   const petch_batch_tangent* tans_b, int B, int max_tris,
                                   int max_verts, float beta_a, float beta_b, const int* step,
                                   uint32_t seed_mul, uint32_t seed_add_a, uint32_t seed_add_b,
                                   int* work, void* stream);

/* One instance's level-set state for the batched stages. */
typedef struct petch_batch_grid {
    float* phi;              /* level set (in / out) */
    float* tmp;              /* advection ping-pong grid */
    float* ua;               /* reinit scratch grids */
    float* ub;
    const float* F;          /* extended speed, -1 on mask cells (petch_extend_velocity fold_mask) */
    const float* mask_phi;
    const int* mask_idx;     /* the mask cells (F == -1) */
    int n_mask;
    const int* active;       /* band cells with F > 0 and their count (petch_extend_velocity) */
    const int* n_active;
    int max_active;
    int nx, ny, nz;
    double dx;
    double dt;               /* the etch step, t_end / n_steps */
    const int* stats;        /* petch_surface_rate's stats: [1] = float bits of max V */
    const int* hdr;          /* the mesh header: [0] = face count */
    int* sub;                /* out, int[2]: [0] substeps, [1] float bits of dt / nsub */
    const int* hold;         /* device int or NULL: nonzero leaves this level set unchanged (no
                              * substeps, no reinit) -- a step whose mesh overflowed */
} petch_batch_grid;

/* Replaces, for B <= 64 instances at once, run_etch_3d's CFL substep count and advect_3d_gpu
 * (petch/threed.py:1750-1764, 1262-1307) as petch_advect_sparse does them: nsub from stats and
 * hdr on the device, then a fixed sequence of 160 substep launches in which instance b steps
 * while s < nsub_b.  Results equal per-instance petch_advect_sparse calls.  Graph-capturable. */
int petch_batch_advect(const petch_batch_grid* grids, int B, void* stream);

/* Replaces, for B <= 64 instances with the same dx, reinit_fsm (petch/threed.py:1515-1537) as
 * petch_reinit_eik mode 0 with band = band_r, in place on each phi: the same values, with each
 * sweep restricted per grid row to the z range the front's distances can have reached (the row
 * ranges live in each instance's tmp grid, which must be 8-byte aligned; nz >= 4).
 * Graph-capturable. */
int petch_batch_reinit(const petch_batch_grid* grids, int B, double band_r, void* stream);

/* The tangent state of one instance for the batched tangent stages (direction-major [3][n]
 * arrays of the instance's n = nx*ny*nz cells). */
typedef struct petch_batch_tangent_grid {
    float* dphi;                 /* level-set tangents (in / out) */
    float* dtmp;                 /* advection ping-pong */
    const float* dF;             /* speed tangents (petch_extend_tangent) */
    const unsigned char* mask;   /* 1 on mask cells: pinned to mask_phi, tangent 0 */
    float* du_a;                 /* reinit scratch */
    float* du_b;
} petch_batch_tangent_grid;

/* petch_batch_advect carrying tangents: the CFL substep count on the device, then 160 substep
 * launches of petch_advect_tangent's dense dual update over all instances (instance b steps while
 * s < nsub_b).  Values equal per-instance petch_advect_tangent calls.  Graph-capturable. */
int petch_batch_advect_tangent(const petch_batch_grid* grids,
                               const petch_batch_tangent_grid* tans, int B, void* stream);

/* petch_batch_reinit carrying tangents (petch_reinit_tangent per instance, same dx for all). */
int petch_batch_reinit_tangent(const petch_batch_grid* grids,
                               const petch_batch_tangent_grid* tans, int B, double band_r,
                               void* stream);

/* *step += 1 on the device (the step counter petch_trace_batch seeds from). */
int petch_batch_step_advance(int* step, void* stream);

/* ---- etch-product redeposition (mc_redep_3d, petch/threed.py:1582-1605) ---- */

/* CUB scratch bytes petch_trace_redep needs for max_tris faces. */
int petch_redep_scratch_bytes(int max_tris, long long* bytes);

/* Replaces mc_redep_3d's emission and trace (petch/threed.py:1590-1604): n product particles,
 * each leaving face j with probability w_j / sum(w), w = max(V * area, 0) (cdf: double[max_tris]
 * receives the inclusive prefix of w), from centroid + 1e-3 fn in a cosine direction about fn
 * (petch_gas_normals), traced like _trace3d_cov_rr with bare = 1 and beta = s_redep and no
 * lateral wrap; flux (float[max_tris], zeroed first) = deposited weight per face.  Philox stream
 * keyed by (seed, particle).  No particles are traced when sum(w) <= 0.  work: as
 * petch_trace_ions. */
int petch_trace_redep(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                      const float* fn, const float* V, float s_redep, uint32_t seed, int n,
                      float* flux, double* cdf, void* scratch, long long scratch_bytes, int* work,
                      void* stream);

/* Replaces mc_redep_3d's normalisation and run_etch_3d's use of it (petch/threed.py:1605, 1743):
 * Rf = flux * (sum(w) / n) / area (written to Rf if not NULL), V = max(V - k_redep * Rf, 0), and,
 * if stats is not NULL, stats[1] = float bits of the new max(V) (as petch_surface_rate). */
int petch_redep_apply(const void* mesh, int max_tris, int max_verts, const float* flux,
                      const double* cdf, int n, float k_redep, float* V, float* Rf, int* stats,
                      void* stream);

/* ---- deterministic radiosity neutrals (mc_flux_3d_radiosity, petch/threed.py:923-991) ---- */

/* Replaces _gas_normals (petch/threed.py:1553-1568): fn (float[3 * max_tris]) = the face's unit
 * winding normal, flipped to agree with -grad(phi) at the grid node nearest its centroid
 * (np.gradient differences: central inside, one-sided at the grid faces). */
int petch_gas_normals(const void* mesh, int max_tris, int max_verts, const float* phi, int nx,
                      int ny, int nz, double dx, float* fn, void* stream);

/* Replaces the form-factor cast of mc_flux_3d_radiosity (petch/threed.py:947-956: origins
 * centroid + 1e-3 fn, _cosine_dirs :1571-1579, _trace_ff :908-920 with _apply_bc's periodic
 * wrap): n_ff cosine-distributed rays per face, hitface[j * n_ff + k] = first face hit by ray k
 * of face j, or -1 if it escapes (entries past F * n_ff are -1).  hitface: int[max_tris * n_ff].
 * Philox stream keyed by (seed, ray).  work: as petch_trace_ions. */
int petch_trace_ff(const void* mesh, int max_tris, int max_verts, const petch_domain* dom,
                   const float* fn, uint32_t seed, int n_ff, int* hitface, int* work,
                   void* stream);

/* Scratch bytes petch_ff_matrix needs for a mesh of max_tris faces and n_ff rays per face. */
int petch_ff_scratch_bytes(int max_tris, int n_ff, long long* bytes);

/* Replaces the matrix assembly of mc_flux_3d_radiosity (petch/threed.py:957-960): from
 * petch_trace_ff's hits, sky[i] = escaping rays of face i / n_ff (double[max_tris]) and the CSR
 * of A[i, j] = F_{j->i}: row_ptr (int[max_tris + 1]) and col (int[max_tris * n_ff]) with one
 * entry of weight 1 / n_ff per ray (repeated j for repeated hits), entries of a row in ascending
 * ray order.  No host synchronisation; the result is identical on every run. */
int petch_ff_matrix(const void* mesh, int max_tris, int max_verts, const int* hitface, int n_ff,
                    int* row_ptr, int* col, double* sky, void* scratch, long long scratch_bytes,
                    void* stream);

/* Replaces solve() of mc_flux_3d_radiosity with the Jacobi solver (petch/threed.py:966-985):
 * for beta in (betaE, betaO): G = sky, then n_iter times G = sky + M G with
 * M[i, j] = A[i, j] (1 - clip(bare_j beta, 0, 1)), in float64; g_E / g_O = clip(G, 0, 8) as float.
 * work2: double[4 * max_tris] scratch. */
int petch_radiosity_solve(const void* mesh, int max_tris, int max_verts, const int* row_ptr,
                          const int* col, const double* sky, int n_ff, const float* bare,
                          double betaE, double betaO, int n_iter, float* g_E, float* g_O,
                          double* work2, void* stream);

/* petch_radiosity_solve with the three recipe tangents (no reference counterpart: the reference's
 * solve is not differentiated): dbare float[3][max_tris] the coverage tangents; the same primal
 * bits in g_E / g_O, and dg_E / dg_O float[3][max_tris] the tangents of the clipped G (the form
 * factors and the sky view are geometry, held fixed; 0 where the clips hold).  n_iter >= 1;
 * work: double[16 * max_tris] scratch. */
int petch_radiosity_solve_tangent(const void* mesh, int max_tris, int max_verts,
                                  const int* row_ptr, const int* col, const double* sky, int n_ff,
                                  const float* bare, const float* dbare, double betaE,
                                  double betaO, int n_iter, float* g_E, float* g_O, float* dg_E,
                                  float* dg_O, double* work, void* stream);

/* ---- DDA neutral transport (deterministic discrete ordinates) ----
 * Replaces dda_neutral_flux (petch/dda.py:132-188) as called by mc_flux_3d_dda
 * (petch/threed.py:1211-1244).  petch_dda_prepare marches every (face, direction) ray of
 * _dda_gather_kernel (dda.py:26-96) once through the occupancy grid and records where it ends
 * (a solid cell, an escape at z >= z_top, or nothing after max_steps), computes the direct view,
 * each face's solid-side wall cell round(centroid - 0.7 dx n) and the cells of the one-cell
 * dilation; petch_dda_solve then runs n_reemit re-emission passes plus the Aitken extrapolation
 * for both sticking fields s = clip(bare * betaE / betaO, 0, 1) from those records.  March and
 * gather sums in float32, the cell re-emission, dilation and extrapolation in float64, every sum in
 * the reference's order: bit-reproducible.
 * Grid: phi float[nx*ny*nz] (phi > 0 solid), node i at x = i dx.  Faces: n_faces is a DEVICE int
 * (the live count, clamped to max_faces; a mesh header's HDR_F word works), origins / normals
 * float[3*max_faces] (surface points and unit into-gas normals), areas float[max_faces].
 * Directions: dirs float[3*n_dirs], weights float[n_dirs] (fib_sphere(2 * dda_n_dir): unit
 * weights).  z_top and max_steps as dda.py:137-151 computes them.  The scratch holds the whole
 * prepared geometry (copies of normals, areas, directions included); petch_dda_solve reads only it,
 * bare float[max_faces], and writes flux_E / flux_O float[max_faces]. */
int petch_dda_scratch_bytes(int max_faces, int nx, int ny, int nz, int n_dirs, long long* bytes);
int petch_dda_prepare(const float* phi, int nx, int ny, int nz, double dx, double z_top,
                      int max_steps, int periodic_y, const int* n_faces, int max_faces,
                      const float* origins, const float* normals, const float* areas,
                      const float* dirs, const float* weights, int n_dirs, void* scratch,
                      long long scratch_bytes, void* stream);
int petch_dda_solve(int max_faces, int nx, int ny, int nz, int n_dirs, const float* bare,
                    double betaE, double betaO, int n_reemit, void* scratch,
                    long long scratch_bytes, float* flux_E, float* flux_O, void* stream);

/* petch_extend_velocity (nearest face) and petch_extend_tangent in one pass: the same nearest-face
 * query gives Fs and dF (dV, dF: [3][max_tris] and [3][nx*ny*nz] tangents). */
int petch_extend_velocity_dual(const void* mesh, int max_tris, int max_verts, const float* phi,
                               const unsigned char* mask, int nx, int ny, int nz, double dx,
                               double band, const float* V, const float* dV, float* Fs, float* dF,
                               int fold_mask, int* active, int* n_active, int max_active,
                               int* work, void* stream);

/* petch_warmstart and petch_warmstart_tangent in one pass (one nearest-face query per face). */
int petch_warmstart_dual(const void* prev_mesh, int prev_max_tris, int prev_max_verts,
                         const float* prev_bare, const float* prev_dbare, const void* mesh,
                         int max_tris, int max_verts, float* bare, float* dbare, int* work,
                         void* stream);

/* ---- Knudsen 1-D conductance tail (mc_flux_3d_knudsen, petch/threed.py:1149-1208) ----
 * petch_knudsen_prepare replaces slice_geometry (petch/knudsen.py:29-68) and the per-face part of
 * knudsen_face_flux (knudsen.py:188-241) that depends only on the geometry: per z-slice below
 * sub_top the gas area and perimeter of phi (hole; trench = 1: mean open x-width and 2), the
 * chain of valid slices with their conductances, each face's slice (its rounded centroid height,
 * snapped to the nearest valid slice), and the floor faces (into-gas n_z > 0.7, below sub_top,
 * within half_width + 2 dx of the axis (cx, cy); half_width < 0: no footprint filter) grouped by
 * slice.  Faces: n_faces a DEVICE int (clamped to max_faces), centroids / normals float[3 * max_faces].
 * petch_knudsen_solve runs one coverage round for both sticking fields
 * s = clip(bare' * betaE / betaO, 0, 1), bare' = min(bare, mean of bare over the open-field faces)
 * when sink_field != 0 (knudsen_sink = 'field'): the slice sinks 0.25 s A (per unit length Ly for a
 * trench), the conductance chain (conductance_profile, knudsen.py:91-150) with loss scale
 * wall_loss_scale, or, front_loss != 0, the passivation-linked per-slice scale of
 * _front_loss_scale (knudsen.py:165-185; W the feature width), and writes flux_E / flux_O
 * (float[max_faces]).  petch_knudsen_profile solves the chain of the prepared geometry for a
 * caller's sink slice_loss (double[nz], device) and loss scale (loss_scale double[nz] device, or
 * NULL for the scalar) into profile (double[nz], device); petch_knudsen_slices copies out the slice
 * areas and perimeters. */
int petch_knudsen_scratch_bytes(int max_faces, int nz, long long* bytes);
int petch_knudsen_prepare(const float* phi, int nx, int ny, int nz, double dx, double sub_top,
                          int trench, const int* n_faces, int max_faces, const float* centroids,
                          const float* normals, double cx, double cy, double half_width,
                          void* scratch, long long scratch_bytes, void* stream);
int petch_knudsen_solve(int max_faces, int nz, const float* bare, const float* areas, double betaE,
                        double betaO, int sink_field, double Ly, double wall_loss_scale,
                        int front_loss, double W, double band_W, double pass_frac, double ar_pass,
                        void* scratch, long long scratch_bytes, float* flux_E, float* flux_O,
                        void* stream);
int petch_knudsen_profile(int max_faces, int nz, const double* slice_loss, const double* loss_scale,
                          double wall_loss_scale, void* scratch, long long scratch_bytes,
                          double* profile, void* stream);
int petch_knudsen_slices(int max_faces, int nz, const void* scratch, long long scratch_bytes,
                         double* area, double* perimeter, void* stream);

/* ---- floor-charging hooks (_apply_hg_charging, petch/threed.py:1046-1110;
 * _apply_floor_charge_throttle, :1112-1147) ----
 * Face classes: in the feature = within `band` of the axis (hole: hypot(x - cx, y - cy); trench:
 * |x - cx|) and below sub_top; floor = in the feature with into-gas n_z > 0.7.
 * petch_charging_floor_stats writes stats (double[5], device): floor faces, the lowest floor
 * centroid z, sum of m_i A over the floor (m_i may be NULL: 0), and the count and summed area of the
 * foot (in the feature, n_z <= 0.7, z <= that lowest z + foot_h).  petch_charging_apply multiplies
 * the floor's m_i, y_sp, y_ie, y_p by q4[0..3] and adds add3[0..2] to y_sp, y_ie, y_p of the
 * non-floor in-feature faces with z <= z_foot (q4, add3: HOST arrays; any of the float arrays may
 * be NULL).  petch_zero_below zeroes values[f] where the centroid z <= z_top (run_etch_3d's
 * redeposition foot cleaning, threed.py:1733-1741). */
int petch_charging_floor_stats(const int* n_faces, int max_faces, const float* centroids,
                               const float* normals, const float* areas, const float* m_i,
                               double cx, double cy, double band, int hole, double sub_top,
                               double foot_h, double* stats, void* stream);
int petch_charging_apply(const int* n_faces, int max_faces, const float* centroids,
                         const float* normals, double cx, double cy, double band, int hole,
                         double sub_top, const double* q4, const double* add3, double z_foot,
                         float* m_i, float* y_sp, float* y_ie, float* y_p, void* stream);
int petch_zero_below(const int* n_faces, int max_faces, const float* centroids, double z_top,
                     float* values, void* stream);

/* Replaces the charging factor of mc_flux_3d_coupled (petch/threed.py:862-868): with
 * sh_e = clip(m_e / max(ref_e, 1e-6), 0, 1) and sh_i likewise from m_i and ref_i, every face's
 * m_i (in place) is multiplied by 1 - alpha clip(1 - sh_e / max(sh_i, 1e-3), 0, 1).  ref_i,
 * ref_e: the 90th percentiles of m_i and m_e over the faces above 1e-6 (1 when none), computed
 * by the caller.  Float64 arithmetic. */
int petch_electron_shadow(const int* n_faces, int max_faces, const float* m_e, double ref_i,
                          double ref_e, double alpha, float* m_i, void* stream);

/* Replaces solve() with radiosity_solver = 'gmres' (petch/threed.py:972-982): restarted GMRES
 * (restart Krylov vectors per cycle, at most maxiter cycles, modified Gram-Schmidt, Givens
 * rotations, x0 = 0) on (I - M) G = D, M[i, j] = A[i, j] (1 - clip(bare_j beta, 0, 1)), with the
 * reference's stopping rule |D - (I - M) G| <= rtol |D| (atol 0).  g_out = clip(G, 0, 8); *info
 * (host int) = 0 when converged, 1 when not (the reference then falls back to the Jacobi sweeps:
 * petch_radiosity_solve).  Float64, every sum in a fixed order; the host reads one scalar per
 * Arnoldi step (the call synchronises the stream).  Scratch: petch_radiosity_gmres_scratch_bytes. */
int petch_radiosity_gmres_scratch_bytes(int max_tris, int restart, long long* bytes);
int petch_radiosity_gmres(const void* mesh, int max_tris, int max_verts, const int* row_ptr,
                          const int* col, const double* sky, int n_ff, const float* bare,
                          double beta, double rtol, int restart, int maxiter, float* g_out,
                          void* scratch, long long scratch_bytes, int* info, void* stream);

/* ---- recipe gradient: tangent (forward-mode) versions of the step's stages ----
 * No reference counterpart (the reference has no loop gradient).  Each call computes the
 * primal result exactly as its plain counterpart and the derivatives of it along 3 directions
 * (the recipe parameters theta_k), taking the primal's branches: ray hits, sticking / roulette
 * and energy-acceptance decisions, upwind and min / max selections, clamps and nearest faces are
 * held fixed (the pathwise derivative; visibility-boundary terms are not included).  Tangent
 * arrays are direction-major: direction k of a field of n entries starts at k * n. */

/* petch_trace_ions plus dtal[3][max_tris] = d(sputter, ion-enhanced, passivation tallies) /
 * d(mean ion energy) along the same paths. */
int petch_trace_ions_tangent(const void* mesh, int max_tris, int max_verts,
                             const petch_domain* dom, const petch_ion_params* p, uint32_t seed,
                             int n_ion, float* tally4, float* ang, float* dtal, int* work,
                             void* stream);

/* petch_trace_neutrals plus dflux[3][max_tris], the tallies' tangents given the coverage
 * tangents dbare[3][max_tris] (NULL = 0). */
int petch_trace_neutrals_tangent(const void* mesh, int max_tris, int max_verts,
                                 const petch_domain* dom, const float* bare, const float* dbare,
                                 float beta, uint32_t seed, uint32_t stream_id, int n_neu,
                                 float* flux, float* dflux, int* work, void* stream);

/* petch_trace_neutral_pair with the weight tangents of petch_trace_neutrals_tangent: both
 * species of a coverage round in one launch (rays [0, n_neu): beta_a, seed_a into flux_a /
 * dflux_a; rays [n_neu, 2 n_neu): beta_b, seed_b into flux_b / dflux_b), each equal to its own
 * tangent launch up to the order of float atomic additions (exactly, with deterministic tallies).
 * dbare, dflux_*: [3][max_tris]; outputs zeroed first; n_neu < 2^30. */
int petch_trace_neutral_pair_tangent(const void* mesh, int max_tris, int max_verts,
                                     const petch_domain* dom, const float* bare,
                                     const float* dbare, float beta_a, float beta_b,
                                     uint32_t seed_a, uint32_t seed_b, uint32_t stream_id,
                                     int n_neu, float* flux_a, float* dflux_a, float* flux_b,
                                     float* dflux_b, int* work, void* stream);

/* Tangent of petch_norm_smooth (blend_last_only = 0) or of petch_ion_post's smoothing
 * (blend_last_only = 1, clip = 0): dout[3][max_tris] from dfl[3][max_tris] (fl: the primal
 * tally, for the clamp).  tmp_a, tmp_b: float[max_tris]. */
int petch_norm_smooth_tangent(const void* mesh, int max_tris, int max_verts, const float* fl,
                              const float* dfl, float scale, float lo, float hi, int clip,
                              int n_smooth, float alpha, int blend_last_only, float* dout,
                              float* tmp_a, float* tmp_b, void* stream);

/* petch_belen_bare (faithful-ion yields) in float64 dual arithmetic: bare and dbare[3][MT] from
 * the tangents of m_F, m_O, y_ie, y_ip ([3][MT] each, NULL = 0) and dOflux[3] (host). */
int petch_belen_bare_tangent(const void* mesh, int max_tris, int max_verts,
                             const petch_chem_params* p, const double* dOflux, const float* m_F,
                             const float* dm_F, const float* m_O, const float* dm_O,
                             const float* y_ie, const float* dy_ie, const float* y_ip,
                             const float* dy_ip, float* bare, float* dbare, void* stream);

/* petch_surface_rate (Belen chemistry, faithful-ion yields) in float64 dual arithmetic: V and
 * dV[3][MT]; dOflux[3], drate[3]: d Oflux / d theta_k and d rate_scale / d theta_k (host). */
int petch_surface_rate_tangent(const void* mesh, int max_tris, int max_verts,
                               const petch_chem_params* p, const double* dOflux,
                               const double* drate, const float* m_F, const float* dm_F,
                               const float* m_O, const float* dm_O, const float* y_sp,
                               const float* dy_sp, const float* y_ie, const float* dy_ie,
                               const float* y_ip, const float* dy_ip, float* V, float* dV,
                               int* stats, void* stream);

/* dF[3][n] = dV[3][max_tris] of the nearest face on cells with |phi| < band (the choice
 * petch_extend_velocity makes), 0 elsewhere. */
int petch_extend_tangent(const void* mesh, int max_tris, int max_verts, const float* phi, int nx,
                         int ny, int nz, double dx, double band, const float* dV, float* dF,
                         int* work, void* stream);

/* dbare[3][MT] of the warm start (petch_warmstart): the previous mesh's nearest-face tangent,
 * 0 where the copied coverage is clamped. */
int petch_warmstart_tangent(const void* prev_mesh, int prev_max_tris, int prev_max_verts,
                            const float* prev_bare, const float* prev_dbare, const void* mesh,
                            int max_tris, int max_verts, float* dbare, int* work, void* stream);

/* petch_advect (mask array) with tangents: phi / dphi[3][n] advanced nsub substeps with F /
 * dF[3][n]; tmp, dtmp: ping-pong scratch of the same sizes. */
int petch_advect_tangent(float* phi, float* tmp, float* dphi, float* dtmp, const float* F,
                         const float* dF, const uint8_t* mask, const float* mask_phi, int nx,
                         int ny, int nz, float inv_dx, float dt_sub, int nsub, void* stream);

/* petch_reinit_eik (mode 0, in place) with tangents of phi ([3][n]); u_a, u_b: float[n],
 * du_a, du_b: float[3][n] scratch. */
int petch_reinit_tangent(float* phi, float* dphi, float* u_a, float* u_b, float* du_a, float* du_b,
                         int nx, int ny, int nz, double dx, float big, float cap, int n_iter,
                         void* stream);

/* ------------------------------------------------------------------------------------------ */
/* The fused step: a workspace planned once, one call per etch step                            */
/* ------------------------------------------------------------------------------------------ */

/* Everything one run needs (run_etch_3d's arguments, petch/threed.py:1643-1648, for the
 * coverage-coupled Monte-Carlo path that Process(..., SF6O2(), ...).run() takes: faithful ions,
 * Belen coverages, coverage-dependent neutral sticking; FSM reinit). */
typedef struct petch_step_config {
    int nx, ny, nz;                  /* grid (round(L / dx) nodes per axis) */
    double dx, Lx, Ly, Lz;
    double sub_top, mask_th, trench_width;
    int hole;                        /* 1 hole, 0 trench */
    double dt;                       /* t_end / n_steps */
    int n_ion, n_neu;                /* rays per launch (n_neu <= 2^29) */
    int seed_offset;                 /* step s uses seed s + seed_offset (threed.py:1690) */
    int max_tris;                    /* face capacity of the two mesh buffers */
    int n_fp;                        /* coverage rounds per step; 0: 4 cold, 1 warm (threed.py:897) */
    int warm_start;                  /* flags.warm_start_coverage */
    int n_smooth;                    /* par['flux_smooth'] */
    float smooth_alpha;              /* par['flux_smooth_alpha'] */
    float betaE, betaO;              /* par['betaE'], par['betaO'] */
    petch_domain dom;                /* source plane, open top, lateral wrap */
    petch_ion_params ion;            /* _trace3d_ion_yield's arguments */
    petch_chem_params chem;          /* Belen chemistry and rate */
} petch_step_config;

typedef struct petch_plan_s petch_plan_t;

/* Status accumulated over the steps since the plan was made. */
typedef struct petch_step_status {
    int steps;                       /* steps taken (the device step counter) */
    int faces, max_faces;            /* the last step's face count, the largest seen */
    int trace_errors, mesh_errors;   /* error bits OR-ed over the steps */
    int nonfinite;                   /* non-finite surface velocities zeroed, summed */
    int nsub, nsub_max;              /* the last step's CFL substeps, the largest count seen */
    float vmax;                      /* the last step's max surface velocity */
    long long queries;               /* BVH queries, summed */
} petch_step_status;

/* Plans a run of the fused step (the set-up of run_etch_3d, petch/threed.py:1649-1669): allocates
 * one workspace (two mesh buffers of cfg->max_tris faces for the warm-started coverage, the
 * per-face arrays, the level-set scratch grids), derives the mask and mask level set from the
 * geometry (make_trench_3d, threed.py:32-59), and with seed_field = 1 writes the seed field into
 * phi (the CSG field redistanced over 24 cells, zero nodes frozen); with seed_field = 0 phi keeps
 * the caller's level set.  phi (float[nx*ny*nz], device) stays caller-owned and is advanced in
 * place by petch_step.  Synchronises `stream` (the workspace allocation, the mask cell count).
 * The workspace comes from a memory pool of the library's own per device that keeps up to 8 GB
 * of freed workspace for the next plan. */
int petch_plan(const petch_step_config* cfg, float* phi, int seed_field, petch_plan_t** plan,
               void* stream);

/* One etch step of run_etch_3d (petch/threed.py:1671-1792): mesh + BVH, warm-started coverage,
 * ions, the coverage fixed point (both neutral species per round in one launch), surface rate,
 * velocity extension, CFL substeps and narrow-band advection, Eikonal reinit.  Issues only
 * stream-ordered work (no synchronisation, no allocation, no host reads): seeds come from a
 * device step counter and the substep count from the device (160 substep launches, each gated),
 * so steps can be captured into a CUDA graph -- one graph for the first (cold) step and one for
 * two consecutive warm steps, since the mesh / coverage buffers alternate.  With deterministic
 * tallies the result equals run_etch_3d's bit for bit. */
int petch_step(petch_plan_t* plan, void* stream);

/* Sets which step the next petch_step call issues, for callers that capture steps into graphs
 * out of order: step 0 is the cold step, and with warm-started coverage step s works on mesh
 * buffer s % 2.  Only the host-side bookkeeping moves; the seeds still come from the device step
 * counter, which counts executed steps. */
int petch_plan_seek(petch_plan_t* plan, long long step);

/* Reads the plan's accumulated status (synchronises `stream`).  Returns PETCH_E_OVERFLOW if a
 * mesh outgrew max_tris: such a step leaves the level set and the step counter unchanged (so do
 * the steps after it, whose meshes overflow the same way), and status->steps counts the steps
 * done -- plan again with more capacity from the level set and continue from there.  Returns
 * PETCH_E_LIMIT if a tracer hit a traversal bound. */
int petch_plan_status(petch_plan_t* plan, petch_step_status* status, void* stream);

/* Device timing of the step's dominant launches (no reference counterpart): with on = 1 the plan
 * creates two CUDA events that every later petch_step records on its stream, before its first
 * and after its last neutral-pair trace launch (a warm step has one), as external event nodes
 * when the step is captured into a graph, so graph replays record them too; on = 0 frees them.
 * Enable before capturing. */
int petch_plan_timing(petch_plan_t* plan, int on);

/* Milliseconds between those two events of the last step issued (waits for its end event). */
int petch_plan_trace_ms(petch_plan_t* plan, float* ms);

/* The plan's mask (make_trench_3d's mask, petch/threed.py:50-55: 1 for the cells of the
 * un-etched mask the loop pins, uint8 per cell in phi's layout) copied into host memory of
 * nx * ny * nz bytes, on `stream`; waits for the copy. */
int petch_plan_mask(petch_plan_t* plan, unsigned char* host_mask, void* stream);

/* Returns the plan's workspace to the library's pool, after waiting for the device (work of the
 * plan on any stream has finished when it returns). */
int petch_destroy(petch_plan_t* plan);

#ifdef __cplusplus
}
#endif

#endif /* PETCH_B200_H */
