// Surface extraction and acceleration structure, rebuilt every etch step on the device:
//
//   1. marching cubes (replaces Warp's MarchingCubes / skimage, petch/threed.py:62-100), in
//      three passes over the grid nodes enumerated in Morton order -- count (classify + per-block
//      totals), vertex emit, face emit -- with a device scan of the per-block totals between them.
//      Faces therefore come out sorted by the Morton index of their cube, which is exactly the
//      primitive order a linear BVH needs: no sort is run;
//   2. per-face geometry (normals _face_normals_k threed.py:228-234, float64 areas and centroids
//      threed.py:96-99, faces_in_mask threed.py:1608-1616);
//   3. edge adjacency (replaces _edge_adjacency's argsort, threed.py:103-125) through a device
//      hash table of (min vertex, max vertex) keys, stored per face as its three edge neighbours
//      with the smoothing weights max(0, n_i . n_j) (_edge_weights_k, threed.py:237-242).  An
//      edge pairs its faces only when it has exactly two (see k_adj_insert);
//   4. a binary linear BVH (Karras 2012) over the surface cubes (one leaf = the 1..5 faces of one
//      cube) with a bottom-up box refit, replacing wp.Mesh (threed.py:1674-1675).
#include <cub/cub.cuh>
#include "common.cuh"
#include "mc_table.cuh"
#include "mesh.cuh"

namespace petch {

static_assert(mc::table_fits(), "marching-cubes table exceeds 5 faces per cube");
__constant__ mc::Table c_mc = mc::make_table();

static long long align256(long long x) { return (x + 255) & ~255LL; }

MeshLayout mesh_layout(int MT, int MV) {
    const long long sz[SEG_COUNT] = {
        4LL * HDR_INTS,              // hdr
        12LL * MV, 12LL * MV,        // vnode, verts
        12LL * MT, 48LL * MT,        // faces, tri
        4LL * MT, 12LL * MT, 12LL * MT, 1LL * MT,  // area, normal, centroid, fmask
        12LL * MT, 12LL * MT,        // nbr, nbrw
        4LL * MT, 4LL * (MT + 1),    // leaf_code, leaf_start
        64LL * MT, 8LL * MT, 4LL * MT, // nodes, parent, flags
        96LL * MT, 24LL * MT          // wnodes, wfront
    };
    MeshLayout L;
    long long o = 0;
    for (int s = 0; s < SEG_COUNT; ++s) {
        L.off[s] = o;
        o += align256(sz[s]);
    }
    L.total = o;
    return L;
}

MeshView mesh_view(void* base, int MT, int MV) {
    MeshLayout L = mesh_layout(MT, MV);
    char* b = (char*)base;
    MeshView v;
    v.hdr = (int*)(b + L.off[SEG_HDR]);
    v.vnode = (float*)(b + L.off[SEG_VNODE]);
    v.verts = (float*)(b + L.off[SEG_VERTS]);
    v.faces = (int*)(b + L.off[SEG_FACES]);
    v.tri = (float4*)(b + L.off[SEG_TRI]);
    v.area = (float*)(b + L.off[SEG_AREA]);
    v.normal = (float*)(b + L.off[SEG_NORMAL]);
    v.centroid = (float*)(b + L.off[SEG_CENTROID]);
    v.fmask = (uint8_t*)(b + L.off[SEG_FMASK]);
    v.nbr = (int*)(b + L.off[SEG_NBR]);
    v.nbrw = (float*)(b + L.off[SEG_NBRW]);
    v.leaf_code = (uint32_t*)(b + L.off[SEG_LEAF_CODE]);
    v.leaf_start = (int*)(b + L.off[SEG_LEAF_START]);
    v.nodes = (float4*)(b + L.off[SEG_NODES]);
    v.parent = (int*)(b + L.off[SEG_PARENT]);
    v.flags = (int*)(b + L.off[SEG_FLAGS]);
    v.wnodes = (WNode*)(b + L.off[SEG_WNODES]);
    v.wfront = (int2*)(b + L.off[SEG_WFRONT]);
    v.MT = MT;
    v.MV = MV;
    return v;
}

namespace {

constexpr int kB = 256;
constexpr int kWideLevels = 32;   // >= the binary tree depth (<= 31 Morton bits + 1)

// Morton enumeration of an (nx, ny, nz) node grid: axis a gets ceil(log2(n_a)) bits and the bits
// are interleaved from the least significant level up (x, y, z within a level); an axis that has
// run out of bits is skipped, so a tall grid splits along z first at the top of the tree.
struct Morton {
    int nbits;
    uint8_t axis[32];
    uint8_t level[32];
};

int ceil_log2(int n) {
    int b = 0;
    while ((1LL << b) < n) ++b;
    return b;
}

Morton make_morton(int nx, int ny, int nz, bool* ok) {
    int bits[3] = {ceil_log2(nx), ceil_log2(ny), ceil_log2(nz)};
    Morton m{};
    int p = 0;
    for (int l = 0; l < 32; ++l)
        for (int a = 0; a < 3; ++a)
            if (l < bits[a]) {
                if (p < 32) {
                    m.axis[p] = (uint8_t)a;
                    m.level[p] = (uint8_t)l;
                }
                ++p;
            }
    m.nbits = p;
    *ok = p <= 31;
    return m;
}

__device__ __forceinline__ void m_decode(const Morton& m, uint32_t t, int c[3]) {
    c[0] = c[1] = c[2] = 0;
    for (int p = 0; p < m.nbits; ++p) c[m.axis[p]] |= (int)((t >> p) & 1u) << m.level[p];
}

__device__ __forceinline__ uint32_t m_encode(const Morton& m, int i, int j, int k) {
    int c[3] = {i, j, k};
    uint32_t t = 0;
    for (int p = 0; p < m.nbits; ++p) t |= (uint32_t)((c[m.axis[p]] >> m.level[p]) & 1) << p;
    return t;
}

struct Dims {
    int nx, ny, nz;
    long long plane;
};

struct Int4Add {
    __host__ __device__ int4 operator()(const int4& a, const int4& b) const {
        return make_int4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
    }
};

// Block-wide exclusive scan of one 32-bit value (kB threads); returns the exclusive prefix and
// writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = (lane < kB / 32) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kB / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t incl = x + (wid > 0 ? warp_sums[wid - 1] : 0u);
    *total = warp_sums[kB / 32 - 1];
    __syncthreads();
    return incl - v;
}

// Pass 1a, grid order: per node, cube configuration + owned-edge crossings (info bits: 0-7 cube
// config (corner c solid <=> phi > 0), 8-10 owned x/y/z edge crossed, 11 cube exists (node is not
// on a max face)).  Threads run along z (one block row per grid row), so the node and its seven
// upper neighbours are read as contiguous row segments.
constexpr int kMcZ = 128, kMcRows = 2;

__global__ void __launch_bounds__(kMcZ * kMcRows) k_mc_classify(const float* __restrict__ phi,
                                                                Dims d, Morton mo,
                                                                uint16_t* __restrict__ info_lin,
                                                                int* __restrict__ bflag) {
    const int rows = d.nx * d.ny;
    for (int row = blockIdx.x * kMcRows + threadIdx.y; row < rows; row += gridDim.x * kMcRows) {
        const int i = row / d.ny, j = row - (row / d.ny) * d.ny;
        const long long base = (long long)row * d.nz;
        for (int k = threadIdx.x; k < d.nz; k += kMcZ) {
            const long long c = base + k;
            const bool s0 = phi[c] > 0.0f;
            uint32_t cross = 0;
            if (i + 1 < d.nx) cross |= (uint32_t)(s0 != (phi[c + d.plane] > 0.0f)) << 0;
            if (j + 1 < d.ny) cross |= (uint32_t)(s0 != (phi[c + d.nz] > 0.0f)) << 1;
            if (k + 1 < d.nz) cross |= (uint32_t)(s0 != (phi[c + 1] > 0.0f)) << 2;
            uint32_t inf = cross << 8;
            if (i + 1 < d.nx && j + 1 < d.ny && k + 1 < d.nz) {
                uint32_t cfg = 0;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const long long cc = c + (q & 1) * d.plane + ((q >> 1) & 1) * (long long)d.nz +
                                         ((q >> 2) & 1);
                    cfg |= (uint32_t)(phi[cc] > 0.0f) << q;
                }
                inf |= cfg | (1u << 11);
            }
            info_lin[c] = (uint16_t)inf;
            // mark the Morton block of a node that emits a vertex or a face (the count pass
            // skips the blocks no such node falls in)
            const uint32_t cfg = inf & 255u;
            if (cross || ((inf >> 11) & 1u && cfg != 0u && cfg != 255u))
                atomicOr(bflag + (m_encode(mo, i, j, k) / kB), 1);
        }
    }
}

// Pass 1b, Morton order: each node's info gathered from the grid-order pass, and per block the
// packed totals (faces, vertices, BVH leaves) the later passes offset from.
__global__ void __launch_bounds__(kB) k_mc_count(const uint16_t* __restrict__ info_lin, Dims d,
                                                 Morton mo, uint32_t npad, uint32_t nb,
                                                 uint16_t* __restrict__ info,
                                                 int4* __restrict__ bsum,
                                                 int* __restrict__ bflag) {
    // each CTA walks Morton blocks (kB nodes each) with a stride of the grid: a launch of tens of
    // thousands of mostly empty blocks would cost more in block scheduling than their work
    for (uint32_t mb = blockIdx.x; mb < nb; mb += gridDim.x) {
        const uint32_t t = mb * kB + threadIdx.x;
        const bool act = bflag[mb] != 0;
        __syncthreads();                      // every thread has read the flag
        if (!act) {
            // no node of this block emits anything: zero info (no cube, no crossing) and totals
            if (t < npad) info[t] = 0;
            if (threadIdx.x == 0) bsum[mb] = make_int4(0, 0, 0, 0);
            continue;
        }
        if (threadIdx.x == 0) bflag[mb] = 0;  // cleared for the next build
        uint32_t nt = 0, nv = 0, nl = 0;
        if (t < npad) {
            int c3[3];
            m_decode(mo, t, c3);
            uint32_t inf = 0;
            if (c3[0] < d.nx && c3[1] < d.ny && c3[2] < d.nz) {
                inf = info_lin[c3[0] * d.plane + (long long)c3[1] * d.nz + c3[2]];
                if ((inf >> 11) & 1u) nt = c_mc.ntri[inf & 255u];
                nv = __popc((inf >> 8) & 7u);
                nl = nt > 0;
            }
            info[t] = (uint16_t)inf;
        }
        uint32_t tot;
        block_excl_scan(nt | (nv << 11) | (nl << 21), &tot);
        if (threadIdx.x == 0)
            bsum[mb] = make_int4((int)(tot & 2047u), (int)((tot >> 11) & 1023u), (int)(tot >> 21), 0);
    }
}

__global__ void k_mc_totals(const int4* bsum, const int4* boff, int nb, MeshView m) {
    int4 last = boff[nb - 1], s = bsum[nb - 1];
    int F = last.x + s.x, V = last.y + s.y, L = last.z + s.z;
    m.hdr[HDR_F] = F;
    m.hdr[HDR_V] = V;
    m.hdr[HDR_L] = L;
    m.hdr[HDR_MT] = m.MT;
    m.hdr[HDR_MV] = m.MV;
    m.hdr[HDR_NONMANIFOLD] = 0;
    int err = 0;
    if (F > m.MT) err |= MESH_ERR_TRI_OVERFLOW;
    if (V > m.MV) err |= MESH_ERR_VERT_OVERFLOW;
    m.hdr[HDR_ERR] = err;
    int Fc = F < m.MT ? F : m.MT;
    int Lc = L < m.MT ? L : m.MT;
    // An overflowed mesh is incomplete (the faces past the capacity were not emitted, and a leaf
    // can straddle the capacity): publish it with no BVH leaves, so no ray or point query can
    // reach a face index at or beyond max_tris.  The counts stay for the caller to regrow.
    if (err) {
        m.hdr[HDR_L] = 0;
        Lc = 0;
    }
    m.leaf_start[Lc] = Fc;
}

// Pass 2: vertices on crossed owned edges, interpolated at phi = 0 from the edge's lower node.
__global__ void __launch_bounds__(kB) k_mc_verts(const float* __restrict__ phi, Dims d, Morton mo,
                                                 uint32_t npad, uint32_t nb,
                                                 const uint16_t* __restrict__ info,
                                                 const int4* __restrict__ bsum,
                                                 const int4* __restrict__ boff,
                                                 uint32_t* __restrict__ voff, double dx,
                                                 MeshView m) {
    for (uint32_t mb = blockIdx.x; mb < nb; mb += gridDim.x) {
        if (bsum[mb].y == 0) continue;        // no vertex in this block
        const uint32_t t = mb * kB + threadIdx.x;
        const uint32_t cross = (t < npad) ? ((info[t] >> 8) & 7u) : 0u;
        uint32_t nv = __popc(cross), tot;
        const uint32_t ex = block_excl_scan(nv, &tot);
        if (!nv) continue;
        const uint32_t base = (uint32_t)boff[mb].y + ex;
        voff[t] = base;
        int c3[3];
        m_decode(mo, t, c3);
        const long long c = c3[0] * d.plane + (long long)c3[1] * d.nz + c3[2];
        const float va = phi[c];
        const long long step[3] = {d.plane, (long long)d.nz, 1};
        uint32_t r = 0;
        for (int a = 0; a < 3; ++a) {
            if (!((cross >> a) & 1u)) continue;
            uint32_t v = base + r++;
            if (v >= (uint32_t)m.MV) continue;
            float vb = phi[c + step[a]];
            float tt = va / (va - vb);
            float p[3] = {(float)c3[0], (float)c3[1], (float)c3[2]};
            p[a] = p[a] + tt;
            for (int q = 0; q < 3; ++q) {
                m.vnode[3 * v + q] = p[q];
                m.verts[3 * v + q] = (float)((double)p[q] * dx);
            }
        }
    }
}

// Pass 3: faces (global vertex ids from the owner nodes' offsets) and BVH leaves.
__global__ void __launch_bounds__(kB) k_mc_faces(Dims d, Morton mo, uint32_t npad, uint32_t nb,
                                                 const uint16_t* __restrict__ info,
                                                 const int4* __restrict__ bsum,
                                                 const int4* __restrict__ boff,
                                                 const uint32_t* __restrict__ voff, MeshView m) {
    for (uint32_t mb = blockIdx.x; mb < nb; mb += gridDim.x) {
        if (bsum[mb].x == 0) continue;        // no face (hence no leaf) in this block
        const uint32_t t = mb * kB + threadIdx.x;
        const uint32_t inf = (t < npad) ? info[t] : 0u;
        const uint32_t cfg = inf & 255u;
        const uint32_t nt = ((inf >> 11) & 1u) ? c_mc.ntri[cfg] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan(nt | ((nt > 0) << 16), &tot);
        if (!nt) continue;
        const int f0 = boff[mb].x + (int)(ex & 0xffffu);
        const int leaf = boff[mb].z + (int)(ex >> 16);
        int c3[3];
        m_decode(mo, t, c3);
        for (uint32_t q = 0; q < nt; ++q) {
            int f = f0 + (int)q;
            if (f >= m.MT) break;
            for (int s = 0; s < 3; ++s) {
                int e = c_mc.tri[cfg][3 * q + s];
                int cc = mc::edge_corner(e), ax = mc::edge_axis(e);
                uint32_t to = m_encode(mo, c3[0] + (cc & 1), c3[1] + ((cc >> 1) & 1), c3[2] + ((cc >> 2) & 1));
                uint32_t oc = (info[to] >> 8) & 7u;
                m.faces[3 * f + s] = (int)(voff[to] + __popc(oc & ((1u << ax) - 1u)));
            }
        }
        if (leaf < m.MT) {
            m.leaf_code[leaf] = t;
            m.leaf_start[leaf] = f0;
        }
    }
}

struct FaceParams {
    double dx, Lx, Ly, sub_top, mask_th, width;
    int hole;
};

// Per-face geometry: tracer triangle, float64 area/centroid (from vnode * dx, as the reference's
// float64 host arrays), float32 winding normal (as _face_normals_k on the float32 vertices),
// faces_in_mask on the float64 centroid.
__global__ void __launch_bounds__(kB) k_face_geometry(MeshView m, FaceParams fp) {
    const int F = min(m.hdr[HDR_F], m.MT);
    for (int f = blockIdx.x * kB + threadIdx.x; f < F; f += gridDim.x * kB) {
        int ia = m.faces[3 * f], ib = m.faces[3 * f + 1], ic = m.faces[3 * f + 2];
        if (ia < 0 || ib < 0 || ic < 0 || ia >= m.MV || ib >= m.MV || ic >= m.MV) {
            // vertex capacity overflowed (HDR_ERR is set): make the face inert
            ia = ib = ic = 0;
        }
        double a[3], b[3], c[3];
        float af[3], bf[3], cf[3];
        for (int q = 0; q < 3; ++q) {
            a[q] = (double)m.vnode[3 * ia + q] * fp.dx;
            b[q] = (double)m.vnode[3 * ib + q] * fp.dx;
            c[q] = (double)m.vnode[3 * ic + q] * fp.dx;
            af[q] = m.verts[3 * ia + q];
            bf[q] = m.verts[3 * ib + q];
            cf[q] = m.verts[3 * ic + q];
        }
        m.tri[3 * f + 0] = make_float4(af[0], af[1], af[2], 0.0f);
        m.tri[3 * f + 1] = make_float4(bf[0], bf[1], bf[2], 0.0f);
        m.tri[3 * f + 2] = make_float4(cf[0], cf[1], cf[2], 0.0f);
        double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        double w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        double area = 0.5 * sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        m.area[f] = (float)fmax(area, 1.0e-9);
        // IEEE float32 without contraction (the normal of near-degenerate faces is sensitive
        // to fused multiply-adds): normalize(cross(b - a, c - a)) on the float32 vertices
        float uf[3] = {__fsub_rn(bf[0], af[0]), __fsub_rn(bf[1], af[1]), __fsub_rn(bf[2], af[2])};
        float wf[3] = {__fsub_rn(cf[0], af[0]), __fsub_rn(cf[1], af[1]), __fsub_rn(cf[2], af[2])};
        float n[3] = {__fsub_rn(__fmul_rn(uf[1], wf[2]), __fmul_rn(uf[2], wf[1])),
                      __fsub_rn(__fmul_rn(uf[2], wf[0]), __fmul_rn(uf[0], wf[2])),
                      __fsub_rn(__fmul_rn(uf[0], wf[1]), __fmul_rn(uf[1], wf[0]))};
        float ln = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(n[0], n[0]), __fmul_rn(n[1], n[1])),
                                        __fmul_rn(n[2], n[2])));
        float inv = ln > 0.0f ? __fdiv_rn(1.0f, ln) : 0.0f;
        double cen[3];
        for (int q = 0; q < 3; ++q) {
            m.normal[3 * f + q] = __fmul_rn(n[q], inv);
            cen[q] = (a[q] + b[q] + c[q]) / 3.0;
            m.centroid[3 * f + q] = (float)cen[q];
        }
        bool in_band = cen[2] >= fp.sub_top && cen[2] < fp.sub_top + fp.mask_th;
        bool opening;
        if (fp.hole) {
            double ex = cen[0] - fp.Lx / 2.0, ey = cen[1] - fp.Ly / 2.0;
            opening = ex * ex + ey * ey < (fp.width / 2.0) * (fp.width / 2.0);
        } else {
            opening = fabs(cen[0] - fp.Lx / 2.0) < fp.width / 2.0;
        }
        m.fmask[f] = (in_band && !opening) ? 1 : 0;
    }
}

constexpr unsigned long long kEmpty = ~0ULL;

__device__ __forceinline__ uint32_t hslot(unsigned long long key, int hbits) {
    return (uint32_t)((key * 0x9E3779B97F4A7C15ULL) >> (64 - hbits));
}

__device__ __forceinline__ unsigned long long edge_key(int a, int b) {
    uint32_t lo = (uint32_t)min(a, b), hi = (uint32_t)max(a, b);
    return ((unsigned long long)lo << 32) | hi;
}

// Each edge key's slot counts its faces and sums their ids; an edge with exactly two faces
// pairs them (the other face is sum - self).  Edges with one face (domain boundary) or more than
// two (fan diagonals that coincide across an ambiguous cube face) get no neighbour, which keeps
// the relation symmetric and independent of thread order.
__global__ void __launch_bounds__(kB) k_adj_insert(MeshView m, unsigned long long* keys, int* hcnt,
                                                   int* hsum, int hbits) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const uint32_t hmask = (1u << hbits) - 1u;
    for (int x = blockIdx.x * kB + threadIdx.x; x < 3 * F; x += gridDim.x * kB) {
        int f = x / 3, e = x - 3 * f;
        unsigned long long key = edge_key(m.faces[3 * f + e], m.faces[3 * f + (e + 1) % 3]);
        uint32_t s = hslot(key, hbits);
        bool placed = false;
        for (uint32_t probe = 0; probe <= hmask; ++probe) {
            unsigned long long old = atomicCAS(&keys[s], kEmpty, key);
            if (old == kEmpty || old == key) {
                placed = true;
                break;
            }
            s = (s + 1) & hmask;
        }
        if (!placed) {
            atomicOr(&m.hdr[HDR_ERR], MESH_ERR_HASH_FULL);
            continue;
        }
        atomicAdd(&hsum[s], f);
        if (atomicAdd(&hcnt[s], 1) == 2) {
            atomicOr(&m.hdr[HDR_ERR], MESH_ERR_NONMANIFOLD);
            atomicAdd(&m.hdr[HDR_NONMANIFOLD], 1);
        }
    }
}

__global__ void __launch_bounds__(kB) k_adj_lookup(MeshView m, const unsigned long long* keys,
                                                   const int* hcnt, const int* hsum, int hbits) {
    const int F = min(m.hdr[HDR_F], m.MT);
    const uint32_t hmask = (1u << hbits) - 1u;
    for (int x = blockIdx.x * kB + threadIdx.x; x < 3 * F; x += gridDim.x * kB) {
        int f = x / 3, e = x - 3 * f;
        unsigned long long key = edge_key(m.faces[3 * f + e], m.faces[3 * f + (e + 1) % 3]);
        uint32_t s = hslot(key, hbits);
        int other = -1;
        for (uint32_t probe = 0; probe <= hmask; ++probe) {
            unsigned long long k = keys[s];
            if (k == key) {
                if (hcnt[s] == 2) other = hsum[s] - f;
                break;
            }
            if (k == kEmpty) break;
            s = (s + 1) & hmask;
        }
        float w = 0.0f;
        if (other >= 0) {
            const float* ni = m.normal + 3 * f;
            const float* nj = m.normal + 3 * other;
            w = fmaxf(0.0f, ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2]);
        }
        m.nbr[x] = other;
        m.nbrw[x] = w;
    }
}

__device__ __forceinline__ int delta(const uint32_t* code, int L, int i, int j) {
    if (j < 0 || j >= L) return -1;
    return __clz(code[i] ^ code[j]);
}

// Karras (2012) radix-tree construction over the Morton-ordered leaves.  Child links: internal
// node i >= 0, leaf l as ~l, each followed by its traversal ref (leaf_ref for a leaf).  Parent
// links store (parent << 1) | slot.
__global__ void __launch_bounds__(kB) k_bvh_internal(MeshView m) {
    const int L = min(m.hdr[HDR_L], m.MT);
    const uint32_t* code = m.leaf_code;
    for (int i = blockIdx.x * kB + threadIdx.x; i < L - 1; i += gridDim.x * kB) {
        int d = (delta(code, L, i, i + 1) - delta(code, L, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = delta(code, L, i, i - d);
        int lmax = 2;
        while (delta(code, L, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(code, L, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dn = delta(code, L, i, j);
        int s = 0, t, div = 2;
        do {
            t = (l + div - 1) / div;
            if (delta(code, L, i, i + (s + t) * d) > dn) s += t;
            div <<= 1;
        } while (t > 1);
        int gamma = i + s * d + min(d, 0);
        int left = (min(i, j) == gamma) ? ~gamma : gamma;
        int right = (max(i, j) == gamma + 1) ? ~(gamma + 1) : gamma + 1;
        const int tl = left < 0 ? leaf_ref(m, ~left) : left;
        const int tr = right < 0 ? leaf_ref(m, ~right) : right;
        m.nodes[4 * i + 3] = make_float4(__int_as_float(left), __int_as_float(right),
                                         __int_as_float(tl), __int_as_float(tr));
        if (left < 0) m.parent[m.MT + ~left] = (i << 1) | 0;
        else m.parent[left] = (i << 1) | 0;
        if (right < 0) m.parent[m.MT + ~right] = (i << 1) | 1;
        else m.parent[right] = (i << 1) | 1;
        if (i == 0) m.parent[0] = -1;
    }
}

__device__ __forceinline__ float pad_lo(float v) { return v - (1.0e-6f * fabsf(v) + 1.0e-5f); }
__device__ __forceinline__ float pad_hi(float v) { return v + (1.0e-6f * fabsf(v) + 1.0e-5f); }

__device__ __forceinline__ void write_slot(float4* nodes, int p, int slot, const float lo[3],
                                           const float hi[3]) {
    float* n = reinterpret_cast<float*>(nodes + 4 * p);
    if (slot == 0) {
        n[0] = lo[0]; n[1] = hi[0]; n[2] = lo[1]; n[3] = hi[1];
        n[8] = lo[2]; n[9] = hi[2];
    } else {
        n[4] = lo[0]; n[5] = hi[0]; n[6] = lo[1]; n[7] = hi[1];
        n[10] = lo[2]; n[11] = hi[2];
    }
}

// Leaf boxes (padded so the float32 slab test never rejects a box whose faces the watertight
// triangle test would hit) and the bottom-up union; the second child to arrive at a node
// completes it.
__global__ void __launch_bounds__(kB) k_bvh_refit(MeshView m) {
    const int L = min(m.hdr[HDR_L], m.MT);
    for (int l = blockIdx.x * kB + threadIdx.x; l < L; l += gridDim.x * kB) {
        const int Fc = min(m.hdr[HDR_F], m.MT);
        int f0 = min(m.leaf_start[l], Fc), f1 = min(m.leaf_start[l + 1], Fc);
        float lo[3] = {3.0e38f, 3.0e38f, 3.0e38f}, hi[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
        for (int f = f0; f < f1; ++f)
            for (int v = 0; v < 3; ++v) {
                float4 p = m.tri[3 * f + v];
                lo[0] = fminf(lo[0], p.x); hi[0] = fmaxf(hi[0], p.x);
                lo[1] = fminf(lo[1], p.y); hi[1] = fmaxf(hi[1], p.y);
                lo[2] = fminf(lo[2], p.z); hi[2] = fmaxf(hi[2], p.z);
            }
        for (int q = 0; q < 3; ++q) {
            lo[q] = pad_lo(lo[q]);
            hi[q] = pad_hi(hi[q]);
        }
        int link = (L == 1) ? -1 : m.parent[m.MT + l];
        for (int guard = 0; guard < 64; ++guard) {
            if (link < 0) {
                for (int q = 0; q < 3; ++q) {
                    m.hdr[HDR_ROOTBOX + q] = __float_as_int(lo[q]);
                    m.hdr[HDR_ROOTBOX + 3 + q] = __float_as_int(hi[q]);
                }
                break;
            }
            int p = link >> 1;
            write_slot(m.nodes, p, link & 1, lo, hi);
            __threadfence();
            if (atomicAdd(&m.flags[p], 1) == 0) break;
            __threadfence();
            const float* n = reinterpret_cast<const float*>(m.nodes + 4 * p);
            float b0lx = __ldcg(n + 0), b0hx = __ldcg(n + 1), b0ly = __ldcg(n + 2), b0hy = __ldcg(n + 3);
            float b1lx = __ldcg(n + 4), b1hx = __ldcg(n + 5), b1ly = __ldcg(n + 6), b1hy = __ldcg(n + 7);
            float b0lz = __ldcg(n + 8), b0hz = __ldcg(n + 9), b1lz = __ldcg(n + 10), b1hz = __ldcg(n + 11);
            lo[0] = fminf(b0lx, b1lx); hi[0] = fmaxf(b0hx, b1hx);
            lo[1] = fminf(b0ly, b1ly); hi[1] = fmaxf(b0hy, b1hy);
            lo[2] = fminf(b0lz, b1lz); hi[2] = fmaxf(b0hz, b1hz);
            link = m.parent[p];
        }
    }
}

// ---- 8-wide BVH: greedy top-down collapse of the binary tree, one launch per level ----------
// Each wide node starts from one binary node's two children and repeatedly opens the internal
// child with the largest box surface area until it holds 8 children or only leaves remain; its
// internal children become the next level's wide nodes.  Levels are BFS-ordered, so the top of
// the tree is a prefix of the node array (staged in shared memory by the tracers).

struct Box {
    float lo[3], hi[3];
};

__device__ __forceinline__ Box slot_box(const float4* nodes, int p, int slot) {
    const float* n = reinterpret_cast<const float*>(nodes + 4 * p);
    Box b;
    if (slot == 0) {
        b.lo[0] = n[0]; b.hi[0] = n[1]; b.lo[1] = n[2]; b.hi[1] = n[3]; b.lo[2] = n[8]; b.hi[2] = n[9];
    } else {
        b.lo[0] = n[4]; b.hi[0] = n[5]; b.lo[1] = n[6]; b.hi[1] = n[7]; b.lo[2] = n[10]; b.hi[2] = n[11];
    }
    return b;
}

__device__ __forceinline__ float box_area(const Box& b) {
    float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
}

// Quantise `nc` child boxes into node w.
__device__ void write_wnode(WNode* out, const Box* cb, const int* ref, int nc) {
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    for (int k = 0; k < nc; ++k)
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], cb[k].lo[a]);
            hi[a] = fmaxf(hi[a], cb[k].hi[a]);
        }
    int eb[3];
    double p[3], sc[3];
    for (int a = 0; a < 3; ++a) {
        // scale s = 2^e with the node's extent in <= 255 quanta from a float origin p <= lo
        double ext = (double)hi[a] - (double)lo[a];
        int e = -60;
        if (ext > 0.0) frexp(ext / 255.0, &e);
        e = max(e, -60);
        double s = 0.0, pf = 0.0;
        for (int tries = 0; tries < 4; ++tries, ++e) {
            s = ldexp(1.0, e);
            float pa = (float)(floor((double)lo[a] / s) * s);
            if ((double)pa > (double)lo[a]) pa = nextafterf(pa, -3e38f);
            pf = (double)pa;
            if (ceil(((double)hi[a] - pf) / s) <= 255.0) break;
        }
        p[a] = pf;
        sc[a] = s;
        eb[a] = min(max(e + 127, 1), 254);
    }
    uint8_t q[48];
    for (int k = 0; k < 8; ++k)
        for (int a = 0; a < 3; ++a) {
            uint8_t ql = 0, qh = 0;
            if (k < nc) {
                double l = floor(((double)cb[k].lo[a] - p[a]) / sc[a]);
                double h = ceil(((double)cb[k].hi[a] - p[a]) / sc[a]);
                ql = (uint8_t)fmin(fmax(l, 0.0), 255.0);
                qh = (uint8_t)fmin(fmax(h, 0.0), 255.0);
            }
            q[16 * a + k] = ql;
            q[16 * a + 8 + k] = qh;
        }
    WNode n;
    n.px = (float)p[0];
    n.py = (float)p[1];
    n.pz = (float)p[2];
    n.meta = (uint32_t)eb[0] | ((uint32_t)eb[1] << 8) | ((uint32_t)eb[2] << 16) | ((uint32_t)nc << 24);
    for (int w = 0; w < 12; ++w)
        n.q[w] = (uint32_t)q[4 * w] | ((uint32_t)q[4 * w + 1] << 8) | ((uint32_t)q[4 * w + 2] << 16) |
                 ((uint32_t)q[4 * w + 3] << 24);
    for (int k = 0; k < 8; ++k) n.child[k] = k < nc ? ref[k] : 0;
    *out = n;
}

__global__ void k_wide_init(MeshView m) {
    const int L = min(m.hdr[HDR_L], m.MT);
    m.hdr[HDR_WC + 0] = 0;
    m.hdr[HDR_WC + 1] = 0;
    m.hdr[HDR_WC + 2] = 0;
    m.hdr[HDR_WLEVELS] = 0;
    if (L <= 0) {
        m.hdr[HDR_WN] = 0;
        return;
    }
    if (L == 1) {
        Box b;
        for (int a = 0; a < 3; ++a) {
            b.lo[a] = __int_as_float(m.hdr[HDR_ROOTBOX + a]);
            b.hi[a] = __int_as_float(m.hdr[HDR_ROOTBOX + 3 + a]);
        }
        int r = leaf_ref(m, 0);
        write_wnode(m.wnodes, &b, &r, 1);
        m.hdr[HDR_WN] = 1;
        m.hdr[HDR_WLEVELS] = 1;
        return;
    }
    m.wfront[0] = make_int2(0, 0);
    m.hdr[HDR_WC + 0] = 1;
    m.hdr[HDR_WN] = 1;
}

__global__ void __launch_bounds__(128) k_wide_level(MeshView m, int level) {
    int* cin = &m.hdr[HDR_WC + level % 3];
    int* cout = &m.hdr[HDR_WC + (level + 1) % 3];
    const int n = *cin;
    if (n == 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        m.hdr[HDR_WC + (level + 2) % 3] = 0;
        atomicMax(&m.hdr[HDR_WLEVELS], level + 1);
    }
    const int2* fin = m.wfront + (long long)(level % 3) * m.MT;
    int2* fout = m.wfront + (long long)((level + 1) % 3) * m.MT;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int2 it = fin[i];
        int b = it.x, w = it.y;
        Box cb[8];
        int ref[8];
        float area[8];
        float4 l = m.nodes[4 * b + 3];
        ref[0] = __float_as_int(l.x);
        ref[1] = __float_as_int(l.y);
        cb[0] = slot_box(m.nodes, b, 0);
        cb[1] = slot_box(m.nodes, b, 1);
        area[0] = box_area(cb[0]);
        area[1] = box_area(cb[1]);
        int nc = 2;
        while (nc < 8) {
            int best = -1;
            float ba = -1.0f;
            for (int k = 0; k < nc; ++k)
                if (ref[k] >= 0 && area[k] > ba) {
                    ba = area[k];
                    best = k;
                }
            if (best < 0) break;
            int bn = ref[best];
            float4 ll = m.nodes[4 * bn + 3];
            ref[best] = __float_as_int(ll.x);
            cb[best] = slot_box(m.nodes, bn, 0);
            area[best] = box_area(cb[best]);
            ref[nc] = __float_as_int(ll.y);
            cb[nc] = slot_box(m.nodes, bn, 1);
            area[nc] = box_area(cb[nc]);
            ++nc;
        }
        int nint = 0;
        for (int k = 0; k < nc; ++k) nint += ref[k] >= 0;
        int base = nint ? atomicAdd(&m.hdr[HDR_WN], nint) : 0;
        int fpos = nint ? atomicAdd(cout, nint) : 0;
        int out[8];
        int r = 0;
        for (int k = 0; k < nc; ++k) {
            if (ref[k] >= 0) {
                int wi = base + r;
                if (wi < m.MT && fpos + r < m.MT) {
                    fout[fpos + r] = make_int2(ref[k], wi);
                    out[k] = wi;
                } else {
                    out[k] = -1;   // capacity cannot be exceeded (wide nodes <= binary nodes)
                    atomicOr(&m.hdr[HDR_ERR], MESH_ERR_TRI_OVERFLOW);
                }
                ++r;
            } else {
                out[k] = leaf_ref(m, ~ref[k]);
            }
        }
        write_wnode(m.wnodes + w, cb, out, nc);
    }
}

struct Scratch {
    uint16_t* info;
    int* bflag;      // per Morton block of kB nodes: some node emits a vertex or a face
    uint32_t* voff;
    int4* bsum;
    int4* boff;
    void* cub_tmp;
    size_t cub_bytes;
    unsigned long long* hkeys;
    int* hf0;
    int* hf1;
    int hbits;
    long long total;
};

int hash_bits(int MT) {
    int b = ceil_log2(6 * (MT > 1 ? MT : 1));
    return b < 8 ? 8 : b;
}

int scratch_layout(int nx, int ny, int nz, int MT, char* base, Scratch* s, bool* morton_ok) {
    Morton mo = make_morton(nx, ny, nz, morton_ok);
    if (!*morton_ok) return PETCH_E_INVALID;
    long long npad = 1LL << mo.nbits;
    long long nb = (npad + kB - 1) / kB;
    size_t cub_bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveScan(nullptr, cub_bytes, (int4*)nullptr,
                                                   (int4*)nullptr, Int4Add(), make_int4(0, 0, 0, 0),
                                                   (int)nb);
    if (e != cudaSuccess) return cuda_fail(e, "cub scan size query");
    int hb = hash_bits(MT);
    long long H = 1LL << hb;
    long long o = 0;
    auto take = [&](long long bytes) {
        long long at = o;
        o += align256(bytes);
        return base ? base + at : nullptr;
    };
    s->info = (uint16_t*)take(2 * npad);
    s->bflag = (int*)take(4 * nb);
    s->voff = (uint32_t*)take(4 * npad);
    s->bsum = (int4*)take(16 * nb);
    s->boff = (int4*)take(16 * nb);
    s->cub_tmp = take((long long)cub_bytes);
    s->cub_bytes = cub_bytes;
    s->hkeys = (unsigned long long*)take(8 * H);
    s->hf0 = (int*)take(4 * H);
    s->hf1 = (int*)take(4 * H);
    s->hbits = hb;
    s->total = o;
    return PETCH_OK;
}

}  // namespace
}  // namespace petch

using namespace petch;

extern "C" int petch_mesh_layout(int max_tris, int max_verts, long long* offsets, int n_offsets,
                                 long long* total_bytes) {
    PETCH_REQUIRE(max_tris > 0 && max_verts > 0, "petch_mesh_layout: capacities must be > 0");
    PETCH_REQUIRE(max_tris < (1 << 28), "petch_mesh_layout: max_tris must be below 2^28");
    MeshLayout L = mesh_layout(max_tris, max_verts);
    if (offsets)
        for (int s = 0; s < n_offsets && s < SEG_COUNT; ++s) offsets[s] = L.off[s];
    if (total_bytes) *total_bytes = L.total;
    return PETCH_OK;
}

extern "C" int petch_mesh_scratch_bytes(int nx, int ny, int nz, int max_tris, long long* bytes) {
    PETCH_REQUIRE(bytes, "petch_mesh_scratch_bytes: null pointer");
    PETCH_REQUIRE(nx > 1 && ny > 1 && nz > 1 && max_tris > 0, "petch_mesh_scratch_bytes: bad size");
    Scratch s;
    bool ok = false;
    int rc = scratch_layout(nx, ny, nz, max_tris, nullptr, &s, &ok);
    if (!ok) {
        set_error("petch_mesh_scratch_bytes: grid needs more than 31 Morton bits");
        return PETCH_E_INVALID;
    }
    if (rc) return rc;
    *bytes = s.total;
    return PETCH_OK;
}

extern "C" int petch_mesh_build(const float* phi, int nx, int ny, int nz, double dx, double Lx,
                                double Ly, double sub_top, double mask_th, double width, int hole,
                                void* mesh, int max_tris, int max_verts, void* scratch,
                                long long scratch_bytes, void* stream) {
    PETCH_REQUIRE(phi && mesh && scratch, "petch_mesh_build: null pointer");
    PETCH_REQUIRE(nx > 1 && ny > 1 && nz > 1 && dx > 0, "petch_mesh_build: bad grid");
    PETCH_REQUIRE(max_tris > 0 && max_verts > 0, "petch_mesh_build: capacities must be > 0");
    PETCH_REQUIRE(max_tris < (1 << 28), "petch_mesh_build: max_tris must be below 2^28");
    Scratch s;
    bool ok = false;
    int rc = scratch_layout(nx, ny, nz, max_tris, (char*)scratch, &s, &ok);
    if (!ok) {
        set_error("petch_mesh_build: grid needs more than 31 Morton bits");
        return PETCH_E_INVALID;
    }
    if (rc) return rc;
    PETCH_REQUIRE(scratch_bytes >= s.total, "petch_mesh_build: scratch too small (%lld < %lld)",
                  scratch_bytes, s.total);
    cudaStream_t st = as_stream(stream);
    Morton mo = make_morton(nx, ny, nz, &ok);
    uint32_t npad = 1u << mo.nbits;
    int nb = (int)((npad + kB - 1) / kB);
    Dims d{nx, ny, nz, (long long)ny * nz};
    MeshView m = mesh_view(mesh, max_tris, max_verts);

    // the grid-order info lives in voff's space until k_mc_verts writes the vertex offsets
    // (npad >= cells, 4 bytes per node >= 2 bytes per cell)
    uint16_t* info_lin = reinterpret_cast<uint16_t*>(s.voff);
    {
        const int rows = nx * ny;
        const int gb = (rows + kMcRows - 1) / kMcRows;
        k_mc_classify<<<gb, dim3(kMcZ, kMcRows), 0, st>>>(phi, d, mo, info_lin, s.bflag);
        PETCH_LAUNCH_CHECK("k_mc_classify");
    }
    const int pb = grid_for(nb, 1, 8);   // block-stride passes: 8 CTAs per SM at most
    k_mc_count<<<pb, kB, 0, st>>>(info_lin, d, mo, npad, (uint32_t)nb, s.info, s.bsum, s.bflag);
    PETCH_LAUNCH_CHECK("k_mc_count");
    PETCH_CUDA(cub::DeviceScan::ExclusiveScan(s.cub_tmp, s.cub_bytes, s.bsum, s.boff, Int4Add(),
                                              make_int4(0, 0, 0, 0), nb, st),
               "cub exclusive scan");
    k_mc_totals<<<1, 1, 0, st>>>(s.bsum, s.boff, nb, m);
    PETCH_LAUNCH_CHECK("k_mc_totals");
    k_mc_verts<<<pb, kB, 0, st>>>(phi, d, mo, npad, (uint32_t)nb, s.info, s.bsum, s.boff, s.voff,
                                  dx, m);
    PETCH_LAUNCH_CHECK("k_mc_verts");
    k_mc_faces<<<pb, kB, 0, st>>>(d, mo, npad, (uint32_t)nb, s.info, s.bsum, s.boff, s.voff, m);
    PETCH_LAUNCH_CHECK("k_mc_faces");

    FaceParams fp{dx, Lx, Ly, sub_top, mask_th, width, hole};
    int fb = grid_for(max_tris, kB);
    k_face_geometry<<<fb, kB, 0, st>>>(m, fp);
    PETCH_LAUNCH_CHECK("k_face_geometry");

    long long H = 1LL << s.hbits;
    PETCH_CUDA(cudaMemsetAsync(s.hkeys, 0xff, 8 * H, st), "memset hash keys");
    PETCH_CUDA(cudaMemsetAsync(s.hf0, 0, 4 * H, st), "memset hash counts");
    PETCH_CUDA(cudaMemsetAsync(s.hf1, 0, 4 * H, st), "memset hash sums");
    int eb = grid_for(3LL * max_tris, kB);
    k_adj_insert<<<eb, kB, 0, st>>>(m, s.hkeys, s.hf0, s.hf1, s.hbits);
    PETCH_LAUNCH_CHECK("k_adj_insert");
    k_adj_lookup<<<eb, kB, 0, st>>>(m, s.hkeys, s.hf0, s.hf1, s.hbits);
    PETCH_LAUNCH_CHECK("k_adj_lookup");

    PETCH_CUDA(cudaMemsetAsync(m.flags, 0, 4LL * max_tris, st), "memset refit flags");
    k_bvh_internal<<<fb, kB, 0, st>>>(m);
    PETCH_LAUNCH_CHECK("k_bvh_internal");
    k_bvh_refit<<<fb, kB, 0, st>>>(m);
    PETCH_LAUNCH_CHECK("k_bvh_refit");
    if (!wide_bvh_enabled()) {
        // no 8-wide tree: WN = 0 and WLEVELS = -1 mark it absent for the wide traversal
        PETCH_CUDA(cudaMemsetAsync(m.hdr + HDR_WN, 0, sizeof(int), st), "memset wide count");
        PETCH_CUDA(cudaMemsetAsync(m.hdr + HDR_WLEVELS, 0xff, sizeof(int), st), "memset wide levels");
        return PETCH_OK;
    }
    k_wide_init<<<1, 1, 0, st>>>(m);
    PETCH_LAUNCH_CHECK("k_wide_init");
    int wb = grid_for(max_tris / 4 + 1, 128);
    for (int level = 0; level < kWideLevels; ++level) {
        k_wide_level<<<wb, 128, 0, st>>>(m, level);
        PETCH_LAUNCH_CHECK("k_wide_level");
    }
    return PETCH_OK;
}
