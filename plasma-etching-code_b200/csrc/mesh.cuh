// Device mesh object: one caller-allocated buffer holding the marching-cubes surface, per-face
// geometry, edge adjacency and the BVH, in a fixed structure-of-arrays layout.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace petch {

enum MeshSeg {
    SEG_HDR = 0,     // int32[16]: see HDR_* below
    SEG_VNODE,       // float[3*MV]  vertex position in node-index units (x/dx)
    SEG_VERTS,       // float[3*MV]  vertex position (um), float32(vnode * dx)
    SEG_FACES,       // int32[3*MT]  vertex ids, wound so cross(b-a, c-a) points into the gas
    SEG_TRI,         // float4[3*MT] per-face vertices for the tracer (w unused)
    SEG_AREA,        // float[MT]    max(area, 1e-9)
    SEG_NORMAL,      // float[3*MT]  unit winding normal (0 for degenerate faces)
    SEG_CENTROID,    // float[3*MT]
    SEG_FMASK,       // uint8[MT]    centroid inside the un-etched mask (faces_in_mask)
    SEG_NBR,         // int32[3*MT]  face across edge (v0v1, v1v2, v2v0), -1 if none
    SEG_NBRW,        // float[3*MT]  smoothing weight max(0, n_i . n_j)
    SEG_LEAF_CODE,   // uint32[MT]   Morton index of the leaf's cube
    SEG_LEAF_START,  // int32[MT+1]  first face of each leaf (faces of a cube are contiguous)
    SEG_NODES,       // float4[4*MT] binary BVH internal nodes (two child boxes + links)
    SEG_PARENT,      // int32[2*MT]  parent link: internal i at [i], leaf l at [MT + l]
    SEG_FLAGS,       // int32[MT]    refit arrival counters
    SEG_WNODES,      // WNode[MT]    8-wide quantised BVH (the tracer's acceleration structure)
    SEG_WFRONT,      // int2[3*MT]   collapse frontiers (binary node, wide node)
    SEG_COUNT
};

enum MeshHdr {
    HDR_F = 0,        // faces
    HDR_V = 1,        // vertices
    HDR_L = 2,        // BVH leaves (surface cubes)
    HDR_ERR = 3,      // error bits (MESH_ERR_*)
    HDR_MT = 4,       // face capacity
    HDR_MV = 5,       // vertex capacity
    HDR_NONMANIFOLD = 6,
    HDR_WN = 7,       // wide BVH nodes
    HDR_ROOTBOX = 8,  // float[6] at hdr[8..13]: root bounds lo.xyz, hi.xyz
    HDR_WLEVELS = 14, // wide BVH depth (levels built)
    HDR_WC = 16,      // int[3] at hdr[16..18]: rotating collapse frontier counters
    HDR_INTS = 32
};

// 8-wide BVH node, 96 bytes.  Child a-axis bounds are lo = p_a + qlo * s_a and
// hi = p_a + qhi * s_a with s_a = 2^(e_a - 127) (the biased exponent byte), rounded outward
// when quantised.  child[k] >= 0: internal node index; child[k] < 0: leaf, -(start * 8 + count)
// - 1 with the leaf's faces [start, start + count) (count <= 5).
struct __align__(16) WNode {
    float px, py, pz;
    uint32_t meta;        // ex | ey << 8 | ez << 16 | nchild << 24
    uint32_t q[12];       // bytes: qlo_x[8] qhi_x[8] qlo_y[8] qhi_y[8] qlo_z[8] qhi_z[8]
    int32_t child[8];
};
static_assert(sizeof(WNode) == 96, "WNode must be 96 bytes");

enum MeshErr {
    MESH_ERR_TRI_OVERFLOW = 1,
    MESH_ERR_VERT_OVERFLOW = 2,
    MESH_ERR_HASH_FULL = 4,
    MESH_ERR_NONMANIFOLD = 8
};

struct MeshLayout {
    long long off[SEG_COUNT];
    long long total;
};

MeshLayout mesh_layout(int max_tris, int max_verts);

// Typed view of a mesh buffer.
struct MeshView {
    int* hdr;
    float* vnode;
    float* verts;
    int* faces;
    float4* tri;
    float* area;
    float* normal;
    float* centroid;
    uint8_t* fmask;
    int* nbr;
    float* nbrw;
    uint32_t* leaf_code;
    int* leaf_start;
    float4* nodes;
    int* parent;
    int* flags;
    WNode* wnodes;
    int2* wfront;
    int MT, MV;
};

MeshView mesh_view(void* base, int max_tris, int max_verts);

// Binary BVH internal node i: nodes[4i] = (lo.x, hi.x, lo.y, hi.y) of child 0, nodes[4i + 1] the
// same of child 1, nodes[4i + 2] = (lo.z, hi.z) of child 0 then of child 1, nodes[4i + 3] = the
// two children's links (internal node j as j, leaf l as ~l) followed by their traversal refs
// (internal node j as j, leaf l as leaf_ref(l)).  The traversal ref of a leaf carries its face
// range, so a resumable query reaches the faces without a lookup in leaf_start.

// Traversal ref of leaf l: -(start * 8 + count) - 1 over its faces [start, start + count), clipped
// at the published face count (the encoding of the 8-wide node's leaf children; face capacities
// stay below 2^28).
__device__ __forceinline__ int leaf_ref(const MeshView& m, int l) {
    const int Fc = min(m.hdr[HDR_F], m.MT);
    const int s = min(m.leaf_start[l], Fc), e = min(m.leaf_start[l + 1], Fc);
    return -((s << 3) | (e - s)) - 1;
}

// Whether mesh builds add the 8-wide BVH (the tracer configuration's BVH width is 8).
bool wide_bvh_enabled();

}  // namespace petch
