// Marching-cubes triangulation table, generated at compile time from first principles (no
// hand-written case table):
//
//   * corner c of a cube sits at offset (c & 1, (c >> 1) & 1, (c >> 2) & 1); a corner is SOLID
//     when phi > 0 (petch's convention: phi > 0 is material);
//   * edge ids: 0-3 run along x from corners 0,2,4,6; 4-7 along y from corners 0,1,4,5; 8-11
//     along z from corners 0,1,2,3;
//   * on each of the six cube faces, walk the four corners counter-clockwise as seen from outside
//     the cube; every sign change is a crossing, tagged EXIT (solid -> gas) or ENTRY;
//   * each EXIT is joined to the ENTRY that precedes it on the walk, i.e. every run of solid
//     corners along a face is cut off on its own.  On the ambiguous face (two diagonal solid
//     corners) this separates the solid corners.  The rule depends only on the face's four signs,
//     so the two cubes sharing a face cut it identically: the mesh is watertight and manifold;
//   * a segment runs EXIT -> ENTRY (solid on its left seen from outside); segments chain into
//     closed loops around the cube, and each loop of m crossings is fanned into m - 2 triangles,
//     wound so that the geometric normal cross(b - a, c - a) points into the gas (phi < 0 side).
#pragma once
#include <cstdint>

namespace petch {
namespace mc {

constexpr int kMaxTriPerCube = 5;

struct Table {
    uint8_t ntri[256];
    int8_t tri[256][3 * kMaxTriPerCube];
};

constexpr int edge_between(int ca, int cb) {
    int x = ca ^ cb;
    int lo = ca < cb ? ca : cb;
    if (x == 1) return lo >> 1;                                   // 0,2,4,6 -> 0..3
    if (x == 2) return 4 + (lo & 1) + ((lo >> 2) & 1) * 2;        // 0,1,4,5 -> 4..7
    return 8 + lo;                                                // 0,1,2,3 -> 8..11
}

constexpr int corner_of(int axis, int side, int pu, int pv) {
    int u = (axis + 1) % 3, v = (axis + 2) % 3;
    return (side << axis) | (pu << u) | (pv << v);
}

constexpr Table make_table() {
    Table t{};
    for (int cfg = 0; cfg < 256; ++cfg) {
        int seg_to[12] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};  // from-edge -> to-edge
        for (int axis = 0; axis < 3; ++axis)
            for (int side = 0; side < 2; ++side) {
                // CCW seen from +axis is (0,0),(1,0),(1,1),(0,1) in (u, v); reverse for side 0.
                int cyc[4] = {corner_of(axis, side, 0, 0), corner_of(axis, side, 1, 0),
                              corner_of(axis, side, 1, 1), corner_of(axis, side, 0, 1)};
                if (side == 0) {
                    int a = cyc[1];
                    cyc[1] = cyc[3];
                    cyc[3] = a;
                }
                int xe[4] = {0, 0, 0, 0}, xt[4] = {0, 0, 0, 0};   // crossing edge, 1 = EXIT
                int nc = 0;
                for (int q = 0; q < 4; ++q) {
                    int a = cyc[q], b = cyc[(q + 1) & 3];
                    bool sa = (cfg >> a) & 1, sb = (cfg >> b) & 1;
                    if (sa != sb) {
                        xe[nc] = edge_between(a, b);
                        xt[nc] = sa ? 1 : 0;
                        ++nc;
                    }
                }
                for (int q = 0; q < nc; ++q)
                    if (xt[q] == 1) {
                        int p = (q + nc - 1) % nc;                // the preceding ENTRY
                        seg_to[xe[q]] = xe[p];
                    }
            }
        bool used[12] = {false, false, false, false, false, false,
                         false, false, false, false, false, false};
        int n = 0;
        for (int e0 = 0; e0 < 12; ++e0) {
            if (seg_to[e0] < 0 || used[e0]) continue;
            int loop[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            int m = 0;
            int e = e0;
            while (!used[e]) {
                used[e] = true;
                loop[m++] = e;
                e = seg_to[e];
            }
            // The loop order (EXIT -> ENTRY chaining) winds toward the solid; fan it reversed.
            for (int k = 1; k + 1 < m; ++k) {
                t.tri[cfg][3 * n + 0] = (int8_t)loop[0];
                t.tri[cfg][3 * n + 1] = (int8_t)loop[k + 1];
                t.tri[cfg][3 * n + 2] = (int8_t)loop[k];
                ++n;
            }
        }
        t.ntri[cfg] = (uint8_t)n;
    }
    return t;
}

constexpr bool table_fits() {
    Table t = make_table();
    for (int c = 0; c < 256; ++c)
        if (t.ntri[c] > kMaxTriPerCube) return false;
    return true;
}

// Cube edge -> (owner node offset bits, axis): the node at the edge's lower corner owns it.
__host__ __device__ constexpr int edge_axis(int e) { return e < 4 ? 0 : (e < 8 ? 1 : 2); }
__host__ __device__ constexpr int edge_corner(int e) {
    // lower corner index of the edge
    return e < 4 ? (e << 1) : (e < 8 ? (((e - 4) & 1) | ((((e - 4) >> 1) & 1) << 2)) : (e - 8));
}

}  // namespace mc
}  // namespace petch
