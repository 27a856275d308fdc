// ORACLE -- test infrastructure only.  FP64 CPU restatement of the surface stages:
//   marching cubes          : extract_mesh_3d(_gpu)            petch/threed.py:62-100
//   per-face geometry       : centroids/areas (:65-68), _face_normals_k (:228-234)
//   faces_in_mask           :                                  petch/threed.py:1608-1616
//   edge adjacency + weights: _edge_adjacency, _edge_weights_k petch/threed.py:103-125, 237-242
//   nearest-face queries    : _extend_kernel, _nearest_face_cov (Warp mesh_query_point_no_sign)
//   closest-hit queries     : Warp mesh_query_ray (closest hit, 0 <= t <= tmax)
//
// Marching cubes follows the triangulation spec of the device library (the reference's Warp/skimage
// tables are third-party and not restated): corner c at offset (c&1, c>>1&1, c>>2&1), solid when
// phi > 0; on each cube face the corners are walked counter-clockwise seen from outside, every sign
// change is a crossing, each solid->gas crossing is joined to the gas->solid crossing before it;
// the segments chain into loops, each loop starts at its lowest cube-edge id (x edges 0-3 by lower
// corner 0,2,4,6; y 4-7 by 0,1,4,5; z 8-11 by 0..3) and is fanned as (l0, l[k+1], l[k]).  Cubes and
// vertices are enumerated in the same generalized Morton order.  This file derives the face cycles
// geometrically at run time (no table), so it checks the device's compile-time table.
// Parity: per-face arithmetic pinned by tests/golden/surface.npz (reference code on oracle meshes).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

struct Morton {
    int nbits = 0;
    int axis[40], level[40];
};

int clog2(int n) {
    int b = 0;
    while ((1LL << b) < n) ++b;
    return b;
}

Morton make_morton(int nx, int ny, int nz) {
    int bits[3] = {clog2(nx), clog2(ny), clog2(nz)};
    Morton m;
    for (int l = 0; l < 32; ++l)
        for (int a = 0; a < 3; ++a)
            if (l < bits[a]) {
                m.axis[m.nbits] = a;
                m.level[m.nbits] = l;
                ++m.nbits;
            }
    return m;
}

void decode(const Morton& m, uint64_t t, int c[3]) {
    c[0] = c[1] = c[2] = 0;
    for (int p = 0; p < m.nbits; ++p) c[m.axis[p]] |= (int)((t >> p) & 1) << m.level[p];
}

}  // namespace

// ---- cube geometry ----
struct V3 {
    double x, y, z;
};

namespace {
V3 corner_pos(int c) { return V3{(double)(c & 1), (double)((c >> 1) & 1), (double)((c >> 2) & 1)}; }

int edge_id(int ca, int cb) {
    int lo = std::min(ca, cb), x = ca ^ cb;
    if (x == 1) return lo / 2;
    if (x == 2) return 4 + (lo & 1) + ((lo >> 2) & 1) * 2;
    return 8 + lo;
}

// Face cycles: the 4 corners of face (axis, side) ordered counter-clockwise as seen from outside,
// found by sorting by angle around the face centre in a frame (u, v) with u x v = outward normal.
struct Cycles {
    int c[6][4];
};

Cycles face_cycles() {
    Cycles cy;
    int f = 0;
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side, ++f) {
            double n[3] = {0, 0, 0};
            n[axis] = side ? 1.0 : -1.0;
            // any u perpendicular to n, v = n x u
            double u[3] = {0, 0, 0};
            u[(axis + 1) % 3] = 1.0;
            double v[3] = {n[1] * u[2] - n[2] * u[1], n[2] * u[0] - n[0] * u[2], n[0] * u[1] - n[1] * u[0]};
            std::vector<std::pair<double, int>> cs;
            for (int c = 0; c < 8; ++c) {
                if (((c >> axis) & 1) != side) continue;
                V3 p = corner_pos(c);
                double d[3] = {p.x - 0.5, p.y - 0.5, p.z - 0.5};
                double a = std::atan2(d[0] * v[0] + d[1] * v[1] + d[2] * v[2], d[0] * u[0] + d[1] * u[1] + d[2] * u[2]);
                cs.push_back({a, c});
            }
            std::sort(cs.begin(), cs.end());
            for (int q = 0; q < 4; ++q) cy.c[f][q] = cs[q].second;
        }
    return cy;
}

// Triangles (as pairs of cube corners per vertex) of configuration cfg.
struct CubeTris {
    int n = 0;
    int e[5][3][2];  // [tri][vertex][corner a, corner b]
};

CubeTris triangulate(int cfg, const Cycles& cy) {
    int seg_to[12];
    int ea[12], eb[12];
    for (int i = 0; i < 12; ++i) seg_to[i] = -1;
    for (int f = 0; f < 6; ++f) {
        int xe[4], xt[4], nc = 0;
        for (int q = 0; q < 4; ++q) {
            int a = cy.c[f][q], b = cy.c[f][(q + 1) % 4];
            bool sa = (cfg >> a) & 1, sb = (cfg >> b) & 1;
            if (sa != sb) {
                int e = edge_id(a, b);
                ea[e] = std::min(a, b);
                eb[e] = std::max(a, b);
                xe[nc] = e;
                xt[nc] = sa ? 1 : 0;
                ++nc;
            }
        }
        for (int q = 0; q < nc; ++q)
            if (xt[q]) seg_to[xe[q]] = xe[(q + nc - 1) % nc];
    }
    CubeTris t;
    bool used[12] = {false};
    for (int e0 = 0; e0 < 12; ++e0) {
        if (seg_to[e0] < 0 || used[e0]) continue;
        int loop[12], m = 0, e = e0;
        while (!used[e]) {
            used[e] = true;
            loop[m++] = e;
            e = seg_to[e];
        }
        for (int k = 1; k + 1 < m; ++k) {
            int vv[3] = {loop[0], loop[k + 1], loop[k]};
            for (int s = 0; s < 3; ++s) {
                t.e[t.n][s][0] = ea[vv[s]];
                t.e[t.n][s][1] = eb[vv[s]];
            }
            ++t.n;
        }
    }
    return t;
}

}  // namespace

// ---- mesh object ----
struct Node {
    double lo[3], hi[3];
    int left, right;   // children (internal) ; for leaves left = first prim index, right = -count
};

struct Mesh {
    int nx, ny, nz;
    double dx;
    std::vector<double> vnode;   // 3 * V, node units
    std::vector<double> verts;   // 3 * V, physical (double of float32(vnode * dx))
    std::vector<int> faces;      // 3 * F
    std::vector<double> area, normal, centroid;
    std::vector<uint8_t> fmask;
    std::vector<int> nbr;
    std::vector<double> nbrw;
    std::vector<int> cube_of_face;
    // BVH over faces
    std::vector<Node> nodes;
    std::vector<int> prim;
};

namespace {

void tri_verts(const Mesh& m, int f, V3 p[3]) {
    for (int s = 0; s < 3; ++s) {
        int v = m.faces[3 * f + s];
        p[s] = V3{m.verts[3 * v], m.verts[3 * v + 1], m.verts[3 * v + 2]};
    }
}

void build_bvh(Mesh& m) {
    int F = (int)m.area.size();
    m.prim.resize(F);
    for (int i = 0; i < F; ++i) m.prim[i] = i;
    m.nodes.clear();
    if (F == 0) return;
    std::vector<double> cen(3 * (size_t)F), blo(3 * (size_t)F), bhi(3 * (size_t)F);
    for (int f = 0; f < F; ++f) {
        V3 p[3];
        tri_verts(m, f, p);
        double xs[3] = {p[0].x, p[1].x, p[2].x}, ys[3] = {p[0].y, p[1].y, p[2].y}, zs[3] = {p[0].z, p[1].z, p[2].z};
        blo[3 * f] = std::min({xs[0], xs[1], xs[2]});
        bhi[3 * f] = std::max({xs[0], xs[1], xs[2]});
        blo[3 * f + 1] = std::min({ys[0], ys[1], ys[2]});
        bhi[3 * f + 1] = std::max({ys[0], ys[1], ys[2]});
        blo[3 * f + 2] = std::min({zs[0], zs[1], zs[2]});
        bhi[3 * f + 2] = std::max({zs[0], zs[1], zs[2]});
        for (int q = 0; q < 3; ++q) cen[3 * f + q] = 0.5 * (blo[3 * f + q] + bhi[3 * f + q]);
    }
    struct Job {
        int node, b, e;
    };
    m.nodes.push_back(Node{});
    std::vector<Job> st{{0, 0, F}};
    while (!st.empty()) {
        Job j = st.back();
        st.pop_back();
        Node nd;
        for (int q = 0; q < 3; ++q) {
            nd.lo[q] = 1e300;
            nd.hi[q] = -1e300;
        }
        for (int i = j.b; i < j.e; ++i)
            for (int q = 0; q < 3; ++q) {
                nd.lo[q] = std::min(nd.lo[q], blo[3 * m.prim[i] + q]);
                nd.hi[q] = std::max(nd.hi[q], bhi[3 * m.prim[i] + q]);
            }
        if (j.e - j.b <= 4) {
            nd.left = j.b;
            nd.right = -(j.e - j.b);
            m.nodes[j.node] = nd;
            continue;
        }
        int ax = 0;
        double ext = -1;
        for (int q = 0; q < 3; ++q)
            if (nd.hi[q] - nd.lo[q] > ext) {
                ext = nd.hi[q] - nd.lo[q];
                ax = q;
            }
        int mid = (j.b + j.e) / 2;
        std::nth_element(m.prim.begin() + j.b, m.prim.begin() + mid, m.prim.begin() + j.e,
                         [&](int a, int b) { return cen[3 * a + ax] < cen[3 * b + ax]; });
        int l = (int)m.nodes.size();
        m.nodes.push_back(Node{});
        m.nodes.push_back(Node{});
        nd.left = l;
        nd.right = l + 1;
        m.nodes[j.node] = nd;
        st.push_back({l, j.b, mid});
        st.push_back({l + 1, mid, j.e});
    }
}

}  // namespace

// exported helpers for the flux oracle (same translation unit family)
namespace orc {

struct HitD {
    double t;
    int f;
};

// Moller-Trumbore in double; closest hit with 0 <= t <= tmax.
HitD closest_hit(const Mesh* m, const double o[3], const double d[3], double tmax) {
    HitD h{tmax, -1};
    if (m->nodes.empty()) return h;
    double inv[3];
    for (int q = 0; q < 3; ++q) inv[q] = 1.0 / (std::fabs(d[q]) > 1e-300 ? d[q] : std::copysign(1e-300, d[q]));
    int stack[128], sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node& n = m->nodes[stack[--sp]];
        double tn = 0.0, tf = h.t;
        for (int q = 0; q < 3; ++q) {
            double t0 = (n.lo[q] - o[q]) * inv[q], t1 = (n.hi[q] - o[q]) * inv[q];
            if (t0 > t1) std::swap(t0, t1);
            tn = std::max(tn, t0);
            tf = std::min(tf, t1 * (1 + 1e-12) + 1e-12);
        }
        if (tn > tf) continue;
        if (n.right <= 0) {
            for (int i = n.left; i < n.left - n.right; ++i) {
                int f = m->prim[i];
                V3 p[3];
                tri_verts(*m, f, p);
                double e1[3] = {p[1].x - p[0].x, p[1].y - p[0].y, p[1].z - p[0].z};
                double e2[3] = {p[2].x - p[0].x, p[2].y - p[0].y, p[2].z - p[0].z};
                double pv[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
                double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
                if (det == 0.0) continue;
                double inv_det = 1.0 / det;
                double s[3] = {o[0] - p[0].x, o[1] - p[0].y, o[2] - p[0].z};
                double u = (s[0] * pv[0] + s[1] * pv[1] + s[2] * pv[2]) * inv_det;
                if (u < 0.0 || u > 1.0) continue;
                double qv[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
                double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) * inv_det;
                if (v < 0.0 || u + v > 1.0) continue;
                double t = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) * inv_det;
                if (t >= 0.0 && (t < h.t || (t == h.t && h.f >= 0 && f < h.f))) {
                    h.t = t;
                    h.f = f;
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return h;
}

double point_tri_d2(const double p[3], const V3 t[3]) {
    // Ericson, Real-Time Collision Detection 5.1.5, in double
    double a[3] = {t[0].x, t[0].y, t[0].z}, b[3] = {t[1].x, t[1].y, t[1].z}, c[3] = {t[2].x, t[2].y, t[2].z};
    auto sub = [](const double* x, const double* y, double* r) { for (int q = 0; q < 3; ++q) r[q] = x[q] - y[q]; };
    auto dot = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    double ab[3], ac[3], ap[3], bp[3], cp[3], q[3];
    sub(b, a, ab); sub(c, a, ac); sub(p, a, ap);
    double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) { memcpy(q, a, sizeof q); }
    else {
        sub(p, b, bp);
        double d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0 && d4 <= d3) { memcpy(q, b, sizeof q); }
        else {
            double vc = d1 * d4 - d3 * d2;
            if (vc <= 0 && d1 >= 0 && d3 <= 0) { double v = d1 / (d1 - d3); for (int k = 0; k < 3; ++k) q[k] = a[k] + v * ab[k]; }
            else {
                sub(p, c, cp);
                double d5 = dot(ab, cp), d6 = dot(ac, cp);
                if (d6 >= 0 && d5 <= d6) { memcpy(q, c, sizeof q); }
                else {
                    double vb = d5 * d2 - d1 * d6;
                    if (vb <= 0 && d2 >= 0 && d6 <= 0) { double w = d2 / (d2 - d6); for (int k = 0; k < 3; ++k) q[k] = a[k] + w * ac[k]; }
                    else {
                        double va = d3 * d6 - d5 * d4;
                        if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
                            double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                            for (int k = 0; k < 3; ++k) q[k] = b[k] + w * (c[k] - b[k]);
                        } else {
                            double den = 1.0 / (va + vb + vc), v = vb * den, w = vc * den;
                            for (int k = 0; k < 3; ++k) q[k] = a[k] + v * ab[k] + w * ac[k];
                        }
                    }
                }
            }
        }
    }
    double dd[3];
    sub(p, q, dd);
    return dot(dd, dd);
}

// Nearest face (ties to the lower index) within sqrt(r2max); -1 if none.
int nearest_face(const Mesh* m, const double p[3], double r2max) {
    int best = -1;
    double bd = r2max;
    if (m->nodes.empty()) return -1;
    int stack[128], sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Node& n = m->nodes[stack[--sp]];
        double e = 0;
        for (int q = 0; q < 3; ++q) {
            double g = std::max(std::max(n.lo[q] - p[q], 0.0), p[q] - n.hi[q]);
            e += g * g;
        }
        if (e > bd) continue;
        if (n.right <= 0) {
            for (int i = n.left; i < n.left - n.right; ++i) {
                int f = m->prim[i];
                V3 t[3];
                tri_verts(*m, f, t);
                double d2 = point_tri_d2(p, t);
                if (d2 < bd || (d2 == bd && (best < 0 || f < best))) {
                    bd = d2;
                    best = f;
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    return best;
}

void face_normal(const Mesh* m, int f, double n[3]) {
    n[0] = m->normal[3 * f];
    n[1] = m->normal[3 * f + 1];
    n[2] = m->normal[3 * f + 2];
}

}  // namespace orc

extern "C" {

// Marching cubes + geometry + adjacency + BVH.  phi is float32 (the device's input precision).
void* orc_mesh_build(const float* phi, int nx, int ny, int nz, double dx, double Lx, double Ly,
                     double sub_top, double mask_th, double width, int hole) {
    Mesh* m = new Mesh;
    m->nx = nx;
    m->ny = ny;
    m->nz = nz;
    m->dx = dx;
    Morton mo = make_morton(nx, ny, nz);
    uint64_t npad = 1ULL << mo.nbits;
    long long plane = (long long)ny * nz;
    auto at = [&](int i, int j, int k) { return (long long)i * plane + (long long)j * nz + k; };
    Cycles cy = face_cycles();
    std::vector<CubeTris> table(256);
    for (int c = 0; c < 256; ++c) table[c] = triangulate(c, cy);
    std::vector<int> vid(3 * (size_t)nx * ny * nz, -1);
    // pass 1: vertices on crossed owned edges, nodes in Morton order, axes x, y, z
    for (uint64_t t = 0; t < npad; ++t) {
        int c3[3];
        decode(mo, t, c3);
        int i = c3[0], j = c3[1], k = c3[2];
        if (i >= nx || j >= ny || k >= nz) continue;
        float va = phi[at(i, j, k)];
        for (int a = 0; a < 3; ++a) {
            int ii = i + (a == 0), jj = j + (a == 1), kk = k + (a == 2);
            if (ii >= nx || jj >= ny || kk >= nz) continue;
            float vb = phi[at(ii, jj, kk)];
            if ((va > 0.0f) == (vb > 0.0f)) continue;
            float tt = va / (va - vb);      // float32, as the device interpolates
            float p[3] = {(float)i, (float)j, (float)k};
            p[a] = p[a] + tt;
            vid[3 * at(i, j, k) + a] = (int)(m->vnode.size() / 3);
            for (int q = 0; q < 3; ++q) {
                m->vnode.push_back((double)p[q]);
                m->verts.push_back((double)(float)((double)p[q] * dx));
            }
        }
    }
    // pass 2: faces, cubes in Morton order
    for (uint64_t t = 0; t < npad; ++t) {
        int c3[3];
        decode(mo, t, c3);
        int i = c3[0], j = c3[1], k = c3[2];
        if (i >= nx - 1 || j >= ny - 1 || k >= nz - 1) continue;
        int cfg = 0;
        for (int c = 0; c < 8; ++c)
            if (phi[at(i + (c & 1), j + ((c >> 1) & 1), k + ((c >> 2) & 1))] > 0.0f) cfg |= 1 << c;
        const CubeTris& ct = table[cfg];
        for (int q = 0; q < ct.n; ++q) {
            for (int s = 0; s < 3; ++s) {
                int ca = ct.e[q][s][0], cb = ct.e[q][s][1];
                int axis = (ca ^ cb) == 1 ? 0 : ((ca ^ cb) == 2 ? 1 : 2);
                int oi = i + (ca & 1), oj = j + ((ca >> 1) & 1), ok = k + ((ca >> 2) & 1);
                m->faces.push_back(vid[3 * at(oi, oj, ok) + axis]);
            }
            m->cube_of_face.push_back((int)at(i, j, k));
        }
    }
    int F = (int)m->faces.size() / 3;
    m->area.resize(F);
    m->normal.resize(3 * (size_t)F);
    m->centroid.resize(3 * (size_t)F);
    m->fmask.resize(F);
    for (int f = 0; f < F; ++f) {
        double a[3], b[3], c[3];
        for (int q = 0; q < 3; ++q) {
            a[q] = m->vnode[3 * m->faces[3 * f] + q] * dx;
            b[q] = m->vnode[3 * m->faces[3 * f + 1] + q] * dx;
            c[q] = m->vnode[3 * m->faces[3 * f + 2] + q] * dx;
        }
        double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        double ln = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        m->area[f] = std::max(0.5 * ln, 1e-9);
        // winding normal as the reference's device path defines it (_face_normals_k on the
        // float32 vertices, in float32): normalize(cross(b - a, c - a))
        float af[3], bf[3], cf[3];
        for (int q = 0; q < 3; ++q) {
            af[q] = (float)m->verts[3 * m->faces[3 * f] + q];
            bf[q] = (float)m->verts[3 * m->faces[3 * f + 1] + q];
            cf[q] = (float)m->verts[3 * m->faces[3 * f + 2] + q];
        }
        float uf[3] = {bf[0] - af[0], bf[1] - af[1], bf[2] - af[2]};
        float wf[3] = {cf[0] - af[0], cf[1] - af[1], cf[2] - af[2]};
        float nf[3] = {uf[1] * wf[2] - uf[2] * wf[1], uf[2] * wf[0] - uf[0] * wf[2], uf[0] * wf[1] - uf[1] * wf[0]};
        float lf = std::sqrt(nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2]);
        float inv = lf > 0.0f ? 1.0f / lf : 0.0f;
        for (int q = 0; q < 3; ++q) {
            m->normal[3 * f + q] = (double)(nf[q] * inv);
            m->centroid[3 * f + q] = (a[q] + b[q] + c[q]) / 3.0;
        }
        double x = m->centroid[3 * f], y = m->centroid[3 * f + 1], z = m->centroid[3 * f + 2];
        bool in_band = z >= sub_top && z < sub_top + mask_th;
        bool opening = hole ? ((x - Lx / 2) * (x - Lx / 2) + (y - Ly / 2) * (y - Ly / 2) < (width / 2) * (width / 2))
                            : (std::fabs(x - Lx / 2) < width / 2);
        m->fmask[f] = (in_band && !opening) ? 1 : 0;
    }
    // adjacency: the other face on each edge (v0v1, v1v2, v2v0); an edge pairs its faces only
    // when it has exactly two (boundary edges and edges of more than two faces give -1)
    std::unordered_map<uint64_t, std::vector<int>> em;
    em.reserve(3 * (size_t)F);
    auto key = [](int a, int b) { return ((uint64_t)(uint32_t)std::min(a, b) << 32) | (uint32_t)std::max(a, b); };
    for (int f = 0; f < F; ++f)
        for (int e = 0; e < 3; ++e) em[key(m->faces[3 * f + e], m->faces[3 * f + (e + 1) % 3])].push_back(f);
    m->nbr.resize(3 * (size_t)F);
    m->nbrw.resize(3 * (size_t)F);
    for (int f = 0; f < F; ++f)
        for (int e = 0; e < 3; ++e) {
            const std::vector<int>& fs = em[key(m->faces[3 * f + e], m->faces[3 * f + (e + 1) % 3])];
            int o = fs.size() == 2 ? (fs[0] == f ? fs[1] : fs[0]) : -1;
            m->nbr[3 * f + e] = o;
            double wv = 0;
            if (o >= 0)
                for (int q = 0; q < 3; ++q) wv += m->normal[3 * f + q] * m->normal[3 * o + q];
            m->nbrw[3 * f + e] = std::max(0.0, wv);
        }
    build_bvh(*m);
    return m;
}

void orc_mesh_free(void* h) { delete (Mesh*)h; }

void orc_mesh_counts(void* h, int* out) {
    Mesh* m = (Mesh*)h;
    out[0] = (int)m->area.size();
    out[1] = (int)m->vnode.size() / 3;
}

// which: 0 vnode(3V) 1 verts(3V) 2 faces(3F,int) 3 area(F) 4 normal(3F) 5 centroid(3F)
//        6 fmask(F,u8) 7 nbr(3F,int) 8 nbrw(3F)
void orc_mesh_get(void* h, int which, void* dst) {
    Mesh* m = (Mesh*)h;
    switch (which) {
        case 0: memcpy(dst, m->vnode.data(), m->vnode.size() * 8); break;
        case 1: memcpy(dst, m->verts.data(), m->verts.size() * 8); break;
        case 2: memcpy(dst, m->faces.data(), m->faces.size() * 4); break;
        case 3: memcpy(dst, m->area.data(), m->area.size() * 8); break;
        case 4: memcpy(dst, m->normal.data(), m->normal.size() * 8); break;
        case 5: memcpy(dst, m->centroid.data(), m->centroid.size() * 8); break;
        case 6: memcpy(dst, m->fmask.data(), m->fmask.size()); break;
        case 7: memcpy(dst, m->nbr.data(), m->nbr.size() * 4); break;
        case 8: memcpy(dst, m->nbrw.data(), m->nbrw.size() * 8); break;
    }
}

// A mesh from explicit arrays (for fixtures built outside marching cubes).
void* orc_mesh_from_arrays(const double* verts, int V, const int* faces, int F) {
    Mesh* m = new Mesh;
    m->dx = 1.0;
    m->verts.assign(verts, verts + 3 * (size_t)V);
    m->vnode = m->verts;
    m->faces.assign(faces, faces + 3 * (size_t)F);
    m->area.resize(F);
    m->normal.resize(3 * (size_t)F);
    m->centroid.resize(3 * (size_t)F);
    m->fmask.assign(F, 0);
    for (int f = 0; f < F; ++f) {
        V3 p[3];
        tri_verts(*m, f, p);
        double u[3] = {p[1].x - p[0].x, p[1].y - p[0].y, p[1].z - p[0].z};
        double w[3] = {p[2].x - p[0].x, p[2].y - p[0].y, p[2].z - p[0].z};
        double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        double ln = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        m->area[f] = std::max(0.5 * ln, 1e-9);
        for (int q = 0; q < 3; ++q) m->normal[3 * f + q] = ln > 0 ? cr[q] / ln : 0.0;
        m->centroid[3 * f] = (p[0].x + p[1].x + p[2].x) / 3;
        m->centroid[3 * f + 1] = (p[0].y + p[1].y + p[2].y) / 3;
        m->centroid[3 * f + 2] = (p[0].z + p[1].z + p[2].z) / 3;
    }
    m->nbr.assign(3 * (size_t)F, -1);
    m->nbrw.assign(3 * (size_t)F, 0.0);
    build_bvh(*m);
    return m;
}

// Closest hits for a batch of rays (tests): face id or -1, and t.
void orc_mesh_raycast(void* h, const double* o, const double* d, int n, int* face, double* t) {
    Mesh* m = (Mesh*)h;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
        orc::HitD r = orc::closest_hit(m, o + 3 * i, d + 3 * i, 1e6);
        face[i] = r.f;
        t[i] = r.t;
    }
}

// Nearest faces for a batch of points (tests and the extension / warm-start oracles).
void orc_mesh_nearest(void* h, const double* p, int n, int* face) {
    Mesh* m = (Mesh*)h;
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) face[i] = orc::nearest_face(m, p + 3 * i, 1e12);
}

}  // extern "C"
