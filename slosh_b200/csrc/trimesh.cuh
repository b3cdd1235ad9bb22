// Triangle-mesh colliders (3D): the packed mesh buffers, their host-side
// construction, and the device point query.
//
// Layout, as slosh's TriMesh (shaders/slosh/collision/trimesh.slang:8-60,
// filled by convert_trimesh_to_gpu, src/trimesh.rs:23-103):
//   vertex buffer (float4 each): [2 per BVH node: AABB min, max]
//                                [mesh vertices] [vertex pseudo-normals]
//                                [3 per triangle: edge pseudo-normals AB, BC, CA]
//   index buffer (u32):          [3 per BVH node: entry, exit, shape]
//                                [3 per triangle: vertex indices]
// The BVH is flattened in depth-first order for stackless traversal: an
// inner node's entry is its first child (the next node), a leaf's entry is
// NONE; exit is the node after the subtree.  slosh builds its BVH with the
// third-party `bvh` crate (SAH); here it is a median split on the longest
// axis of the triangle centroids.  The query's result (the closest surface
// point within the distance cap) does not depend on the tree.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <utility>
#include <vector>

#include "common.cuh"

namespace slosh {

// Offsets and counts of one mesh in the shape record (bit-cast in the floats
// of slosh_body::shape_a / shape_b).
struct TriMeshRef {
    uint32_t vtx_root, idx_root, n_nodes, n_tris, n_verts, ordinal;
};

__host__ __device__ inline TriMeshRef trimesh_ref(const float *sa, const float *sb) {
    TriMeshRef m;
#ifdef __CUDA_ARCH__
    m.vtx_root = __float_as_uint(sa[0]);
    m.idx_root = __float_as_uint(sa[1]);
    m.n_nodes = __float_as_uint(sa[2]);
    m.n_tris = __float_as_uint(sb[0]);
    m.n_verts = __float_as_uint(sb[1]);
    m.ordinal = __float_as_uint(sb[2]);
#else
    std::memcpy(&m.vtx_root, &sa[0], 4);
    std::memcpy(&m.idx_root, &sa[1], 4);
    std::memcpy(&m.n_nodes, &sa[2], 4);
    std::memcpy(&m.n_tris, &sb[0], 4);
    std::memcpy(&m.n_verts, &sb[1], 4);
    std::memcpy(&m.ordinal, &sb[2], 4);
#endif
    return m;
}

// ---- host: mesh buffers ---------------------------------------------------

// Appends the mesh to `vtx` / `idx` and returns its reference.  The vertex
// pseudo-normals are the angle-weighted sums of the incident face normals
// and an edge's pseudo-normal the sum of its faces' normals (Baerentzen and
// Aanaes, "Signed distance computation using the angle weighted
// pseudonormal", 2005), the normals slosh takes from parry.  Returns false
// for out-of-range vertex indices.
inline bool build_trimesh(const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt, std::vector<float4> &vtx,
                          std::vector<uint32_t> &idx, uint32_t ordinal, TriMeshRef &ref) {
    for (uint64_t k = 0; k < 3ull * nt; ++k)
        if (tri[k] >= nv) return false;
    auto P = [&](uint32_t i, int k) { return (double)v[3 * (size_t)i + k]; };
    // BVH over the triangles, one triangle a leaf
    struct Node {
        float mn[3], mx[3];
        uint32_t entry, exit, shape;
    };
    std::vector<Node> nodes;
    nodes.reserve(nt ? 2 * (size_t)nt - 1 : 0);
    std::vector<uint32_t> order(nt);
    std::vector<float> cen(3 * (size_t)nt), tmn(3 * (size_t)nt), tmx(3 * (size_t)nt);
    for (uint32_t t = 0; t < nt; ++t) {
        order[t] = t;
        for (int k = 0; k < 3; ++k) {
            const float a = v[3 * (size_t)tri[3 * t] + k], b = v[3 * (size_t)tri[3 * t + 1] + k],
                        c = v[3 * (size_t)tri[3 * t + 2] + k];
            tmn[3 * t + k] = std::min(a, std::min(b, c));
            tmx[3 * t + k] = std::max(a, std::max(b, c));
            cen[3 * t + k] = (tmn[3 * t + k] + tmx[3 * t + k]) * 0.5f;
        }
    }
    // recursive depth-first construction over order[lo, hi)
    auto build = [&](auto &&self, uint32_t lo, uint32_t hi) -> void {
        const uint32_t id = (uint32_t)nodes.size();
        nodes.push_back(Node{});
        Node nd{};
        for (int k = 0; k < 3; ++k) {
            nd.mn[k] = INFINITY;
            nd.mx[k] = -INFINITY;
        }
        float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t q = lo; q < hi; ++q) {
            const uint32_t t = order[q];
            for (int k = 0; k < 3; ++k) {
                nd.mn[k] = std::min(nd.mn[k], tmn[3 * t + k]);
                nd.mx[k] = std::max(nd.mx[k], tmx[3 * t + k]);
                cmn[k] = std::min(cmn[k], cen[3 * t + k]);
                cmx[k] = std::max(cmx[k], cen[3 * t + k]);
            }
        }
        if (hi - lo == 1) {
            nd.entry = NONE;
            nd.shape = order[lo];
        } else {
            int ax = 0;
            for (int k = 1; k < 3; ++k)
                if (cmx[k] - cmn[k] > cmx[ax] - cmn[ax]) ax = k;
            const uint32_t mid = lo + (hi - lo) / 2;
            std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi,
                             [&](uint32_t a, uint32_t b) {
                                 const float ca = cen[3 * a + ax], cb = cen[3 * b + ax];
                                 return ca < cb || (ca == cb && a < b);
                             });
            nd.entry = id + 1;
            nd.shape = 0;
            nodes[id] = nd;
            self(self, lo, mid);
            self(self, mid, hi);
            nd = nodes[id];
        }
        nd.exit = (uint32_t)nodes.size();
        nodes[id] = nd;
    };
    if (nt) build(build, 0, nt);
    // face normals (unit) and pseudo-normals
    std::vector<double> vpn(3 * (size_t)nv, 0.0);
    std::map<std::pair<uint32_t, uint32_t>, std::array<double, 3>> epn;
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t ia = tri[3 * t], ib = tri[3 * t + 1], ic = tri[3 * t + 2];
        double ab[3], ac[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = P(ib, k) - P(ia, k);
            ac[k] = P(ic, k) - P(ia, k);
        }
        double n[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
        const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > 0)
            for (int k = 0; k < 3; ++k) n[k] /= nn;
        const uint32_t vs[3] = {ia, ib, ic};
        for (int c = 0; c < 3; ++c) {
            const uint32_t p0 = vs[c], p1 = vs[(c + 1) % 3], p2 = vs[(c + 2) % 3];
            double e1[3], e2[3], l1 = 0, l2 = 0, d = 0;
            for (int k = 0; k < 3; ++k) {
                e1[k] = P(p1, k) - P(p0, k);
                e2[k] = P(p2, k) - P(p0, k);
                l1 += e1[k] * e1[k];
                l2 += e2[k] * e2[k];
                d += e1[k] * e2[k];
            }
            const double den = std::sqrt(l1 * l2);
            const double ang = den > 0 ? std::acos(std::max(-1.0, std::min(1.0, d / den))) : 0.0;
            for (int k = 0; k < 3; ++k) vpn[3 * (size_t)p0 + k] += ang * n[k];
            auto key = std::make_pair(std::min(p0, p1), std::max(p0, p1));
            auto &e = epn[key];
            for (int k = 0; k < 3; ++k) e[k] += n[k];
        }
    }
    ref.vtx_root = (uint32_t)vtx.size();
    ref.idx_root = (uint32_t)idx.size();
    ref.n_nodes = (uint32_t)nodes.size();
    ref.n_tris = nt;
    ref.n_verts = nv;
    ref.ordinal = ordinal;
    for (const Node &nd : nodes) {
        vtx.push_back(make_float4(nd.mn[0], nd.mn[1], nd.mn[2], 0.f));
        vtx.push_back(make_float4(nd.mx[0], nd.mx[1], nd.mx[2], 0.f));
        idx.push_back(nd.entry);
        idx.push_back(nd.exit);
        idx.push_back(nd.shape);
    }
    for (uint32_t i = 0; i < nv; ++i) vtx.push_back(make_float4(v[3 * (size_t)i], v[3 * (size_t)i + 1], v[3 * (size_t)i + 2], 0.f));
    for (uint32_t i = 0; i < nv; ++i) {
        double n[3] = {vpn[3 * (size_t)i], vpn[3 * (size_t)i + 1], vpn[3 * (size_t)i + 2]};
        const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > 0)
            for (int k = 0; k < 3; ++k) n[k] /= nn;
        vtx.push_back(make_float4((float)n[0], (float)n[1], (float)n[2], 0.f));
    }
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t vs[3] = {tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]};
        for (int c = 0; c < 3; ++c) {  // edges AB, BC, CA
            const uint32_t p0 = vs[c], p1 = vs[(c + 1) % 3];
            const auto &e = epn[std::make_pair(std::min(p0, p1), std::max(p0, p1))];
            vtx.push_back(make_float4((float)e[0], (float)e[1], (float)e[2], 0.f));
        }
    }
    for (uint32_t t = 0; t < nt; ++t)
        for (int c = 0; c < 3; ++c) idx.push_back(tri[3 * t + c]);
    return true;
}

// ---- device: point query --------------------------------------------------

// Closest point on triangle abc to p by Voronoi regions (Ericson, Real-Time
// Collision Detection, 5.1.5), with the feature it lies on: vertex a/b/c
// (feature 0, id 0/1/2), edge AB/BC/CA (feature 1, id 0/1/2) or the face
// (feature 2), the feature ids of trimesh.slang:214-377.
__device__ __forceinline__ void triangle_closest(const float3 a, const float3 b, const float3 c, const float3 p,
                                                 float3 &q, uint32_t &feat, uint32_t &fid) {
    const float3 ab = make_float3(b.x - a.x, b.y - a.y, b.z - a.z), ac = make_float3(c.x - a.x, c.y - a.y, c.z - a.z);
    const float3 ap = make_float3(p.x - a.x, p.y - a.y, p.z - a.z);
    auto dot3 = [](float3 u, float3 w) { return u.x * w.x + u.y * w.y + u.z * w.z; };
    const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) {
        q = a, feat = 0, fid = 0;
        return;
    }
    const float3 bp = make_float3(p.x - b.x, p.y - b.y, p.z - b.z);
    const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.f && d4 <= d3) {
        q = b, feat = 0, fid = 1;
        return;
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float t = d1 / (d1 - d3);
        q = make_float3(a.x + t * ab.x, a.y + t * ab.y, a.z + t * ab.z), feat = 1, fid = 0;
        return;
    }
    const float3 cp = make_float3(p.x - c.x, p.y - c.y, p.z - c.z);
    const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.f && d5 <= d6) {
        q = c, feat = 0, fid = 2;
        return;
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float t = d2 / (d2 - d6);
        q = make_float3(a.x + t * ac.x, a.y + t * ac.y, a.z + t * ac.z), feat = 1, fid = 2;
        return;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        q = make_float3(b.x + t * (c.x - b.x), b.y + t * (c.y - b.y), b.z + t * (c.z - b.z)), feat = 1, fid = 1;
        return;
    }
    const float den = va + vb + vc;
    if (den != 0.f) {
        const float inv = 1.f / den, v = vb * inv, w = vc * inv;
        q = make_float3(a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w);
    } else {
        q = a;  // degenerate triangle
    }
    feat = 2, fid = 0;
}

// TriMesh::project_local_point (trimesh.slang:116-155): the closest surface
// point within `max_dist` of the body-frame point p by stackless BVH
// traversal, and whether p is inside (pseudo-normal test).  Returns false
// when no triangle is that close.
__device__ __forceinline__ bool trimesh_project(const TriMeshRef &m, const float4 *vtx, const uint32_t *idx,
                                                const float *p, float max_dist, float *out, bool &inside) {
    const float3 pt = make_float3(p[0], p[1], p[2]);
    float best = max_dist;
    bool found = false;
    float3 bq = pt;
    uint32_t bfeat = 0, bfid = 0, btri = 0;
    const uint32_t vbase = m.vtx_root + 2u * m.n_nodes, tbase = m.idx_root + 3u * m.n_nodes;
    uint32_t curr = 0;
    for (uint32_t guard = 0; curr < m.n_nodes && guard < m.n_nodes; ++guard) {  // curr only grows
        const uint32_t entry = idx[m.idx_root + 3u * curr], exit = idx[m.idx_root + 3u * curr + 1u];
        if (entry == NONE) {
            const uint32_t t = idx[m.idx_root + 3u * curr + 2u];
            const float4 a4 = vtx[vbase + idx[tbase + 3u * t]], b4 = vtx[vbase + idx[tbase + 3u * t + 1u]],
                         c4 = vtx[vbase + idx[tbase + 3u * t + 2u]];
            float3 q;
            uint32_t feat, fid;
            triangle_closest(make_float3(a4.x, a4.y, a4.z), make_float3(b4.x, b4.y, b4.z),
                             make_float3(c4.x, c4.y, c4.z), pt, q, feat, fid);
            const float dx = q.x - pt.x, dy = q.y - pt.y, dz = q.z - pt.z;
            const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
            if (dist <= best) {
                best = dist, bq = q, bfeat = feat, bfid = fid, btri = t;
                found = true;
            }
            curr = exit;
        } else {
            const float4 mn = vtx[m.vtx_root + 2u * curr], mx = vtx[m.vtx_root + 2u * curr + 1u];
            const float sx = fmaxf(mn.x - pt.x, 0.f) - fmaxf(pt.x - mx.x, 0.f);
            const float sy = fmaxf(mn.y - pt.y, 0.f) - fmaxf(pt.y - mx.y, 0.f);
            const float sz = fmaxf(mn.z - pt.z, 0.f) - fmaxf(pt.z - mx.z, 0.f);
            curr = sqrtf(sx * sx + sy * sy + sz * sz) < best ? entry : exit;
        }
    }
    if (!found) return false;
    float3 pn;
    if (bfeat == 0) {  // vertex pseudo-normal
        const float4 n4 = vtx[vbase + m.n_verts + idx[tbase + 3u * btri + bfid]];
        pn = make_float3(n4.x, n4.y, n4.z);
    } else if (bfeat == 1) {  // edge pseudo-normal
        const float4 n4 = vtx[vbase + 2u * m.n_verts + 3u * btri + bfid];
        pn = make_float3(n4.x, n4.y, n4.z);
    } else {  // face normal
        const float4 a4 = vtx[vbase + idx[tbase + 3u * btri]], b4 = vtx[vbase + idx[tbase + 3u * btri + 1u]],
                     c4 = vtx[vbase + idx[tbase + 3u * btri + 2u]];
        const float3 ab = make_float3(b4.x - a4.x, b4.y - a4.y, b4.z - a4.z),
                     ac = make_float3(c4.x - a4.x, c4.y - a4.y, c4.z - a4.z);
        pn = make_float3(ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x);
    }
    inside = pn.x * (pt.x - bq.x) + pn.y * (pt.y - bq.y) + pn.z * (pt.z - bq.z) <= 0.f;
    out[0] = bq.x, out[1] = bq.y, out[2] = bq.z;
    return true;
}

}  // namespace slosh
