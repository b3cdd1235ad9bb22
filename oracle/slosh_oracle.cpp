// TEST INFRASTRUCTURE — the oracle.  Not part of the product: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, as the
// checker.  The product (slosh_b200/) never links or calls anything here.
//
// CPU restatement of slosh's MPM substep (dimforge/slosh,
// MpmPipeline::launch_step, src/pipeline.rs:562-770), written from the Slang
// shaders it launches.  Templated on the dimension (2, 3) and on the scalar
// (float restates the shader arithmetic operation by operation; double is the
// FP64 twin used for the conservation and precision studies).  Built without
// FMA contraction (-ffp-contract=off) so every float operation rounds as
// written in the shaders.
//
// PARITY STATUS.  The reference has no CPU implementation, no active tests
// and no golden vectors (its only CPU routine is the prefix sum's eval_cpu,
// src/grid/prefix_sum.rs:97-110, which this file restates and the tests pin
// with the reference's own commented-out test recipe).  The reference cannot
// be built here (Rust, Slang and wgpu are absent), so apart from that scan
// the oracle is "parity unpinned": it is checked against analytic invariants
// (conservation, SVD identities, closed-form single-particle cases) instead
// of reference outputs.  The 3x3 SVD lives in the third-party crate
// stensor 0.4.2 (not vendored); the oracle uses its own one-sided Jacobi SVD.
//
// Canonical order.  The reference numbers active blocks with an atomic
// counter and fills each sort bucket with atomics, so its order is not
// deterministic.  The oracle fixes it: blocks in ascending packed key;
// inside a block the primaries (buckets 0..NPB-1) first, ordered by (cell,
// particle id) with the cell index x + BW y (+ BW^2 z) -- slab-major, so each
// slab bucket remains one contiguous range as the reference requires -- then
// the extras ordered by (bucket, particle id).  Every per-block quantity of
// the reference (counts per bucket, first_particle, sorted ids) is then a
// deterministic function of the positions.
//
// Rounding conventions: `round` is round-half-to-even (WGSL round, the
// reference's primary target); divisions are IEEE divisions.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/slosh_b200.h"

namespace orc {

static constexpr uint32_t NONE = 0xffffffffu;

// Per-dimension constants of shaders/slosh/grid/grid.slang:224-257 and
// shaders/slosh/solver/g2p.slang:12-24.
template <int D> struct Geo;
template <> struct Geo<3> {
    static constexpr int BW = 4;          // cells per block edge (grid.slang:348)
    static constexpr int NASSOC = 8;      // NUM_ASSOC_BLOCKS
    static constexpr int NPB = 4;         // NUM_PRIMARY_SORT_BUCKETS
    static constexpr int NEB = 6;         // NUM_EXTRA_SORT_BUCKETS
    static constexpr int NB = 10;         // NUM_SORT_BUCKETS
    static constexpr int MIN_SHIFT = 2;   // EXTRA_PARTICLE_MIN_SHIFT
    static constexpr int SW = 6;          // shared halo width in g2p
    static constexpr int NBH = 27;        // NBH_LEN
};
template <> struct Geo<2> {
    static constexpr int BW = 8;
    static constexpr int NASSOC = 4;
    static constexpr int NPB = 8;
    static constexpr int NEB = 10;
    static constexpr int NB = 18;
    static constexpr int MIN_SHIFT = 6;
    static constexpr int SW = 10;
    static constexpr int NBH = 9;
};

// The 27 (9 in 2D) stencil shifts in the order g2p sums them
// (shaders/slosh/grid/kernel.slang:7-54).  The order fixes the FP32
// summation order of the gather.
static const int NBH_SHIFTS3[27][3] = {
    {2, 2, 2}, {2, 0, 2}, {2, 1, 2}, {0, 2, 2}, {0, 0, 2}, {0, 1, 2}, {1, 2, 2}, {1, 0, 2}, {1, 1, 2},
    {2, 2, 0}, {2, 0, 0}, {2, 1, 0}, {0, 2, 0}, {0, 0, 0}, {0, 1, 0}, {1, 2, 0}, {1, 0, 0}, {1, 1, 0},
    {2, 2, 1}, {2, 0, 1}, {2, 1, 1}, {0, 2, 1}, {0, 0, 1}, {0, 1, 1}, {1, 2, 1}, {1, 0, 1}, {1, 1, 1}};
static const int NBH_SHIFTS2[9][2] = {{2, 2}, {2, 0}, {2, 1}, {0, 2}, {0, 0},
                                      {0, 1}, {1, 2}, {1, 0}, {1, 1}};

// Block offsets of blocks_associated_to_block (grid.slang:362-382).
static const int ASSOC3[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                                 {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
static const int ASSOC2[4][2] = {{0, 0}, {0, 1}, {1, 0}, {1, 1}};

template <int D> inline const int *assoc_shift(int i) {
    if constexpr (D == 3) return ASSOC3[i];
    else return ASSOC2[i];
}
template <int D> inline const int *nbh_shift(int i) {
    if constexpr (D == 3) return NBH_SHIFTS3[i];
    else return NBH_SHIFTS2[i];
}

// pack_key (grid.slang:77-91).
template <int D> inline uint32_t pack_key(const int *b) {
    if constexpr (D == 3) {
        return ((uint32_t)(b[0] + 0x3ff) & 0x7ffu) | (((uint32_t)(b[1] + 0x1ff) & 0x3ffu) << 11) |
               (((uint32_t)(b[2] + 0x3ff) & 0x7ffu) << 21);
    } else {
        return ((uint32_t)(b[0] + 0x7fff) & 0xffffu) | (((uint32_t)(b[1] + 0x7fff) & 0xffffu) << 16);
    }
}

// Round half to even (WGSL `round`).
template <typename T> inline T round_even(T x) { return std::nearbyint(x); }

// --------------------------------------------------------------------------
// Small dense helpers (math convention: M[i][j] = row i, column j).
// --------------------------------------------------------------------------
template <typename T, int D> struct Mat {
    T m[D][D];
};

template <typename T, int D> inline T det(const Mat<T, D> &a) {
    if constexpr (D == 3) {
        // cofactor expansion along the first row.
        return a.m[0][0] * (a.m[1][1] * a.m[2][2] - a.m[1][2] * a.m[2][1]) -
               a.m[0][1] * (a.m[1][0] * a.m[2][2] - a.m[1][2] * a.m[2][0]) +
               a.m[0][2] * (a.m[1][0] * a.m[2][1] - a.m[1][1] * a.m[2][0]);
    } else {
        return a.m[0][0] * a.m[1][1] - a.m[0][1] * a.m[1][0];
    }
}

// --------------------------------------------------------------------------
// SVD.  Own implementation (the reference's stensor svd3/svd2 is not
// available): one-sided Jacobi on the columns of F, computed in double and
// rounded to T.  F = U diag(s) V^T with U, V proper rotations and
// s[0] >= s[1] >= |s[2]|, the sign of det F carried by the last value.
// --------------------------------------------------------------------------
template <int D> void svd_jacobi(const double *F, double *U, double *S, double *V) {
    double A[D][D], Vm[D][D];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            A[i][j] = F[i * D + j];
            Vm[i][j] = (i == j) ? 1.0 : 0.0;
        }
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < D - 1; ++p)
            for (int q = p + 1; q < D; ++q) {
                double alpha = 0, beta = 0, gamma = 0;
                for (int i = 0; i < D; ++i) {
                    alpha += A[i][p] * A[i][p];
                    beta += A[i][q] * A[i][q];
                    gamma += A[i][p] * A[i][q];
                }
                if (gamma == 0.0) continue;
                off = std::max(off, std::fabs(gamma) / std::sqrt(alpha * beta + 1e-300));
                double zeta = (beta - alpha) / (2.0 * gamma);
                double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < D; ++i) {
                    double ap = A[i][p], aq = A[i][q];
                    A[i][p] = c * ap - s * aq;
                    A[i][q] = s * ap + c * aq;
                    double vp = Vm[i][p], vq = Vm[i][q];
                    Vm[i][p] = c * vp - s * vq;
                    Vm[i][q] = s * vp + c * vq;
                }
            }
        if (off < 1e-15) break;
    }
    double sig[D];
    int order[D];
    for (int j = 0; j < D; ++j) {
        double s2 = 0;
        for (int i = 0; i < D; ++i) s2 += A[i][j] * A[i][j];
        sig[j] = std::sqrt(s2);
        order[j] = j;
    }
    std::sort(order, order + D, [&](int a, int b) { return sig[a] > sig[b]; });
    double Us[D][D], Vs[D][D], ss[D];
    for (int k = 0; k < D; ++k) {
        int j = order[k];
        ss[k] = sig[j];
        for (int i = 0; i < D; ++i) {
            Vs[i][k] = Vm[i][j];
            Us[i][k] = sig[j] > 1e-300 ? A[i][j] / sig[j] : 0.0;
        }
    }
    // Complete U where columns vanished (rank deficiency).
    for (int k = 0; k < D; ++k) {
        double n2 = 0;
        for (int i = 0; i < D; ++i) n2 += Us[i][k] * Us[i][k];
        if (n2 > 0.5) continue;
        // Gram-Schmidt against the other columns from a unit axis.
        for (int axis = 0; axis < D; ++axis) {
            double v[D];
            for (int i = 0; i < D; ++i) v[i] = (i == axis) ? 1.0 : 0.0;
            for (int o = 0; o < D; ++o) {
                if (o == k) continue;
                double on = 0, d = 0;
                for (int i = 0; i < D; ++i) {
                    on += Us[i][o] * Us[i][o];
                    d += Us[i][o] * v[i];
                }
                if (on < 0.5) continue;
                for (int i = 0; i < D; ++i) v[i] -= d * Us[i][o];
            }
            double vn = 0;
            for (int i = 0; i < D; ++i) vn += v[i] * v[i];
            if (vn > 1e-6) {
                vn = std::sqrt(vn);
                for (int i = 0; i < D; ++i) Us[i][k] = v[i] / vn;
                break;
            }
        }
    }
    auto detm = [](double M[D][D]) {
        if constexpr (D == 3)
            return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                   M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                   M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        else
            return M[0][0] * M[1][1] - M[0][1] * M[1][0];
    };
    // Make V and U proper rotations; the sign goes to the smallest value.
    if (detm(Vs) < 0) {
        for (int i = 0; i < D; ++i) Vs[i][D - 1] = -Vs[i][D - 1];
        ss[D - 1] = -ss[D - 1];
    }
    if (detm(Us) < 0) {
        for (int i = 0; i < D; ++i) Us[i][D - 1] = -Us[i][D - 1];
        ss[D - 1] = -ss[D - 1];
    }
    for (int i = 0; i < D; ++i) {
        S[i] = ss[i];
        for (int j = 0; j < D; ++j) {
            U[i * D + j] = Us[i][j];
            V[i * D + j] = Vs[i][j];
        }
    }
}

template <typename T, int D> struct Svd {
    Mat<T, D> U, V;
    T s[D];
};

template <typename T, int D> Svd<T, D> svd(const Mat<T, D> &F) {
    double f[D * D], u[D * D], s[D], v[D * D];
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) f[i * D + j] = (double)F.m[i][j];
    svd_jacobi<D>(f, u, s, v);
    Svd<T, D> r;
    for (int i = 0; i < D; ++i) {
        r.s[i] = (T)s[i];
        for (int j = 0; j < D; ++j) {
            r.U.m[i][j] = (T)u[i * D + j];
            r.V.m[i][j] = (T)v[i * D + j];
        }
    }
    return r;
}

// U diag(s) V^T, accumulated in T (Svd3::recompose).
template <typename T, int D> Mat<T, D> recompose(const Mat<T, D> &U, const T *s, const Mat<T, D> &V) {
    Mat<T, D> r;
    for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
            T acc = 0;
            for (int k = 0; k < D; ++k) acc += (U.m[i][k] * s[k]) * V.m[j][k];
            r.m[i][j] = acc;
        }
    return r;
}

// --------------------------------------------------------------------------
// Constitutive models (shaders/slosh/models/*.slang), math convention.
// --------------------------------------------------------------------------

// LinearElasticModel::kirchoff_stress (linear_elasticity.slang:69-82):
// tau = 2 mu (F - R) F^T + lambda (J - 1) J I, from one SVD of F.
template <typename T, int D> Mat<T, D> fixed_corotated(const Mat<T, D> &F, T lambda, T mu) {
    Svd<T, D> sv = svd<T, D>(F);
    T j = sv.s[0] * sv.s[1];
    if constexpr (D == 3) j = j * sv.s[2];
    T sm1[D];
    for (int i = 0; i < D; ++i) sm1[i] = sv.s[i] - T(1);
    Mat<T, D> rec = recompose<T, D>(sv.U, sm1, sv.V);  // F - R
    T diag = lambda * (j - T(1)) * j;
    Mat<T, D> tau;
    for (int i = 0; i < D; ++i)
        for (int k = 0; k < D; ++k) {
            T acc = 0;
            for (int l = 0; l < D; ++l) acc += F.m[k][l] * rec.m[i][l];
            tau.m[i][k] = acc * (T(2) * mu);
        }
    for (int i = 0; i < D; ++i) tau.m[i][i] += diag;
    return tau;
}

// NeoHookeanModel::kirchoff_stress (neo_hookean_elasticity.slang:16-27).
template <typename T, int D> Mat<T, D> neo_hookean(const Mat<T, D> &F, T lambda, T mu) {
    T j = std::max(det<T, D>(F), T(1.0e-10));
    T diag = lambda * std::log(j) - mu;
    Mat<T, D> tau;
    for (int i = 0; i < D; ++i)
        for (int k = 0; k < D; ++k) {
            T acc = 0;
            for (int l = 0; l < D; ++l) acc += F.m[i][l] * F.m[k][l];
            tau.m[i][k] = mu * acc;
        }
    for (int i = 0; i < D; ++i) tau.m[i][i] += diag;
    return tau;
}

// DruckerPragerPlasticity::project (drucker_prager.slang:46-50, 144-200).
// State: [plastic det, hardening q, log_vol_gain]; params
// [h0, h1, h2, h3, lambda, mu].  Returns false when the particle is left
// unchanged.
template <typename T, int D> void drucker_prager(T *state, const T *p, Mat<T, D> &F) {
    const T ha = p[0], hb = p[1], hc = p[2], hd = p[3], lambda = p[4], mu = p[5];
    if (lambda == T(0)) return;
    Svd<T, D> sv = svd<T, D>(F);
    const T q = state[1];
    // alpha(q)
    T angle = ha + (hb * q - hd) * std::exp(-hc * q);
    T s_angle = std::sin(angle);
    T alpha = std::sqrt(T(2.0) / T(3.0)) * (T(2.0) * s_angle) / (T(3.0) - s_angle);
    // project_deformation_gradient
    const T d = T(D);
    T strain[D], tr = 0;
    for (int i = 0; i < D; ++i) strain[i] = std::log(sv.s[i]) + state[2] / d;
    for (int i = 0; i < D; ++i) tr += strain[i];
    T dev[D];
    bool dev_zero = true;
    for (int i = 0; i < D; ++i) {
        dev[i] = strain[i] - tr / d;
        dev_zero = dev_zero && (dev[i] == T(0));
    }
    T newsig[D], dq;
    if (tr > T(0) || dev_zero) {
        T n2 = 0;
        for (int i = 0; i < D; ++i) n2 += strain[i] * strain[i];
        for (int i = 0; i < D; ++i) newsig[i] = T(1);
        dq = std::sqrt(n2);
    } else {
        T n2 = 0;
        for (int i = 0; i < D; ++i) n2 += dev[i] * dev[i];
        T devn = std::sqrt(n2);
        T gamma = devn + (d * lambda + T(2.0) * mu) / (T(2.0) * mu) * tr * alpha;
        if (gamma <= T(0)) return;  // invalid projection: state and F unchanged
        for (int i = 0; i < D; ++i) newsig[i] = std::exp(strain[i] - dev[i] * (gamma / devn));
        dq = gamma;
    }
    T prev_det = sv.s[0] * sv.s[1], new_det = newsig[0] * newsig[1];
    if constexpr (D == 3) {
        prev_det = prev_det * sv.s[2];
        new_det = new_det * newsig[2];
    }
    state[0] = state[0] * prev_det / new_det;
    state[2] = state[2] + std::log(prev_det) - std::log(new_det);
    state[1] = q + dq;
    F = recompose<T, D>(sv.U, newsig, sv.V);
}

// Weakly compressible Tait fluid (extension, see slosh_b200.h).
template <typename T, int D> Mat<T, D> tait_fluid(const Mat<T, D> &F, T bulk, T gamma) {
    T J = F.m[0][0];
    T pressure = (bulk / gamma) * (std::pow(J, -gamma) - T(1));
    Mat<T, D> tau{};
    for (int i = 0; i < D; ++i) tau.m[i][i] = -J * pressure;
    return tau;
}

// --------------------------------------------------------------------------
// Scene state.
// --------------------------------------------------------------------------
template <typename T, int D> struct Particles {
    size_t n = 0;
    std::vector<T> x, v, fdt;       // n * D
    std::vector<T> C, F;            // n * D * D (row-major math)
    std::vector<T> vgd, V0, r0, mass, damping, phase;
    std::vector<uint32_t> enabled, fixed, tag;
    std::vector<T> model;  // n * 12 model payload words
};

// Triangle mesh of a trimesh collider (3D): vertices (3 a vertex), triangles
// (3 vertex indices), and the pseudo-normals of Baerentzen and Aanaes (2005):
// per vertex the angle-weighted sum of the incident unit face normals, per
// edge the sum of its faces' unit normals (3 a triangle: AB, BC, CA).
template <typename T> struct Mesh {
    std::vector<T> v, vpn, epn;
    std::vector<uint32_t> tri;
};

template <typename T> Mesh<T> make_mesh(const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt) {
    Mesh<T> m;
    m.v.assign(v, v + 3 * (size_t)nv);
    m.tri.assign(tri, tri + 3 * (size_t)nt);
    m.vpn.assign(3 * (size_t)nv, T(0));
    m.epn.assign(9 * (size_t)nt, T(0));
    std::unordered_map<uint64_t, std::array<T, 3>> edge;
    std::vector<T> fn(3 * (size_t)nt, T(0));
    for (uint32_t f = 0; f < nt; ++f) {
        const uint32_t vs[3] = {tri[3 * f], tri[3 * f + 1], tri[3 * f + 2]};
        T ab[3], ac[3];
        for (int k = 0; k < 3; ++k) {
            ab[k] = m.v[3 * vs[1] + k] - m.v[3 * vs[0] + k];
            ac[k] = m.v[3 * vs[2] + k] - m.v[3 * vs[0] + k];
        }
        T n[3] = {ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]};
        const T nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > T(0))
            for (int k = 0; k < 3; ++k) n[k] /= nn;
        for (int k = 0; k < 3; ++k) fn[3 * f + k] = n[k];
        for (int c = 0; c < 3; ++c) {
            const uint32_t p0 = vs[c], p1 = vs[(c + 1) % 3], p2 = vs[(c + 2) % 3];
            T e1[3], e2[3], l1 = 0, l2 = 0, d = 0;
            for (int k = 0; k < 3; ++k) {
                e1[k] = m.v[3 * p1 + k] - m.v[3 * p0 + k];
                e2[k] = m.v[3 * p2 + k] - m.v[3 * p0 + k];
                l1 += e1[k] * e1[k];
                l2 += e2[k] * e2[k];
                d += e1[k] * e2[k];
            }
            const T den = std::sqrt(l1 * l2);
            const T ang = den > T(0) ? std::acos(std::max(T(-1), std::min(T(1), d / den))) : T(0);
            for (int k = 0; k < 3; ++k) m.vpn[3 * (size_t)p0 + k] += ang * n[k];
            const uint64_t key = ((uint64_t)std::min(p0, p1) << 32) | std::max(p0, p1);
            auto it = edge.find(key);
            if (it == edge.end()) it = edge.emplace(key, std::array<T, 3>{T(0), T(0), T(0)}).first;
            for (int k = 0; k < 3; ++k) it->second[k] += n[k];
        }
    }
    for (uint32_t i = 0; i < nv; ++i) {
        T *n = &m.vpn[3 * (size_t)i];
        const T nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > T(0))
            for (int k = 0; k < 3; ++k) n[k] /= nn;
    }
    for (uint32_t f = 0; f < nt; ++f)
        for (int c = 0; c < 3; ++c) {
            const uint32_t p0 = tri[3 * f + c], p1 = tri[3 * f + (c + 1) % 3];
            const auto &e = edge[((uint64_t)std::min(p0, p1) << 32) | std::max(p0, p1)];
            for (int k = 0; k < 3; ++k) m.epn[9 * (size_t)f + 3 * c + k] = e[k];
        }
    return m;
}

// Closest point on triangle abc to p (Ericson, Real-Time Collision
// Detection, 5.1.5) and its feature: vertex (0; id 0 a, 1 b, 2 c), edge
// (1; id 0 AB, 1 BC, 2 CA) or face (2), as in trimesh.slang:214-377.
template <typename T>
void tri_closest(const T *a, const T *b, const T *c, const T *p, T *q, int &feat, int &fid) {
    T ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int k = 0; k < 3; ++k) {
        ab[k] = b[k] - a[k];
        ac[k] = c[k] - a[k];
        ap[k] = p[k] - a[k];
        bp[k] = p[k] - b[k];
        cp[k] = p[k] - c[k];
    }
    auto dot = [](const T *u, const T *w) { return u[0] * w[0] + u[1] * w[1] + u[2] * w[2]; };
    const T d1 = dot(ab, ap), d2 = dot(ac, ap);
    auto set = [&](const T *s, int f, int i) {
        for (int k = 0; k < 3; ++k) q[k] = s[k];
        feat = f, fid = i;
    };
    if (d1 <= T(0) && d2 <= T(0)) return set(a, 0, 0);
    const T d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= T(0) && d4 <= d3) return set(b, 0, 1);
    const T vc = d1 * d4 - d3 * d2;
    if (vc <= T(0) && d1 >= T(0) && d3 <= T(0)) {
        const T t = d1 / (d1 - d3);
        for (int k = 0; k < 3; ++k) q[k] = a[k] + t * ab[k];
        feat = 1, fid = 0;
        return;
    }
    const T d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= T(0) && d5 <= d6) return set(c, 0, 2);
    const T vb = d5 * d2 - d1 * d6;
    if (vb <= T(0) && d2 >= T(0) && d6 <= T(0)) {
        const T t = d2 / (d2 - d6);
        for (int k = 0; k < 3; ++k) q[k] = a[k] + t * ac[k];
        feat = 1, fid = 2;
        return;
    }
    const T va = d3 * d6 - d5 * d4;
    if (va <= T(0) && (d4 - d3) >= T(0) && (d5 - d6) >= T(0)) {
        const T t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; ++k) q[k] = b[k] + t * (c[k] - b[k]);
        feat = 1, fid = 1;
        return;
    }
    const T den = va + vb + vc;
    if (den != T(0)) {
        const T v = vb / den, w = vc / den;
        for (int k = 0; k < 3; ++k) q[k] = a[k] + ab[k] * v + ac[k] * w;
    } else {
        for (int k = 0; k < 3; ++k) q[k] = a[k];
    }
    feat = 2, fid = 0;
}

// TriMesh::project_local_point (collision/trimesh.slang:116-155), by a scan
// of every triangle instead of slosh's BVH: the closest surface point within
// `max_dist` (ties to the later triangle) and the pseudo-normal inside test.
template <typename T> bool mesh_project(const Mesh<T> &m, const T *p, T max_dist, T *out, bool *inside) {
    T best = max_dist, bq[3] = {p[0], p[1], p[2]};
    int bfeat = 0, bfid = 0;
    size_t btri = 0;
    bool found = false;
    const size_t nt = m.tri.size() / 3;
    for (size_t f = 0; f < nt; ++f) {
        T q[3];
        int feat, fid;
        tri_closest<T>(&m.v[3 * m.tri[3 * f]], &m.v[3 * m.tri[3 * f + 1]], &m.v[3 * m.tri[3 * f + 2]], p, q, feat, fid);
        const T dist = std::sqrt((q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) + (q[2] - p[2]) * (q[2] - p[2]));
        if (dist <= best) {
            best = dist;
            for (int k = 0; k < 3; ++k) bq[k] = q[k];
            bfeat = feat, bfid = fid, btri = f, found = true;
        }
    }
    if (!found) return false;
    T pn[3];
    if (bfeat == 0) {
        for (int k = 0; k < 3; ++k) pn[k] = m.vpn[3 * (size_t)m.tri[3 * btri + bfid] + k];
    } else if (bfeat == 1) {
        for (int k = 0; k < 3; ++k) pn[k] = m.epn[9 * btri + 3 * bfid + k];
    } else {
        const T *a = &m.v[3 * m.tri[3 * btri]], *b = &m.v[3 * m.tri[3 * btri + 1]], *c = &m.v[3 * m.tri[3 * btri + 2]];
        const T ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        pn[0] = ab[1] * ac[2] - ab[2] * ac[1];
        pn[1] = ab[2] * ac[0] - ab[0] * ac[2];
        pn[2] = ab[0] * ac[1] - ab[1] * ac[0];
    }
    *inside = pn[0] * (p[0] - bq[0]) + pn[1] * (p[1] - bq[1]) + pn[2] * (p[2] - bq[2]) <= T(0);
    for (int k = 0; k < 3; ++k) out[k] = bq[k];
    return true;
}

template <typename T, int D> struct Body {
    uint32_t shape_type;
    const Mesh<T> *mesh = nullptr;  // trimesh colliders
    T sa[4], sb[4];
    T rot[4];  // 3D quaternion (i, j, k, w); 2D (cos, sin)
    T tra[3];
    T scale;
    T linvel[3], angvel[3];
    T inv_mass[3], local_com[3];
    float inv_inertia[12];
    uint32_t bc_type;
    T friction;
    uint32_t coupling;  // SLOSH_COUPLING_*
    T inv_inertia_local[9];  // body-frame inverse inertia, row-major (2D: [0])
};

// Rotation matrix of a unit quaternion (i, j, k, w), and R M R^T / R^T M R.
template <typename T> inline void quat_to_mat(const T *q, T (&R)[3][3]) {
    const T x = q[0], y = q[1], z = q[2], w = q[3];
    R[0][0] = T(1) - T(2) * (y * y + z * z);
    R[0][1] = T(2) * (x * y - z * w);
    R[0][2] = T(2) * (x * z + y * w);
    R[1][0] = T(2) * (x * y + z * w);
    R[1][1] = T(1) - T(2) * (x * x + z * z);
    R[1][2] = T(2) * (y * z - x * w);
    R[2][0] = T(2) * (x * z - y * w);
    R[2][1] = T(2) * (y * z + x * w);
    R[2][2] = T(1) - T(2) * (x * x + y * y);
}
template <typename T> inline void conjugate(const T (&R)[3][3], const T *M, T *out, bool forward) {
    T A[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T a = 0;
            for (int k = 0; k < 3; ++k) a += (forward ? R[i][k] : R[k][i]) * M[k * 3 + j];
            A[i][j] = a;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T a = 0;
            for (int k = 0; k < 3; ++k) a += A[i][k] * (forward ? R[j][k] : R[k][j]);
            out[i * 3 + j] = a;
        }
}

// Two-way coupling impulse sums: 64-bit fixed point, 2^40 units per N s.
constexpr double IMPULSE_UNITS = 1099511627776.0;
inline long long impulse_units(double v) { return std::llrint(v * IMPULSE_UNITS); }

// Quaternion helpers (stensor Quat / Sim3, restated from their definitions:
// rotation of v by q, Hamilton product).
template <typename T> inline void quat_rotate(const T *q, const T *v, T *out) {
    // t = 2 q_v x v ; out = v + w t + q_v x t
    T t[3] = {T(2) * (q[1] * v[2] - q[2] * v[1]), T(2) * (q[2] * v[0] - q[0] * v[2]),
              T(2) * (q[0] * v[1] - q[1] * v[0])};
    out[0] = v[0] + q[3] * t[0] + (q[1] * t[2] - q[2] * t[1]);
    out[1] = v[1] + q[3] * t[1] + (q[2] * t[0] - q[0] * t[2]);
    out[2] = v[2] + q[3] * t[2] + (q[0] * t[1] - q[1] * t[0]);
}
template <typename T> inline void quat_mul(const T *a, const T *b, T *o) {
    o[0] = a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1];
    o[1] = a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0];
    o[2] = a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3];
    o[3] = a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2];
}

template <typename T, int D> struct Pose {
    // pose.mul_pt(p) = R (s p) + t ; inv_mul_pt(p) = R^-1 (p - t) / s
    static void mul_pt(const Body<T, D> &b, const T *p, T *out) {
        if constexpr (D == 3) {
            T sp[3] = {p[0] * b.scale, p[1] * b.scale, p[2] * b.scale};
            T r[3];
            quat_rotate(b.rot, sp, r);
            for (int i = 0; i < 3; ++i) out[i] = r[i] + b.tra[i];
        } else {
            T sp0 = p[0] * b.scale, sp1 = p[1] * b.scale;
            out[0] = b.rot[0] * sp0 - b.rot[1] * sp1 + b.tra[0];
            out[1] = b.rot[1] * sp0 + b.rot[0] * sp1 + b.tra[1];
        }
    }
    static void inv_mul_pt(const Body<T, D> &b, const T *p, T *out) {
        if constexpr (D == 3) {
            T d[3] = {p[0] - b.tra[0], p[1] - b.tra[1], p[2] - b.tra[2]};
            T qi[4] = {-b.rot[0], -b.rot[1], -b.rot[2], b.rot[3]};
            T r[3];
            quat_rotate(qi, d, r);
            for (int i = 0; i < 3; ++i) out[i] = r[i] / b.scale;
        } else {
            T d0 = p[0] - b.tra[0], d1 = p[1] - b.tra[1];
            out[0] = (b.rot[0] * d0 + b.rot[1] * d1) / b.scale;
            out[1] = (-b.rot[1] * d0 + b.rot[0] * d1) / b.scale;
        }
    }
};

// Shape::project_point_on_boundary for ball and cuboid
// (shaders/slosh/rbd/shapes/ball.slang, cuboid.slang:34-63).
// Segment::project_local_point (rbd/shapes/segment.slang:9-28).
template <typename T, int D> void segment_project(const T *a, const T *b, const T *p, T *q) {
    T ab[D], ab_ap = 0, sqn = 0;
    for (int k = 0; k < D; ++k) {
        ab[k] = b[k] - a[k];
        ab_ap += ab[k] * (p[k] - a[k]);
        sqn += ab[k] * ab[k];
    }
    if (ab_ap <= T(0)) {
        for (int k = 0; k < D; ++k) q[k] = a[k];
    } else if (ab_ap >= sqn) {
        for (int k = 0; k < D; ++k) q[k] = b[k];
    } else {
        T u = ab_ap / sqn;
        for (int k = 0; k < D; ++k) q[k] = a[k] + ab[k] * u;
    }
}

// Capsule::project_local_point_on_boundary (rbd/shapes/capsule.slang:38-55),
// any_orthogonal_vector / orthonormal_basis3 (capsule.slang:66-95).
template <typename T, int D> bool capsule_project(const T *a, const T *b, T radius, const T *p, T *out) {
    T q[D], d[D], n2 = 0;
    segment_project<T, D>(a, b, p, q);
    for (int k = 0; k < D; ++k) {
        d[k] = p[k] - q[k];
        n2 += d[k] * d[k];
    }
    T dist = std::sqrt(n2);
    if (dist > T(0)) {
        for (int k = 0; k < D; ++k) out[k] = q[k] + d[k] * (radius / dist);
        return dist <= radius;
    }
    T ax[D], l2 = 0;
    for (int k = 0; k < D; ++k) {
        ax[k] = b[k] - a[k];
        l2 += ax[k] * ax[k];
    }
    T len = std::sqrt(l2);
    for (int k = 0; k < D; ++k) ax[k] = ax[k] / len;
    T o[D];
    if constexpr (D == 2) {
        o[0] = ax[1];
        o[1] = -ax[0];
    } else {
        T sg = ax[2] >= T(0) ? T(1) : T(-1);
        T aa = T(-1) / (sg + ax[2]);
        T bb = ax[0] * ax[1] * aa;
        o[0] = T(1) + sg * ax[0] * ax[0] * aa;
        o[1] = sg * bb;
        o[2] = -sg * ax[0];
    }
    for (int k = 0; k < D; ++k) out[k] = q[k] + o[k] * radius;
    return true;
}

// Cylinder::project_local_point_on_boundary (rbd/shapes/cylinder.slang:72-125).
template <typename T> bool cylinder_project(T hh, T r, const T *p, T *out) {
    T rxz = std::sqrt(p[0] * p[0] + p[2] * p[2]);
    T dx = rxz > T(0) ? p[0] / rxz : T(1), dz = rxz > T(0) ? p[2] / rxz : T(0);
    T px = dx * r, pz = dz * r;
    if (p[1] >= -hh && p[1] <= hh && rxz <= r) {
        T top = hh - p[1], bottom = p[1] - (-hh), side = r - rxz;
        if (top < bottom && top < side) {
            out[0] = p[0], out[1] = hh, out[2] = p[2];
        } else if (bottom < top && bottom < side) {
            out[0] = p[0], out[1] = -hh, out[2] = p[2];
        } else {
            out[0] = px, out[1] = p[1], out[2] = pz;
        }
        return true;
    }
    if (p[1] > hh) {
        if (rxz <= r) out[0] = p[0], out[1] = hh, out[2] = p[2];
        else out[0] = px, out[1] = hh, out[2] = pz;
    } else if (p[1] < -hh) {
        if (rxz <= r) out[0] = p[0], out[1] = -hh, out[2] = p[2];
        else out[0] = px, out[1] = -hh, out[2] = pz;
    } else {
        out[0] = px, out[1] = p[1], out[2] = pz;
    }
    return false;
}

// Cone::project_local_point_on_boundary (rbd/shapes/cone.slang:82-131).
template <typename T> bool cone_project(T hh, T r, const T *p, T *out) {
    T rxz = std::sqrt(p[0] * p[0] + p[2] * p[2]);
    T dx = rxz > T(0) ? p[0] / rxz : T(1), dz = rxz > T(0) ? p[2] / rxz : T(0);
    T basis[3] = {p[0], -hh, p[2]};
    if (p[1] < -hh && rxz <= r) {
        for (int k = 0; k < 3; ++k) out[k] = basis[k];
        return false;
    }
    T circle[3] = {dx * r, -hh, dz * r};
    T apex[3] = {T(0), hh, T(0)};
    T seg_dir[3] = {circle[0] - apex[0], circle[1] - apex[1], circle[2] - apex[2]};
    T proj[3];
    segment_project<T, 3>(apex, circle, p, proj);
    T rel[3] = {p[0] - apex[0], p[1] - apex[1], p[2] - apex[2]};
    T down[3] = {T(0), T(-2) * hh, T(0)};
    auto cross = [](const T *u, const T *v, T *w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    T c1[3], c2[3];
    cross(seg_dir, rel, c1);
    cross(seg_dir, down, c2);
    bool in = p[1] >= -hh && p[1] <= hh && (c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2]) >= T(0);
    if (in) {
        T dp = 0, db = 0;
        for (int k = 0; k < 3; ++k) {
            dp += (proj[k] - p[k]) * (proj[k] - p[k]);
            db += (basis[k] - p[k]) * (basis[k] - p[k]);
        }
        const T *src = dp > db ? basis : proj;
        for (int k = 0; k < 3; ++k) out[k] = src[k];
        return true;
    }
    for (int k = 0; k < 3; ++k) out[k] = proj[k];
    return false;
}

template <typename T, int D>
bool project_on_boundary(const Body<T, D> &b, const T *pt, T *proj, bool *is_inside, T cap = T(1e30)) {
    T local[D];
    Pose<T, D>::inv_mul_pt(b, pt, local);
    T lp[D];
    if (b.shape_type == SLOSH_SHAPE_CUBOID) {
        T out_proj[D];
        for (int i = 0; i < D; ++i) {
            T mins_pt = -b.sa[i] - local[i];
            T pt_maxs = local[i] - b.sa[i];
            T shift = std::max(mins_pt, T(0)) - std::max(pt_maxs, T(0));
            out_proj[i] = local[i] + shift;
        }
        T sgn[D], diff[D];
        for (int i = 0; i < D; ++i) {
            T sw = (local[i] > 0) ? T(1) : ((local[i] < 0) ? T(-1) : T(0));
            sgn[i] = sw + (std::fabs(sw) - T(1));
            diff[i] = b.sa[i] - sgn[i] * local[i];
        }
        T in_proj[D];
        for (int i = 0; i < D; ++i) in_proj[i] = local[i];
        if constexpr (D == 3) {
            bool pick_x = diff[0] <= diff[1] && diff[0] <= diff[2];
            bool pick_y = diff[1] <= diff[0] && diff[1] <= diff[2];
            if (pick_x) in_proj[0] = local[0] + diff[0] * sgn[0];
            else if (pick_y) in_proj[1] = local[1] + diff[1] * sgn[1];
            else in_proj[2] = local[2] + diff[2] * sgn[2];
        } else {
            bool pick_x = diff[0] <= diff[1];
            if (pick_x) in_proj[0] = local[0] + diff[0] * sgn[0];
            else in_proj[1] = local[1] + diff[1] * sgn[1];
        }
        bool inside = true;
        for (int i = 0; i < D; ++i) inside = inside && (local[i] == out_proj[i]);
        for (int i = 0; i < D; ++i) lp[i] = inside ? in_proj[i] : out_proj[i];
        *is_inside = inside;
    } else if (b.shape_type == SLOSH_SHAPE_BALL) {
        T n2 = 0;
        for (int i = 0; i < D; ++i) n2 += local[i] * local[i];
        T dist = std::sqrt(n2);
        T r = b.sa[0];
        for (int i = 0; i < D; ++i) lp[i] = (dist != T(0)) ? local[i] * (r / dist) : T(0);
        if (dist == T(0)) lp[1] = r;
        *is_inside = dist <= r;
    } else if (b.shape_type == SLOSH_SHAPE_CAPSULE) {
        *is_inside = capsule_project<T, D>(b.sa, b.sb, b.sb[3], local, lp);
    } else if (D == 3 && b.shape_type == SLOSH_SHAPE_CYLINDER) {
        if constexpr (D == 3) *is_inside = cylinder_project<T>(b.sa[0], b.sa[1], local, lp);
    } else if (D == 3 && b.shape_type == SLOSH_SHAPE_CONE) {
        if constexpr (D == 3) *is_inside = cone_project<T>(b.sa[0], b.sa[1], local, lp);
    } else if (D == 3 && b.shape_type == SLOSH_SHAPE_TRIMESH && b.mesh) {
        if constexpr (D == 3)
            if (!mesh_project<T>(*b.mesh, local, cap, lp, is_inside)) return false;
    } else {
        return false;
    }
    Pose<T, D>::mul_pt(b, lp, proj);
    return true;
}

template <typename T, int D> struct NodeCollision {
    T normal[D];
    T point[D];
    uint32_t collider_id;
    uint32_t valid;
};

// collide (shaders/slosh/collision/collide.slang:87-153).
template <typename T, int D>
NodeCollision<T, D> collide(const std::vector<Body<T, D>> &bodies, T cell_width, const T *point) {
    NodeCollision<T, D> c{};
    const T dist_cap = cell_width * T(1.5);
    T best_dist = T(1.0e10);
    for (size_t i = 0; i < bodies.size() && i < 16; ++i) {
        T proj[D];
        bool inside = false;
        if (!project_on_boundary<T, D>(bodies[i], point, proj, &inside, dist_cap)) continue;
        T dpt[D];
        bool within = true;
        for (int k = 0; k < D; ++k) {
            dpt[k] = proj[k] - point[k];
            within = within && (std::fabs(dpt[k]) <= dist_cap);
        }
        if (inside || within) {
            T sign = inside ? T(-1) : T(1);
            T n2 = 0;
            for (int k = 0; k < D; ++k) n2 += dpt[k] * dpt[k];
            T dist = std::sqrt(n2);
            if (sign * dist < best_dist && dist != T(0)) {
                for (int k = 0; k < D; ++k) {
                    c.normal[k] = dpt[k] / (dist * -sign);
                    c.point[k] = proj[k];
                }
                c.collider_id = (uint32_t)i;
                c.valid = 1;
                best_dist = dist;
            }
        }
    }
    return c;
}

// BoundaryCondition::project_velocity (boundary_condition.slang:31-89),
// including its use of `this.friction` where the local `friction` was meant.
template <typename T, int D> void project_velocity(uint32_t type, T friction, T *vel, const T *n, T dist, T dt) {
    switch (type) {
        case SLOSH_BC_STICK:
            if (dist <= T(0))
                for (int k = 0; k < D; ++k) vel[k] = T(0);
            return;
        case SLOSH_BC_SLIP:
            if (dist <= T(0)) {
                T nv = 0;
                for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
                for (int k = 0; k < D; ++k) vel[k] = vel[k] - n[k] * nv;
            }
            return;
        case SLOSH_BC_SEPARATE:
        case SLOSH_BC_FRICTION_Z_UP: {
            T nv = 0;
            for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
            if (nv < T(0)) {
                if (dist <= T(0)) {
                    T tv[D], tl2 = 0;
                    for (int k = 0; k < D; ++k) {
                        tv[k] = vel[k] - n[k] * nv;
                        tl2 += tv[k] * tv[k];
                    }
                    T tl = std::sqrt(tl2);
                    T scale = std::max(T(0), tl + friction * nv);
                    for (int k = 0; k < D; ++k) {
                        T dir = (tl > T(1.0e-8)) ? tv[k] / tl : T(0);
                        vel[k] = dir * scale;
                    }
                } else if (-nv * dt > dist) {
                    T a = dist / dt + nv;
                    for (int k = 0; k < D; ++k) vel[k] = vel[k] - a * n[k];
                }
            }
            return;
        }
        default:
            return;
    }
}

// QuadraticKernel (kernel.slang:57-84).
template <typename T> inline T kernel_eval(T x) {
    T xa = std::fabs(x);
    T part1 = T(0.75) - xa * xa;
    T part2 = T(0.5) * (T(1.5) - xa) * (T(1.5) - xa);
    return xa < T(0.5) ? part1 : (xa < T(1.5) ? part2 : T(0));
}
template <typename T> inline void kernel_eval_all(T x, T *w) {
    w[0] = T(0.5) * (T(1.5) - x) * (T(1.5) - x);
    w[1] = T(0.75) - (x - T(1.0)) * (x - T(1.0));
    w[2] = T(0.5) * (x - T(0.5)) * (x - T(0.5));
}

template <typename T, int D> struct Grid {
    // canonical block list
    std::vector<uint32_t> keys;           // ascending packed keys
    std::vector<std::array<int, 3>> vid;  // virtual ids
    std::unordered_map<uint32_t, uint32_t> rank;
    std::vector<uint32_t> first, np, npe;  // first_particle, num_particles, with extras
    std::vector<uint32_t> counts;          // nb * NB
    std::vector<uint32_t> sorted;          // sorted particle ids (with extras)
    std::vector<T> nodes;                  // nb * 64 * 4 (D+1 used)
    std::vector<NodeCollision<T, D>> coll; // nb * 64
};

template <typename T, int D> struct Ctx {
    T h;
    T gravity[3] = {0, 0, 0};
    T dt = 0;
    uint32_t capacity;
    Particles<T, D> p;
    std::vector<Body<T, D>> bodies;
    std::vector<Mesh<T>> meshes;  // trimesh colliders, by ordinal
    std::vector<long long> impulses;  // 6 fixed-point sums per body (two-way coupling)
    Grid<T, D> grid, prev;
    int nthreads = 1;

    bool coll_dynamic() const {
        for (const auto &b : bodies)
            if (b.coupling == SLOSH_COUPLING_TWO_WAY) return true;
        return false;
    }

    // block_associated_to_point and associated_cell_index_in_block_off_by_one
    // (grid.slang:346-354; particle.slang:79-87).
    void cell_of(size_t i, int *block, int *local) const {
        for (int k = 0; k < D; ++k) {
            T assoc_cell = round_even(p.x[i * D + k] / h) - T(1.0);
            T ab = std::floor(assoc_cell / T(Geo<D>::BW));
            block[k] = (int)ab;
            local[k] = (int)(assoc_cell - ab * T(Geo<D>::BW));
        }
    }

    static uint32_t primary_bucket(const int *a) { return (uint32_t)a[D - 1]; }
    static uint32_t extra_bucket(const int *a, const int *bshift) {
        int local = a[D - 1] - bshift[D - 1] * Geo<D>::BW;
        return (uint32_t)(Geo<D>::NPB + (std::max(local, -2) + 2));
    }
    static bool extra_spills(const int *a, const int *bshift) {
        for (int k = 0; k < D; ++k)
            if (bshift[k] == 1 && !(a[k] >= Geo<D>::MIN_SHIFT)) return false;
        return true;
    }

    // Grid build (src/grid/grid.rs:78-238 and the kernels it launches in
    // grid.slang / sort.slang) in canonical order.  Returns false on overflow.
    bool grid_build(Grid<T, D> &g) {
        const size_t n = p.n;
        std::vector<uint32_t> pkey(n);
        std::vector<uint8_t> plocal(n * D);
        std::vector<std::array<int, 3>> pblock(n);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long i = 0; i < (long long)n; ++i) {
            int b[D], a[D];
            cell_of((size_t)i, b, a);
            pkey[i] = pack_key<D>(b);
            for (int k = 0; k < D; ++k) {
                plocal[i * D + k] = (uint8_t)a[k];
                pblock[i][k] = b[k];
            }
        }
        // Active blocks: primaries, then their +1 neighbours.
        std::unordered_map<uint32_t, std::array<int, 3>> active;
        active.reserve(capacity * 2);
        uint32_t prev_key = NONE;
        for (size_t i = 0; i < n; ++i) {
            if (pkey[i] == prev_key && i > 0) continue;
            prev_key = pkey[i];
            active.emplace(pkey[i], pblock[i]);
        }
        std::vector<std::array<int, 3>> primaries;
        primaries.reserve(active.size());
        for (auto &kv : active) primaries.push_back(kv.second);
        for (auto &pb : primaries)
            for (int s = 1; s < Geo<D>::NASSOC; ++s) {
                const int *sh = assoc_shift<D>(s);
                int nb[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) nb[k] = pb[k] + sh[k];
                std::array<int, 3> v = {nb[0], nb[1], nb[2]};
                active.emplace(pack_key<D>(nb), v);
            }
        if (active.size() > capacity) return false;
        g.keys.clear();
        for (auto &kv : active) g.keys.push_back(kv.first);
        std::sort(g.keys.begin(), g.keys.end());
        const size_t nb = g.keys.size();
        g.vid.resize(nb);
        g.rank.clear();
        g.rank.reserve(nb * 2);
        for (size_t r = 0; r < nb; ++r) {
            g.rank[g.keys[r]] = (uint32_t)r;
            g.vid[r] = active[g.keys[r]];
        }
        // Per-bucket counts (update_block_particle_count, sort.slang:208-246).
        const int NB = Geo<D>::NB;
        g.counts.assign(nb * NB, 0);
        std::vector<uint32_t> nbh(nb * (Geo<D>::NASSOC - 1), NONE);
        for (size_t r = 0; r < nb; ++r)
            for (int s = 1; s < Geo<D>::NASSOC; ++s) {
                const int *sh = assoc_shift<D>(s);
                int q[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) q[k] = g.vid[r][k] + sh[k];
                auto it = g.rank.find(pack_key<D>(q));
                if (it != g.rank.end()) nbh[r * (Geo<D>::NASSOC - 1) + s - 1] = it->second;
            }
        std::vector<uint32_t> prank(n);
        for (size_t i = 0; i < n; ++i) {
            uint32_t r0 = g.rank[pkey[i]];
            prank[i] = r0;
            int a[D];
            for (int k = 0; k < D; ++k) a[k] = plocal[i * D + k];
            g.counts[r0 * NB + primary_bucket(a)] += 1;
            for (int s = 1; s < Geo<D>::NASSOC; ++s) {
                const int *sh = assoc_shift<D>(s);
                if (extra_spills(a, sh)) {
                    uint32_t rb = nbh[r0 * (Geo<D>::NASSOC - 1) + s - 1];
                    g.counts[rb * NB + extra_bucket(a, sh)] += 1;
                }
            }
        }
        // copy_particles_len_to_scan_value + prefix sum + prepare_for_finalize.
        g.first.assign(nb, 0);
        g.np.assign(nb, 0);
        g.npe.assign(nb, 0);
        std::vector<uint32_t> cursor(nb * NB);
        uint32_t running = 0;
        for (size_t r = 0; r < nb; ++r) {
            g.first[r] = running;
            uint32_t run = running;
            for (int k = 0; k < NB; ++k) {
                if (k == Geo<D>::NPB) g.np[r] = run - running;
                cursor[r * NB + k] = run;
                run += g.counts[r * NB + k];
            }
            g.npe[r] = run - running;
            running = run;
        }
        // finalize_particles_sort in canonical order: primaries by (cell, id),
        // the cell index being x + BW y (+ BW^2 z), i.e. slab-major so that
        // every primary slab bucket stays one contiguous range; extras by
        // (bucket, id).
        constexpr int NCELL = 64;
        std::vector<uint32_t> cellcnt(nb * NCELL, 0), cellcur(nb * NCELL);
        auto cell_index = [](const int *a) {
            int c = 0, mul = 1;
            for (int k = 0; k < D; ++k) {
                c += a[k] * mul;
                mul *= Geo<D>::BW;
            }
            return c;
        };
        for (size_t i = 0; i < n; ++i) {
            int a[D];
            for (int k = 0; k < D; ++k) a[k] = plocal[i * D + k];
            cellcnt[prank[i] * NCELL + cell_index(a)] += 1;
        }
        for (size_t r = 0; r < nb; ++r) {
            uint32_t run = g.first[r];
            for (int c = 0; c < NCELL; ++c) {
                cellcur[r * NCELL + c] = run;
                run += cellcnt[r * NCELL + c];
            }
        }
        g.sorted.assign(running, 0);
        for (size_t i = 0; i < n; ++i) {
            uint32_t r0 = prank[i];
            int a[D];
            for (int k = 0; k < D; ++k) a[k] = plocal[i * D + k];
            g.sorted[cellcur[r0 * NCELL + cell_index(a)]++] = (uint32_t)i;
            for (int s = 1; s < Geo<D>::NASSOC; ++s) {
                const int *sh = assoc_shift<D>(s);
                if (extra_spills(a, sh)) {
                    uint32_t rb = nbh[r0 * (Geo<D>::NASSOC - 1) + s - 1];
                    g.sorted[cursor[rb * NB + extra_bucket(a, sh)]++] = (uint32_t)i;
                }
            }
        }
        return true;
    }

    // p2g_scatter_style (shaders/slosh/solver/p2g_scatter_style.slang:43-155).
    void p2g(Grid<T, D> &g) {
        const size_t nb = g.keys.size();
        g.nodes.assign(nb * 64 * 4, T(0));
        const T inv_cell_width = T(1.0) / h;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
        for (long long rb = 0; rb < (long long)nb; ++rb) {
            const size_t r = (size_t)rb;
            const uint32_t first = g.first[r], last = first + g.npe[r];
            const uint32_t primaries_end = first + g.np[r];
            const int *bv = g.vid[r].data();
            // per-entry slab keys (shared_zkey)
            std::vector<int> zkey(g.npe[r]);
            for (uint32_t e = first; e < last; ++e) {
                size_t pid = g.sorted[e];
                T assoc_cell = round_even(p.x[pid * D + (D - 1)] / h) - T(1.0);
                zkey[e - first] = std::max((int)assoc_cell - bv[D - 1] * Geo<D>::BW, -2);
            }
            for (int tid = 0; tid < 64; ++tid) {
                int lc[D];
                if constexpr (D == 3) {
                    lc[0] = tid % 4;
                    lc[1] = (tid / 4) % 4;
                    lc[2] = tid / 16;
                } else {
                    lc[0] = tid % 8;
                    lc[1] = tid / 8;
                }
                T cell_pos[D];
                for (int k = 0; k < D; ++k) cell_pos[k] = T(bv[k] * Geo<D>::BW + lc[k]) * h;
                const int node_slab = lc[D - 1];
                T acc[D + 1];
                for (int k = 0; k <= D; ++k) acc[k] = T(0);
                for (uint32_t chunk = first; chunk < last; chunk += 64) {
                    uint32_t chunk_len = std::min<uint32_t>(64, last - chunk);
                    int zmin = zkey[chunk - first], zmax = zkey[chunk - first + chunk_len - 1];
                    if (primaries_end > chunk && primaries_end < chunk + chunk_len) {
                        uint32_t bb = primaries_end - chunk;
                        zmin = std::min(zmin, zkey[chunk - first + bb]);
                        zmax = std::max(zmax, zkey[chunk - first + bb - 1]);
                    }
                    if (!(node_slab >= zmin && node_slab <= zmax + 2)) continue;
                    for (uint32_t e = chunk; e < chunk + chunk_len; ++e) {
                        size_t pid = g.sorted[e];
                        T dpt[D];
                        for (int k = 0; k < D; ++k) dpt[k] = cell_pos[k] - p.x[pid * D + k];
                        T weight = kernel_eval(dpt[0] * inv_cell_width) * kernel_eval(dpt[1] * inv_cell_width);
                        if constexpr (D == 3) weight = weight * kernel_eval(dpt[2] * inv_cell_width);
                        if (weight != T(0)) {
                            const T m = p.mass[pid];
                            for (int j = 0; j < D; ++j) {
                                // mul(dpt, C_s)_j = sum_k dpt_k C[j][k]
                                T cm = 0;
                                for (int k = 0; k < D; ++k) cm += dpt[k] * p.C[pid * D * D + j * D + k];
                                T mom = cm + (p.v[pid * D + j] * m + p.fdt[pid * D + j]);
                                acc[j] += mom * weight;
                            }
                            acc[D] += m * weight;
                        }
                    }
                }
                for (int k = 0; k <= D; ++k) g.nodes[(r * 64 + tid) * 4 + k] = acc[k];
            }
        }
    }

    static void local_of(int tid, int *lc) {
        if constexpr (D == 3) {
            lc[0] = tid % 4;
            lc[1] = (tid / 4) % 4;
            lc[2] = tid / 16;
        } else {
            lc[0] = tid % 8;
            lc[1] = tid / 8;
        }
    }

    // grid_update (shaders/slosh/solver/grid_update.slang:38-163).  Bodies
    // coupled two-way (an extension: slosh's GPU never fills its impulse
    // buffer) project the node velocity relative to the body velocity at the
    // node and receive the momentum the node loses as an impulse at the
    // node, summed in 64-bit fixed point; while one exists, every node runs
    // collision detection instead of the cache.
    void grid_update(Grid<T, D> &g, const Grid<T, D> &pg) {
        const size_t nb = g.keys.size();
        g.coll.assign(nb * 64, NodeCollision<T, D>{});
        const T vel_limit = h / dt;
        const bool dynamic = coll_dynamic();
        impulses.assign(bodies.size() * 6, 0);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long rb = 0; rb < (long long)nb; ++rb) {
            const size_t r = (size_t)rb;
            auto pit = pg.rank.find(g.keys[r]);
            for (int tid = 0; tid < 64; ++tid) {
                int lc[D];
                local_of(tid, lc);
                T cell_pos[D];
                for (int k = 0; k < D; ++k) cell_pos[k] = T(g.vid[r][k] * Geo<D>::BW + lc[k]) * h;
                T *node = &g.nodes[(r * 64 + tid) * 4];
                // update_single_cell
                const T mass = node[D];
                const T inv_mass = mass > T(0) ? T(1.0) / mass : T(0);
                T vel[D];
                for (int k = 0; k < D; ++k) {
                    T v = (node[k] + mass * gravity[k] * dt) * inv_mass;
                    vel[k] = std::min(std::max(v, -vel_limit), vel_limit);
                }
                NodeCollision<T, D> c;
                if (pit != pg.rank.end() && !pg.coll.empty() && !dynamic) {
                    c = pg.coll[(size_t)pit->second * 64 + tid];
                } else {
                    c = collide<T, D>(bodies, h, cell_pos);
                }
                g.coll[r * 64 + tid] = c;
                if (c.valid != 0) {
                    const Body<T, D> &b = bodies[c.collider_id];
                    T dd = 0;
                    for (int k = 0; k < D; ++k) dd += (cell_pos[k] - c.point[k]) * c.normal[k];
                    T dist = dd - h;
                    if (b.coupling == SLOSH_COUPLING_TWO_WAY) {
                        T com[3] = {0, 0, 0}, r[3] = {0, 0, 0}, vb[3] = {0, 0, 0};
                        Pose<T, D>::mul_pt(b, b.local_com, com);
                        for (int k = 0; k < D; ++k) r[k] = cell_pos[k] - com[k];
                        if constexpr (D == 3) {
                            vb[0] = b.linvel[0] + b.angvel[1] * r[2] - b.angvel[2] * r[1];
                            vb[1] = b.linvel[1] + b.angvel[2] * r[0] - b.angvel[0] * r[2];
                            vb[2] = b.linvel[2] + b.angvel[0] * r[1] - b.angvel[1] * r[0];
                        } else {
                            vb[0] = b.linvel[0] - b.angvel[0] * r[1];
                            vb[1] = b.linvel[1] + b.angvel[0] * r[0];
                        }
                        T rel[D];
                        for (int k = 0; k < D; ++k) rel[k] = vel[k] - vb[k];
                        project_velocity<T, D>(b.bc_type, b.friction, rel, c.normal, dist, dt);
                        T J[3] = {0, 0, 0};
                        for (int k = 0; k < D; ++k) {
                            const T nv = rel[k] + vb[k];
                            J[k] = mass * (vel[k] - nv);
                            vel[k] = nv;
                        }
                        if (mass > T(0)) {
                            T A[3] = {0, 0, 0};
                            if constexpr (D == 3) {
                                A[0] = r[1] * J[2] - r[2] * J[1];
                                A[1] = r[2] * J[0] - r[0] * J[2];
                                A[2] = r[0] * J[1] - r[1] * J[0];
                            } else {
                                A[0] = r[0] * J[1] - r[1] * J[0];
                            }
                            long long *acc = &impulses[(size_t)c.collider_id * 6];
                            for (int k = 0; k < 3; ++k) {
                                const long long jl = impulse_units((double)J[k]), ja = impulse_units((double)A[k]);
#pragma omp atomic
                                acc[k] += jl;
#pragma omp atomic
                                acc[3 + k] += ja;
                            }
                        }
                    } else {
                        project_velocity<T, D>(b.bc_type, b.friction, vel, c.normal, dist, dt);
                    }
                }
                for (int k = 0; k < D; ++k) node[k] = vel[k];
                node[D] = mass;
            }
        }
    }

    // g2p (shaders/slosh/solver/g2p.slang:36-265).  Writes v, grad v (into C)
    // and vel_grad_det for every primary particle.
    void g2p(const Grid<T, D> &g) {
        const size_t nb = g.keys.size();
        const int SW = Geo<D>::SW;
        const int NS = (D == 3) ? SW * SW * SW : SW * SW;
        const T inv_d = T(4.0) / (h * h);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 4)
        for (long long rb = 0; rb < (long long)nb; ++rb) {
            const size_t r = (size_t)rb;
            std::vector<T> sh(NS * 4, T(0));
            for (int oct = 0; oct < Geo<D>::NASSOC; ++oct) {
                const int *o = assoc_shift<D>(oct);
                int q[3] = {0, 0, 0};
                for (int k = 0; k < D; ++k) q[k] = g.vid[r][k] + o[k];
                auto it = g.rank.find(pack_key<D>(q));
                for (int tid = 0; tid < 64; ++tid) {
                    int lc[D];
                    local_of(tid, lc);
                    bool exists = true;
                    for (int k = 0; k < D; ++k)
                        if (o[k] == 1 && lc[k] > 1) exists = false;
                    if (!exists) continue;
                    int si[D];
                    for (int k = 0; k < D; ++k) si[k] = o[k] * Geo<D>::BW + lc[k];
                    int flat = (D == 3) ? si[0] + si[1] * SW + si[2] * SW * SW : si[0] + si[1] * SW;
                    for (int c = 0; c < 4; ++c)
                        sh[flat * 4 + c] =
                            (it != g.rank.end()) ? g.nodes[((size_t)it->second * 64 + tid) * 4 + c] : T(0);
                }
            }
            for (uint32_t e = g.first[r]; e < g.first[r] + g.np[r]; ++e) {
                const size_t pid = g.sorted[e];
                T vel[D], grad[D][D], vgd = 0;
                for (int k = 0; k < D; ++k) {
                    vel[k] = 0;
                    for (int l = 0; l < D; ++l) grad[k][l] = 0;
                }
                if (p.enabled[pid] != 0) {
                    T ref[D], w[D][3];
                    int a[D];
                    for (int k = 0; k < D; ++k) {
                        T xk = p.x[pid * D + k];
                        ref[k] = (round_even(xk / h) - T(1.0)) * h - xk;
                        kernel_eval_all(-ref[k] / h, w[k]);
                        T assoc_cell = round_even(xk / h) - T(1.0);
                        T ab = std::floor(assoc_cell / T(Geo<D>::BW)) * T(Geo<D>::BW);
                        a[k] = (int)(assoc_cell - ab);
                    }
                    for (int i = 0; i < Geo<D>::NBH; ++i) {
                        const int *s = nbh_shift<D>(i);
                        int si[D];
                        for (int k = 0; k < D; ++k) si[k] = a[k] + s[k];
                        int flat = (D == 3) ? si[0] + si[1] * SW + si[2] * SW * SW : si[0] + si[1] * SW;
                        const T *cell = &sh[flat * 4];
                        T dpt[D];
                        for (int k = 0; k < D; ++k) dpt[k] = ref[k] + T(s[k]) * h;
                        T weight = w[0][s[0]] * w[1][s[1]];
                        if constexpr (D == 3) weight = weight * w[2][s[2]];
                        for (int k = 0; k < D; ++k) vel[k] += cell[k] * weight;
                        const T wi = weight * inv_d;
                        // grad[c][r] += wi * (v_c * dpt_r)
                        for (int rr = 0; rr < D; ++rr)
                            for (int cc = 0; cc < D; ++cc) grad[cc][rr] += wi * (cell[cc] * dpt[rr]);
                        T dotv = 0;
                        for (int k = 0; k < D; ++k) dotv += cell[k] * dpt[k];
                        vgd += weight * inv_d * dotv;
                    }
                }
                for (int k = 0; k < D; ++k) {
                    p.v[pid * D + k] = vel[k];
                    for (int l = 0; l < D; ++l) p.C[pid * D * D + k * D + l] = grad[k][l];
                }
                p.vgd[pid] = vgd;
            }
        }
    }

    // particle_update (shaders/slosh/solver/particle_update.slang:34-160)
    // with DefaultParticleModel::update (models/default.slang:51-92) and the
    // Tait fluid extension.
    void particle_update() {
        const T inv_d = T(4.0) / (h * h);
        const T vlim = h / dt;
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long long ii = 0; ii < (long long)p.n; ++ii) {
            const size_t i = (size_t)ii;
            const uint32_t tag = p.tag[i];
            const bool fluid = tag == SLOSH_MODEL_FLUID_TAIT;
            T vel[D];
            T len2 = 0;
            for (int k = 0; k < D; ++k) {
                vel[k] = p.v[i * D + k];
                len2 += vel[k] * vel[k];
            }
            T len = std::sqrt(len2);
            if (len > h / dt)
                for (int k = 0; k < D; ++k) vel[k] = vel[k] / len * h / dt;
            (void)vlim;
            for (int k = 0; k < D; ++k) vel[k] = vel[k] / (T(1.0) + p.damping[i] * dt);
            if (p.fixed[i] != 0)
                for (int k = 0; k < D; ++k) vel[k] = T(0);
            T newx[D];
            for (int k = 0; k < D; ++k) newx[k] = p.x[i * D + k] + vel[k] * dt;
            Mat<T, D> F, A;
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) {
                    F.m[r][c] = p.F[i * D * D + r * D + c];
                    A.m[r][c] = p.C[i * D * D + r * D + c];  // velocity gradient
                }
            if (!fluid) {
                // F += (grad v * dt) F
                Mat<T, D> Ad, Fn;
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) Ad.m[r][c] = A.m[r][c] * dt;
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) {
                        T acc = 0;
                        for (int k = 0; k < D; ++k) acc += F.m[k][c] * Ad.m[r][k];
                        Fn.m[r][c] = F.m[r][c] + acc;
                    }
                F = Fn;
            } else {
                T f0 = F.m[0][0];
                T nf = f0 + f0 * p.vgd[i] * dt;
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) F.m[r][c] = (r == c) ? nf : T(0);
            }
            if (p.fixed[i] != 0)
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) A.m[r][c] = T(0);
            // Constitutive model.
            T *mp = &p.model[i * 12];
            Mat<T, D> tau{};
            switch (tag) {
                case SLOSH_MODEL_ELASTIC_LINEAR:
                    tau = fixed_corotated<T, D>(F, mp[0], mp[1]);
                    break;
                case SLOSH_MODEL_ELASTIC_NEO_HOOKEAN:
                    tau = neo_hookean<T, D>(F, mp[0], mp[1]);
                    break;
                case SLOSH_MODEL_SAND_LINEAR:
                    drucker_prager<T, D>(mp, mp + 3, F);
                    tau = fixed_corotated<T, D>(F, mp[9], mp[10]);
                    break;
                case SLOSH_MODEL_SAND_NEO_HOOKEAN:
                    drucker_prager<T, D>(mp, mp + 3, F);
                    tau = neo_hookean<T, D>(F, mp[9], mp[10]);
                    break;
                case SLOSH_MODEL_FLUID_TAIT:
                    tau = tait_fluid<T, D>(F, mp[1], mp[2]);
                    break;
                default:
                    break;
            }
            const T m = p.mass[i];
            const T coef = p.V0[i] * inv_d * dt;
            Mat<T, D> aff;
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) aff.m[r][c] = A.m[r][c] * m - tau.m[r][c] * coef;
            bool finite = true;
            for (int k = 0; k < D; ++k) finite = finite && (newx[k] == newx[k]);
            if (finite && det<T, D>(F) > T(0)) {
                for (int k = 0; k < D; ++k) p.x[i * D + k] = newx[k];
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) p.C[i * D * D + r * D + c] = aff.m[r][c];
                for (int k = 0; k < D; ++k) p.v[i * D + k] = vel[k];
            } else {
                p.enabled[i] = 0;
                for (int k = 0; k < D; ++k) p.v[i * D + k] = T(0);
                for (int r = 0; r < D; ++r)
                    for (int c = 0; c < D; ++c) {
                        F.m[r][c] = (r == c) ? T(1) : T(0);
                        p.C[i * D * D + r * D + c] = T(0);
                    }
                p.mass[i] = T(0);
            }
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) p.F[i * D * D + r * D + c] = F.m[r][c];
            for (int k = 0; k < D; ++k) p.fdt[i * D + k] = T(0);
        }
    }

    // update (shaders/slosh/solver/rigid_impulses.slang:72-121) with
    // integrate_velocity (shaders/slosh/rbd/dynamics/body.slang:117-130).
    // The incremental impulse is always zero in the reference (no kernel
    // writes it); bodies coupled two-way apply the grid's impulse sums here
    // (apply_impulse, body.slang:62-70) followed by the velocity caps.
    void rigid_update() {
        for (size_t bi = 0; bi < bodies.size(); ++bi) {
            Body<T, D> &b = bodies[bi];
            if (b.coupling == SLOSH_COUPLING_TWO_WAY && impulses.size() >= (bi + 1) * 6) {
                T jl[3], ja[3];
                for (int k = 0; k < 3; ++k) {
                    jl[k] = (T)((double)impulses[bi * 6 + k] / IMPULSE_UNITS);
                    ja[k] = (T)((double)impulses[bi * 6 + 3 + k] / IMPULSE_UNITS);
                }
                for (int k = 0; k < D; ++k) b.linvel[k] += b.inv_mass[k] * jl[k];
                if constexpr (D == 3) {
                    T R[3][3], Iw[9];
                    quat_to_mat(b.rot, R);
                    conjugate(R, b.inv_inertia_local, Iw, true);
                    for (int i = 0; i < 3; ++i)
                        b.angvel[i] += Iw[i * 3] * ja[0] + Iw[i * 3 + 1] * ja[1] + Iw[i * 3 + 2] * ja[2];
                } else {
                    b.angvel[0] += b.inv_inertia_local[0] * ja[0];
                }
                bool pushed = false;
                for (int k = 0; k < 3; ++k) pushed = pushed || jl[k] != T(0) || ja[k] != T(0);
                if (pushed) {
                    const T lin_limit = T(0.1) * h / dt, ang_limit = T(1);
                    const int na = D == 3 ? 3 : 1;
                    T l2 = 0, a2 = 0;
                    for (int k = 0; k < D; ++k) l2 += b.linvel[k] * b.linvel[k];
                    for (int k = 0; k < na; ++k) a2 += b.angvel[k] * b.angvel[k];
                    const T ln = std::sqrt(l2), an = std::sqrt(a2);
                    if (ln > lin_limit)
                        for (int k = 0; k < D; ++k) b.linvel[k] = b.linvel[k] * (lin_limit / ln);
                    if (an > ang_limit)
                        for (int k = 0; k < na; ++k) b.angvel[k] = b.angvel[k] * (ang_limit / an);
                }
            }
            T init_com[3] = {0, 0, 0};
            Pose<T, D>::mul_pt(b, b.local_com, init_com);
            if constexpr (D == 3) {
                T sa[3] = {b.angvel[0] * dt, b.angvel[1] * dt, b.angvel[2] * dt};
                T ang = std::sqrt(sa[0] * sa[0] + sa[1] * sa[1] + sa[2] * sa[2]);
                T dq[4] = {0, 0, 0, 1};
                if (ang > T(0)) {
                    T s = std::sin(ang / T(2)) / ang;
                    dq[0] = sa[0] * s;
                    dq[1] = sa[1] * s;
                    dq[2] = sa[2] * s;
                    dq[3] = std::cos(ang / T(2));
                }
                T rel[3] = {b.tra[0] - init_com[0], b.tra[1] - init_com[1], b.tra[2] - init_com[2]};
                T rr[3];
                quat_rotate(dq, rel, rr);
                for (int k = 0; k < 3; ++k) b.tra[k] = init_com[k] + rr[k] * b.scale + b.linvel[k] * dt;
                T nq[4];
                quat_mul(dq, b.rot, nq);
                T n2 = nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3];
                T f = T(0.5) * (T(3.0) - n2);
                for (int k = 0; k < 4; ++k) b.rot[k] = nq[k] * f;
            } else {
                T a = b.angvel[0] * dt;
                T c = std::cos(a), s = std::sin(a);
                T rel0 = b.tra[0] - init_com[0], rel1 = b.tra[1] - init_com[1];
                T r0 = c * rel0 - s * rel1, r1 = s * rel0 + c * rel1;
                b.tra[0] = init_com[0] + r0 * b.scale + b.linvel[0] * dt;
                b.tra[1] = init_com[1] + r1 * b.scale + b.linvel[1] * dt;
                T nc = c * b.rot[0] - s * b.rot[1], ns = s * b.rot[0] + c * b.rot[1];
                b.rot[0] = nc;
                b.rot[1] = ns;
            }
            for (int k = 0; k < D; ++k)
                b.linvel[k] = b.linvel[k] + gravity[k] * ((b.inv_mass[k] != T(0)) ? T(1) : T(0)) * dt;
        }
    }

    // One substep in the order of MpmPipeline::launch_step.  The grid of the
    // previous substep is kept for the node-collision cache.
    int step() {
        std::swap(grid, prev);
        if (!grid_build(grid)) return SLOSH_E_OVERFLOW;
        p2g(grid);
        grid_update(grid, prev);
        g2p(grid);
        particle_update();
        rigid_update();
        return SLOSH_OK;
    }
};

// --------------------------------------------------------------------------
// Record conversion.
// --------------------------------------------------------------------------
template <typename T, int D> void load_particles(Particles<T, D> &p, const slosh_particle *src, size_t n) {
    p.n = n;
    p.x.assign(n * D, 0);
    p.v.assign(n * D, 0);
    p.fdt.assign(n * D, 0);
    p.C.assign(n * D * D, 0);
    p.F.assign(n * D * D, 0);
    p.vgd.assign(n, 0);
    p.V0.assign(n, 0);
    p.r0.assign(n, 0);
    p.mass.assign(n, 0);
    p.damping.assign(n, 0);
    p.phase.assign(n, 0);
    p.enabled.assign(n, 0);
    p.fixed.assign(n, 0);
    p.tag.assign(n, 0);
    p.model.assign(n * 12, 0);
    for (size_t i = 0; i < n; ++i) {
        const slosh_particle &s = src[i];
        for (int k = 0; k < D; ++k) {
            p.x[i * D + k] = s.position[k];
            p.v[i * D + k] = s.velocity[k];
            p.fdt[i * D + k] = s.force_dt[k];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                // column-major record: element (r, c) at c*3 + r
                p.F[i * D * D + r * D + c] = s.def_grad[c * 3 + r];
                p.C[i * D * D + r * D + c] = s.affine[c * 3 + r];
            }
        p.vgd[i] = s.vel_grad_det;
        p.V0[i] = s.init_volume;
        p.r0[i] = s.init_radius;
        p.mass[i] = s.mass;
        p.damping[i] = s.damping;
        p.phase[i] = s.phase;
        p.enabled[i] = s.enabled;
        p.fixed[i] = s.fixed;
        p.tag[i] = s.model.tag;
        for (int k = 0; k < 12; ++k) p.model[i * 12 + k] = s.model.data[k];
    }
}

template <typename T, int D> void store_particles(const Particles<T, D> &p, slosh_particle *dst, size_t n) {
    for (size_t i = 0; i < n && i < p.n; ++i) {
        slosh_particle &s = dst[i];
        std::memset(&s, 0, sizeof(s));
        for (int k = 0; k < D; ++k) {
            s.position[k] = (float)p.x[i * D + k];
            s.velocity[k] = (float)p.v[i * D + k];
            s.force_dt[k] = (float)p.fdt[i * D + k];
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                s.def_grad[c * 3 + r] = (float)p.F[i * D * D + r * D + c];
                s.affine[c * 3 + r] = (float)p.C[i * D * D + r * D + c];
            }
        s.vel_grad_det = (float)p.vgd[i];
        s.init_volume = (float)p.V0[i];
        s.init_radius = (float)p.r0[i];
        s.mass = (float)p.mass[i];
        s.damping = (float)p.damping[i];
        s.phase = (float)p.phase[i];
        s.enabled = p.enabled[i];
        s.fixed = p.fixed[i];
        s.model.tag = p.tag[i];
        for (int k = 0; k < 12; ++k) s.model.data[k] = (float)p.model[i * 12 + k];
    }
}

template <typename T, int D> Body<T, D> load_body(const slosh_body &s) {
    Body<T, D> b{};
    uint32_t ty;
    std::memcpy(&ty, &s.shape_a[3], 4);
    b.shape_type = ty;
    for (int k = 0; k < 4; ++k) {
        b.sa[k] = s.shape_a[k];
        b.sb[k] = s.shape_b[k];
        b.rot[k] = s.rotation[k];
    }
    for (int k = 0; k < 3; ++k) {
        b.tra[k] = s.translation[k];
        b.linvel[k] = s.linvel[k];
        b.angvel[k] = s.angvel[k];
        b.inv_mass[k] = s.inv_mass[k];
        b.local_com[k] = s.local_com[k];
    }
    b.scale = s.translation[3];
    std::memcpy(b.inv_inertia, s.inv_inertia, sizeof(b.inv_inertia));
    b.bc_type = s.bc_type;
    b.friction = s.bc_friction;
    b.coupling = s.coupling;
    if constexpr (D == 3) {  // the world-space record taken to the body frame
        T W[9], R[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) W[r * 3 + c] = (T)s.inv_inertia[c * 4 + r];
        quat_to_mat(b.rot, R);
        conjugate(R, W, b.inv_inertia_local, false);
    } else {
        b.inv_inertia_local[0] = (T)s.inv_inertia[0];
    }
    return b;
}

template <typename T, int D> void store_body(const Body<T, D> &b, slosh_body &s) {
    std::memset(&s, 0, sizeof(s));
    for (int k = 0; k < 4; ++k) {
        s.shape_a[k] = (float)b.sa[k];
        s.shape_b[k] = (float)b.sb[k];
        s.rotation[k] = (float)b.rot[k];
    }
    std::memcpy(&s.shape_a[3], &b.shape_type, 4);
    for (int k = 0; k < 3; ++k) {
        s.translation[k] = (float)b.tra[k];
        s.linvel[k] = (float)b.linvel[k];
        s.angvel[k] = (float)b.angvel[k];
        s.inv_mass[k] = (float)b.inv_mass[k];
        s.local_com[k] = (float)b.local_com[k];
    }
    s.translation[3] = (float)b.scale;
    std::memcpy(s.inv_inertia, b.inv_inertia, sizeof(s.inv_inertia));
    s.bc_type = b.bc_type;
    s.bc_friction = (float)b.friction;
    s.coupling = b.coupling;
    if constexpr (D == 3) {  // world-space inverse inertia at the current pose
        T W[9], R[3][3];
        quat_to_mat(b.rot, R);
        conjugate(R, b.inv_inertia_local, W, true);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) s.inv_inertia[c * 4 + r] = (float)W[r * 3 + c];
    } else {
        s.inv_inertia[0] = (float)b.inv_inertia_local[0];
    }
}

// Type-erased context.
struct AnyCtx {
    virtual ~AnyCtx() {}
    virtual void set_params(const float *g, float dt) = 0;
    virtual int set_particles(const slosh_particle *p, uint32_t n) = 0;
    virtual int get_particles(slosh_particle *p, uint32_t n) = 0;
    virtual int set_bodies(const slosh_body *b, uint32_t n) = 0;
    virtual int add_trimesh(const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt) = 0;
    virtual int get_bodies(slosh_body *b, uint32_t n) = 0;
    virtual int step(uint32_t nsteps, int nthreads) = 0;
    virtual int stages(int last, int nthreads) = 0;
    virtual uint32_t num_blocks() = 0;
    virtual uint32_t num_sorted() = 0;
    virtual int grid_get(uint32_t *, uint32_t *, uint32_t *, uint32_t *, uint32_t *, uint32_t *) = 0;
    virtual int nodes_get(float *out) = 0;
    virtual void totals(double *out) = 0;
    virtual void node_totals(double *out) = 0;
    virtual uint32_t timestep_bound() = 0;
};

// GpuTimestepBounds::secs_to_int (shaders/slosh/solver/timestep_bound.slang:20-27):
// floor(secs * 1e12) as u32, saturating.
template <typename T> inline uint32_t secs_to_int(T secs) {
    const T x = std::floor(secs * T(1.0e12));
    if (!(x > T(0))) return 0u;
    return x >= T(4294967296.0) ? 0xffffffffu : (uint32_t)x;
}

// ElasticitySoundSpeedTimestepBound::timestep_bound (models/utils.slang:119-136).
template <typename T>
inline T sound_speed_bound(T alpha, T bulk, T shear, T density0, T det_f, T vlen, T h) {
    const T rho = density0 / std::max(det_f, T(1.0e-6));
    const T c = std::sqrt((bulk + shear * T(4.0) / T(3.0)) / rho);
    return alpha * h / std::max(vlen, c);
}

// LinearElasticModel / NeoHookeanModel::timestep_bound
// (linear_elasticity.slang:117-133, neo_hookean_elasticity.slang:29-45):
// bulk = lambda + 2 mu / 3, shear = mu (models/utils.slang:22-28).
template <typename T> inline T elastic_bound(const T *p, T density0, T det_f, T vlen, T h) {
    const T bulk = p[0] + T(2.0) * p[1] / T(3.0);
    return sound_speed_bound(p[2], bulk, p[1], density0, det_f, vlen, h);
}

template <typename T, int D> struct CtxImpl : AnyCtx {
    Ctx<T, D> c;
    void set_params(const float *g, float dt) override {
        for (int k = 0; k < 3; ++k) c.gravity[k] = g[k];
        c.dt = dt;
    }
    int set_particles(const slosh_particle *p, uint32_t n) override {
        load_particles<T, D>(c.p, p, n);
        c.grid = Grid<T, D>();
        c.prev = Grid<T, D>();
        return SLOSH_OK;
    }
    int get_particles(slosh_particle *p, uint32_t n) override {
        store_particles<T, D>(c.p, p, n);
        return SLOSH_OK;
    }
    int set_bodies(const slosh_body *b, uint32_t n) override {
        c.bodies.clear();
        for (uint32_t i = 0; i < n; ++i) c.bodies.push_back(load_body<T, D>(b[i]));
        return link_meshes();
    }
    // A trimesh record names its mesh by the ordinal in shape_b[2].
    int link_meshes() {
        for (auto &bd : c.bodies) {
            bd.mesh = nullptr;
            if (bd.shape_type != SLOSH_SHAPE_TRIMESH) continue;
            uint32_t ord;
            const float f = (float)bd.sb[2];
            std::memcpy(&ord, &f, 4);
            if (D != 3 || ord >= c.meshes.size()) return SLOSH_E_INVALID;
            bd.mesh = &c.meshes[ord];
        }
        return SLOSH_OK;
    }
    int add_trimesh(const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt) override {
        for (size_t k = 0; k < 3 * (size_t)nt; ++k)
            if (tri[k] >= nv) return SLOSH_E_INVALID;
        c.meshes.push_back(make_mesh<T>(v, nv, tri, nt));
        link_meshes();
        return (int)c.meshes.size() - 1;
    }
    int get_bodies(slosh_body *b, uint32_t n) override {
        for (uint32_t i = 0; i < n && i < c.bodies.size(); ++i) store_body<T, D>(c.bodies[i], b[i]);
        return SLOSH_OK;
    }
    int step(uint32_t nsteps, int nthreads) override {
        c.nthreads = nthreads;
        for (uint32_t s = 0; s < nsteps; ++s) {
            int st = c.step();
            if (st) return st;
        }
        return SLOSH_OK;
    }
    // Runs the first stages of one substep without committing it
    // (0 = grid build, 1 = + P2G, 2 = + grid update).
    int stages(int last, int nthreads) override {
        c.nthreads = nthreads;
        Grid<T, D> g;
        if (!c.grid_build(g)) return SLOSH_E_OVERFLOW;
        if (last >= 1) c.p2g(g);
        if (last >= 2) c.grid_update(g, c.grid);
        scratch = std::move(g);
        return SLOSH_OK;
    }
    uint32_t num_blocks() override { return (uint32_t)scratch.keys.size(); }
    uint32_t num_sorted() override { return (uint32_t)scratch.sorted.size(); }
    int grid_get(uint32_t *keys, uint32_t *first, uint32_t *np, uint32_t *npe, uint32_t *counts,
                 uint32_t *sorted) override {
        const size_t nb = scratch.keys.size();
        if (keys) std::memcpy(keys, scratch.keys.data(), nb * 4);
        if (first) std::memcpy(first, scratch.first.data(), nb * 4);
        if (np) std::memcpy(np, scratch.np.data(), nb * 4);
        if (npe) std::memcpy(npe, scratch.npe.data(), nb * 4);
        if (counts) std::memcpy(counts, scratch.counts.data(), scratch.counts.size() * 4);
        if (sorted) std::memcpy(sorted, scratch.sorted.data(), scratch.sorted.size() * 4);
        return SLOSH_OK;
    }
    // Nodes as 4 floats: (momentum or velocity with z = 0 in 2D, mass).
    int nodes_get(float *out) override {
        const size_t nn = scratch.nodes.size() / 4;
        for (size_t i = 0; i < nn; ++i) {
            for (int k = 0; k < 3; ++k) out[i * 4 + k] = (k < D) ? (float)scratch.nodes[i * 4 + k] : 0.f;
            out[i * 4 + 3] = (float)scratch.nodes[i * 4 + D];
        }
        return SLOSH_OK;
    }
    // Sums of node mass and momentum in double (conservation checks).
    void node_totals(double *out) override {
        for (int k = 0; k < 4; ++k) out[k] = 0;
        const size_t nn = scratch.nodes.size() / 4;
        for (size_t i = 0; i < nn; ++i) {
            for (int k = 0; k < D; ++k) out[k] += (double)scratch.nodes[i * 4 + k];
            out[3] += (double)scratch.nodes[i * 4 + D];
        }
    }
    // Totals in double: mass, momentum (D), for conservation checks.
    void totals(double *out) override {
        for (int k = 0; k < 4; ++k) out[k] = 0;
        for (size_t i = 0; i < c.p.n; ++i) {
            out[0] += (double)c.p.mass[i];
            for (int k = 0; k < D; ++k) out[1 + k] += (double)c.p.mass[i] * (double)c.p.v[i * D + k];
        }
    }
    // estimate_timestep_bound (timestep_bound.slang:37-91) over all particles,
    // as the u32 picosecond count; DefaultParticleModel::timestep_bound
    // (models/default.slang:94-127) per model, and for the Tait fluid the
    // sound speed c^2 = K J^-gamma / rho with CFL 0.5.
    uint32_t timestep_bound() override {
        uint32_t best = 0xffffffffu;
        const T h = c.h;
        for (size_t i = 0; i < c.p.n; ++i) {
            if (!c.p.enabled[i]) continue;
            const T density0 = c.p.mass[i] / c.p.V0[i];
            Mat<T, D> F;
            for (int r = 0; r < D; ++r)
                for (int q = 0; q < D; ++q) F.m[r][q] = c.p.F[i * D * D + r * D + q];
            const T det_f = det<T, D>(F);
            T v2 = T(0);
            for (int k = 0; k < D; ++k) v2 = v2 + c.p.v[i * D + k] * c.p.v[i * D + k];
            const T vlen = std::sqrt(v2);
            const T *p = &c.p.model[i * 12];
            T dt;
            switch (c.p.tag[i]) {
                case SLOSH_MODEL_ELASTIC_LINEAR:
                case SLOSH_MODEL_ELASTIC_NEO_HOOKEAN:
                    dt = elastic_bound<T>(p, density0, det_f, vlen, h);
                    break;
                case SLOSH_MODEL_SAND_LINEAR:
                case SLOSH_MODEL_SAND_NEO_HOOKEAN:
                    dt = elastic_bound<T>(p + 9, density0, det_f, vlen, h);
                    break;
                case SLOSH_MODEL_FLUID_TAIT: {
                    const T J = F.m[0][0];
                    const T rho = density0 / std::max(J, T(1.0e-6));
                    const T cs = std::sqrt(p[1] * std::pow(std::max(J, T(1.0e-6)), -p[2]) / rho);
                    dt = T(0.5) * h / std::max(vlen, cs);
                    break;
                }
                default:
                    dt = T(0);
                    break;
            }
            dt = std::min(dt, h / vlen);
            best = std::min(best, secs_to_int<T>(dt));
        }
        return best;
    }
    Grid<T, D> scratch;
};

}  // namespace orc

extern "C" {

void *orc_create(uint32_t dim, uint32_t use_double, float cell_width, uint32_t grid_capacity) {
    orc::AnyCtx *c = nullptr;
    uint32_t cap = 1;
    while (cap < grid_capacity) cap <<= 1;
    if (dim == 3 && !use_double) {
        auto *x = new orc::CtxImpl<float, 3>();
        x->c.h = cell_width;
        x->c.capacity = cap;
        c = x;
    } else if (dim == 3) {
        auto *x = new orc::CtxImpl<double, 3>();
        x->c.h = cell_width;
        x->c.capacity = cap;
        c = x;
    } else if (dim == 2 && !use_double) {
        auto *x = new orc::CtxImpl<float, 2>();
        x->c.h = cell_width;
        x->c.capacity = cap;
        c = x;
    } else if (dim == 2) {
        auto *x = new orc::CtxImpl<double, 2>();
        x->c.h = cell_width;
        x->c.capacity = cap;
        c = x;
    }
    return c;
}

void orc_destroy(void *c) { delete (orc::AnyCtx *)c; }
uint32_t orc_timestep_bound(void *c) { return ((orc::AnyCtx *)c)->timestep_bound(); }

// Shape::project_point_on_boundary of one body record (FP32), for tests:
// returns 1 when the shape is supported, with the projection and "inside".
int orc_project(uint32_t dim, const slosh_body *body, const float *pt, float *out, int *inside) {
    bool in = false;
    bool ok;
    if (dim == 3) {
        const orc::Body<float, 3> b = orc::load_body<float, 3>(*body);
        ok = orc::project_on_boundary<float, 3>(b, pt, out, &in);
    } else {
        const orc::Body<float, 2> b = orc::load_body<float, 2>(*body);
        ok = orc::project_on_boundary<float, 2>(b, pt, out, &in);
    }
    *inside = in ? 1 : 0;
    return ok ? 1 : 0;
}
void orc_set_params(void *c, const float *gravity, float dt) { ((orc::AnyCtx *)c)->set_params(gravity, dt); }
int orc_set_particles(void *c, const slosh_particle *p, uint32_t n) {
    return ((orc::AnyCtx *)c)->set_particles(p, n);
}
int orc_get_particles(void *c, slosh_particle *p, uint32_t n) { return ((orc::AnyCtx *)c)->get_particles(p, n); }
int orc_set_bodies(void *c, const slosh_body *b, uint32_t n) { return ((orc::AnyCtx *)c)->set_bodies(b, n); }
// Adds a triangle mesh; returns its ordinal (for shape_b[2] of trimesh
// records) or SLOSH_E_INVALID.
int orc_add_trimesh(void *c, const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt) {
    return ((orc::AnyCtx *)c)->add_trimesh(v, nv, tri, nt);
}
// Projection of a world point on a posed triangle mesh (FP64), within `cap`.
int orc_project_trimesh(const float *v, uint32_t nv, const uint32_t *tri, uint32_t nt, const slosh_body *body,
                        const float *pt, float cap, float *out, int *inside) {
    const orc::Mesh<double> m = orc::make_mesh<double>(v, nv, tri, nt);
    orc::Body<double, 3> b = orc::load_body<double, 3>(*body);
    b.shape_type = SLOSH_SHAPE_TRIMESH;
    b.mesh = &m;
    const double p[3] = {pt[0], pt[1], pt[2]};
    double q[3];
    bool in = false;
    const bool ok = orc::project_on_boundary<double, 3>(b, p, q, &in, (double)cap);
    for (int k = 0; k < 3; ++k) out[k] = (float)q[k];
    *inside = in ? 1 : 0;
    return ok ? 1 : 0;
}
int orc_get_bodies(void *c, slosh_body *b, uint32_t n) { return ((orc::AnyCtx *)c)->get_bodies(b, n); }
int orc_step(void *c, uint32_t nsteps, int nthreads) { return ((orc::AnyCtx *)c)->step(nsteps, nthreads); }
int orc_stages(void *c, int last, int nthreads) { return ((orc::AnyCtx *)c)->stages(last, nthreads); }
uint32_t orc_num_blocks(void *c) { return ((orc::AnyCtx *)c)->num_blocks(); }
uint32_t orc_num_sorted(void *c) { return ((orc::AnyCtx *)c)->num_sorted(); }
int orc_grid_get(void *c, uint32_t *keys, uint32_t *first, uint32_t *np, uint32_t *npe, uint32_t *counts,
                 uint32_t *sorted) {
    return ((orc::AnyCtx *)c)->grid_get(keys, first, np, npe, counts, sorted);
}
int orc_nodes_get(void *c, float *out) { return ((orc::AnyCtx *)c)->nodes_get(out); }
void orc_totals(void *c, double *out) { ((orc::AnyCtx *)c)->totals(out); }
void orc_node_totals(void *c, double *out) { ((orc::AnyCtx *)c)->node_totals(out); }

// WgPrefixSum::eval_cpu (src/grid/prefix_sum.rs:97-110): inclusive running
// sum, then shift right by one with a leading 0.
void orc_prefix_sum(uint32_t *v, uint32_t n) {
    if (n == 0) return;
    for (uint32_t i = 0; i + 1 < n; ++i) v[i + 1] += v[i];
    for (uint32_t i = n - 1; i >= 1; --i) v[i] = v[i - 1];
    v[0] = 0;
}

// The oracle's own SVD (for invariant tests): row-major 3x3 / 2x2 in double.
void orc_svd(uint32_t dim, const double *F, double *U, double *S, double *V) {
    if (dim == 3) orc::svd_jacobi<3>(F, U, S, V);
    else orc::svd_jacobi<2>(F, U, S, V);
}

// Kirchhoff stress of one model for one F (row-major), FP64, for per-model
// checks.  `model` is the 12-word payload; state words may be updated.
int orc_model_stress(uint32_t dim, uint32_t tag, double *model, double *F, double *tau) {
    if (dim == 3) {
        orc::Mat<double, 3> f, t{};
        for (int i = 0; i < 9; ++i) f.m[i / 3][i % 3] = F[i];
        switch (tag) {
            case SLOSH_MODEL_ELASTIC_LINEAR: t = orc::fixed_corotated<double, 3>(f, model[0], model[1]); break;
            case SLOSH_MODEL_ELASTIC_NEO_HOOKEAN: t = orc::neo_hookean<double, 3>(f, model[0], model[1]); break;
            case SLOSH_MODEL_SAND_LINEAR:
                orc::drucker_prager<double, 3>(model, model + 3, f);
                t = orc::fixed_corotated<double, 3>(f, model[9], model[10]);
                break;
            case SLOSH_MODEL_SAND_NEO_HOOKEAN:
                orc::drucker_prager<double, 3>(model, model + 3, f);
                t = orc::neo_hookean<double, 3>(f, model[9], model[10]);
                break;
            case SLOSH_MODEL_FLUID_TAIT: t = orc::tait_fluid<double, 3>(f, model[1], model[2]); break;
            default: return SLOSH_E_INVALID;
        }
        for (int i = 0; i < 9; ++i) {
            tau[i] = t.m[i / 3][i % 3];
            F[i] = f.m[i / 3][i % 3];
        }
        return SLOSH_OK;
    }
    return SLOSH_E_INVALID;
}

}  // extern "C"
