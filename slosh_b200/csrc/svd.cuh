// 3x3 and 2x2 singular value decompositions for the constitutive models.
//
// slosh takes its SVD from the third-party stensor crate (svd3/svd2, called
// at shaders/slosh/models/linear_elasticity.slang:70 and
// shaders/slosh/models/drucker_prager.slang:181).  This file is an own
// implementation of the method of McAdams, Selle, Tamstorf, Teran and
// Sifakis, "Computing the Singular Value Decomposition of 3x3 matrices with
// minimal branching and elementary floating point operations" (2011):
//   1. symmetric eigen-decomposition of A = F^T F by cyclic Jacobi rotations
//      (exact rotation angles here, where the paper uses approximate ones),
//   2. eigenvalues sorted in decreasing order, V kept a proper rotation,
//   3. Givens QR of B = F V, so that F = U R V^T with U a proper rotation
//      (FP32 with a converged Jacobi, singular values within a factor 2 and
//      F not inverted: the columns of B normalised instead, which the
//      converged Jacobi leaves orthogonal to its residual).
// The singular values are the diagonal of R: s0 >= s1 >= |s2|, the sign of
// det F carried by s2.  The QR step keeps the factorisation backward stable
// when singular values coincide or vanish.
//
// Precision policy: the FP32 result is recomputed in FP64 when it is not
// trustworthy:
//  - F nearly singular or inverted (s2 <= 1e-3 s0);
//  - R keeps off-diagonal mass above 1e-5 s0, which is how nearly repeated
//    singular values show up (the eigenvectors of F^T F inside a
//    near-degenerate subspace are poorly determined in FP32);
//  - all singular values within 1e-5 s0 of each other while F is not near
//    a rotation (|s0 - 1| > 1e-5).  Drucker-Prager tests the deviatoric
//    log strain for exact zero (drucker_prager.slang:165-200), a
//    discontinuity at isotropic stretch: FP32 singular values that come out
//    equal where FP64 resolves a difference of a few ulps would project a
//    compressed particle to the yield surface's tip (a jump of |s - 1| in
//    F).  Near a rotation that jump is below FP32 resolution, so the common
//    F ~ I case stays in FP32.
#pragma once

#include <cuda_runtime.h>

namespace slosh {

// Per-precision helpers.  The Jacobi angle only steers convergence: any t
// yields an orthogonal rotation (c = 1/sqrt(1+t^2), s = t c), so the FP32
// path takes approximate reciprocals and square roots there.  EPS is the relative
// off-diagonal size at which a sweep stops (near the rounding floor of A).
template <typename T> struct SvdT;
template <> struct SvdT<float> {
    static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
    // only used on theta^2 + 1 >= 1, where x rsqrt(x) is finite
    static __device__ __forceinline__ float sqrt_(float x) { return x * rsqrtf(x); }
    static __device__ __forceinline__ float rcp_(float x) { return __fdividef(1.0f, x); }
    static constexpr int SWEEPS = 5;
    static constexpr float TINY = 1e-30f;
    static constexpr float EPS = 1e-7f;
};
template <> struct SvdT<double> {
    static __device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double rcp_(double x) { return 1.0 / x; }
    static constexpr int SWEEPS = 8;
    static constexpr double TINY = 1e-300;
    static constexpr double EPS = 1e-16;
};

template <typename T> struct Svd3 {
    T U[3][3];
    T V[3][3];
    T s[3];
    T offdiag;  // |R01| + |R02| + |R12| of the QR step
};

// One Jacobi rotation of the symmetric matrix A (upper triangle in a[3][3])
// in the (p, q) plane, accumulated into V.
template <typename T, int p, int q>
__device__ __forceinline__ void jacobi_rotate(T (&a)[3][3], T (&V)[3][3]) {
    constexpr int r = 3 - p - q;
    const T apq = a[p][q];
    if (!(fabs(apq) > SvdT<T>::TINY)) return;
    const T theta = (a[q][q] - a[p][p]) * SvdT<T>::rcp_(T(2) * apq);
    // |theta| + sqrt(theta^2 + 1) without overflow for huge theta
    const T at = fabs(theta);
    const T den = at > T(1e15) ? T(2) * at : at + SvdT<T>::sqrt_(theta * theta + T(1));
    const T t = copysign(SvdT<T>::rcp_(den), theta);
    const T c = SvdT<T>::rsqrt_(t * t + T(1));
    const T s = t * c;
    a[p][p] = a[p][p] - t * apq;
    a[q][q] = a[q][q] + t * apq;
    a[p][q] = T(0);
    a[q][p] = T(0);
    const T arp = a[r][p], arq = a[r][q];
    a[r][p] = a[p][r] = c * arp - s * arq;
    a[r][q] = a[q][r] = s * arp + c * arq;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T vp = V[i][p], vq = V[i][q];
        V[i][p] = c * vp - s * vq;
        V[i][q] = s * vp + c * vq;
    }
}

template <typename T>
__device__ __forceinline__ void swap_cols(T (&V)[3][3], T &la, T &lb, int ca, int cb) {
    const T tl = la;
    la = lb;
    lb = tl;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T t = V[i][ca];
        V[i][ca] = -V[i][cb];  // one sign flip keeps det V = +1
        V[i][cb] = t;
    }
}

// Givens rotation zeroing `b` against `a`: [c s; -s c] [a; b] = [r; 0].
template <typename T> __device__ __forceinline__ void givens(T a, T b, T &c, T &s) {
    const T n2 = a * a + b * b;
    if (n2 > SvdT<T>::TINY) {
        const T inv = SvdT<T>::rsqrt_(n2);
        c = a * inv;
        s = b * inv;
    } else {
        c = T(1);
        s = T(0);
    }
}

template <typename T> __device__ void svd3_impl(const T (&F)[3][3], Svd3<T> &out) {
    T a[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = i; j < 3; ++j) {
            T acc = F[0][i] * F[0][j];
            acc += F[1][i] * F[1][j];
            acc += F[2][i] * F[2][j];
            a[i][j] = acc;
            a[j][i] = acc;
        }
    T V[3][3] = {{T(1), T(0), T(0)}, {T(0), T(1), T(0)}, {T(0), T(0), T(1)}};
    bool converged = false;
    T off = T(0);
    for (int sweep = 0; sweep < SvdT<T>::SWEEPS; ++sweep) {
        jacobi_rotate<T, 0, 1>(a, V);
        jacobi_rotate<T, 0, 2>(a, V);
        jacobi_rotate<T, 1, 2>(a, V);
        off = fabs(a[0][1]) + fabs(a[0][2]) + fabs(a[1][2]);
        const T dia = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]);
        if (!(off > dia * SvdT<T>::EPS)) {
            converged = true;
            break;
        }
    }
    T l0 = a[0][0], l1 = a[1][1], l2 = a[2][2];
    if (l0 < l1) swap_cols<T>(V, l0, l1, 0, 1);
    if (l0 < l2) swap_cols<T>(V, l0, l2, 0, 2);
    if (l1 < l2) swap_cols<T>(V, l1, l2, 1, 2);
    // B = F V
    T B[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) B[i][j] = F[i][0] * V[0][j] + F[i][1] * V[1][j] + F[i][2] * V[2][j];
    if constexpr (sizeof(T) == 4) {
        // FP32, the common case: a converged Jacobi leaves the columns of
        // B = F V orthogonal up to its residual (B^T B = V^T F^T F V), so U is
        // B with normalised columns.  That orthogonality error is at most
        // the residual over s_i s_j, so this path is taken only when the
        // singular values stay within a factor 2 of each other and F is not
        // inverted (det B = det F); the Givens QR below keeps the other cases
        // backward stable.
        T n2[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) n2[j] = B[0][j] * B[0][j] + B[1][j] * B[1][j] + B[2][j] * B[2][j];
        const T detb = B[0][0] * (B[1][1] * B[2][2] - B[1][2] * B[2][1]) - B[0][1] * (B[1][0] * B[2][2] - B[1][2] * B[2][0]) +
                       B[0][2] * (B[1][0] * B[2][1] - B[1][1] * B[2][0]);
        if (converged && n2[2] > T(0.25) * n2[0] && detb > T(0)) {
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const T inv = rsqrtf(n2[j]);
                out.s[j] = n2[j] * inv;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    out.U[i][j] = B[i][j] * inv;
                    out.V[i][j] = V[i][j];
                }
            }
            out.offdiag = off * rsqrtf(n2[0]);  // the residual, in units of s0 like R's off-diagonal
            return;
        }
    }
    // QR by Givens: rows (0,1) col 0, rows (0,2) col 0, rows (1,2) col 1.
    T U[3][3] = {{T(1), T(0), T(0)}, {T(0), T(1), T(0)}, {T(0), T(0), T(1)}};
    T c, s;
    givens<T>(B[0][0], B[1][0], c, s);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const T b0 = B[0][j], b1 = B[1][j];
        B[0][j] = c * b0 + s * b1;
        B[1][j] = -s * b0 + c * b1;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T u0 = U[i][0], u1 = U[i][1];
        U[i][0] = c * u0 + s * u1;
        U[i][1] = -s * u0 + c * u1;
    }
    givens<T>(B[0][0], B[2][0], c, s);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const T b0 = B[0][j], b2 = B[2][j];
        B[0][j] = c * b0 + s * b2;
        B[2][j] = -s * b0 + c * b2;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T u0 = U[i][0], u2 = U[i][2];
        U[i][0] = c * u0 + s * u2;
        U[i][2] = -s * u0 + c * u2;
    }
    givens<T>(B[1][1], B[2][1], c, s);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const T b1 = B[1][j], b2 = B[2][j];
        B[1][j] = c * b1 + s * b2;
        B[2][j] = -s * b1 + c * b2;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T u1 = U[i][1], u2 = U[i][2];
        U[i][1] = c * u1 + s * u2;
        U[i][2] = -s * u1 + c * u2;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            out.U[i][j] = U[i][j];
            out.V[i][j] = V[i][j];
        }
    out.s[0] = B[0][0];
    out.s[1] = B[1][1];
    out.s[2] = B[2][2];
    out.offdiag = fabs(B[0][1]) + fabs(B[0][2]) + fabs(B[1][2]);
}

// FP32 SVD with the FP64 fallback described above.  Increments *fp64_count
// when the fallback runs (diagnostics).
__device__ __forceinline__ void svd3(const float (&F)[3][3], Svd3<float> &out, unsigned *fp64_count) {
    svd3_impl<float>(F, out);
    const float s0 = fabsf(out.s[0]);
    const bool isotropic = out.s[0] - out.s[2] <= 1e-5f * s0 && fabsf(s0 - 1.0f) > 1e-5f;
    const bool degenerate = !(out.s[2] > 1e-3f * s0) || !(out.offdiag <= 1e-5f * s0) || isotropic;
    if (degenerate && s0 > 0.0f) {
        double Fd[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) Fd[i][j] = (double)F[i][j];
        Svd3<double> d;
        svd3_impl<double>(Fd, d);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            out.s[i] = (float)d.s[i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                out.U[i][j] = (float)d.U[i][j];
                out.V[i][j] = (float)d.V[i][j];
            }
        }
        out.offdiag = (float)d.offdiag;
        if (fp64_count) atomicAdd(fp64_count, 1u);
    }
}

// 2x2 SVD in closed form: F = R(phi) diag(sx, sy) R(theta), sx >= |sy|,
// sy < 0 when det F < 0 (Blinn, "Consider the lowly 2x2 matrix", 1996).
template <typename T> struct Svd2 {
    T U[2][2];
    T V[2][2];
    T s[2];
};

template <typename T> __device__ void svd2_impl(const T (&F)[2][2], Svd2<T> &out) {
    const T E = (F[0][0] + F[1][1]) * T(0.5);
    const T Fm = (F[0][0] - F[1][1]) * T(0.5);
    const T G = (F[1][0] + F[0][1]) * T(0.5);
    const T H = (F[1][0] - F[0][1]) * T(0.5);
    const T Q = sqrt(E * E + H * H);
    const T R = sqrt(Fm * Fm + G * G);
    const T sx = Q + R, sy = Q - R;
    const T a1 = atan2(G, Fm), a2 = atan2(H, E);
    const T theta = (a2 - a1) * T(0.5), phi = (a2 + a1) * T(0.5);
    T ct, st, cp, sp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    // F = R(phi) diag(sx, sy) R(theta): U = R(phi), V = R(theta)^T = R(-theta).
    out.U[0][0] = cp;
    out.U[0][1] = -sp;
    out.U[1][0] = sp;
    out.U[1][1] = cp;
    out.V[0][0] = ct;
    out.V[0][1] = st;
    out.V[1][0] = -st;
    out.V[1][1] = ct;
    out.s[0] = sx;
    out.s[1] = sy;
}

__device__ __forceinline__ void svd2(const float (&F)[2][2], Svd2<float> &out, unsigned *fp64_count) {
    svd2_impl<float>(F, out);
    const bool isotropic = out.s[0] - out.s[1] <= 1e-5f * out.s[0] && fabsf(out.s[0] - 1.0f) > 1e-5f;
    if ((!(out.s[1] > 1e-3f * out.s[0]) || isotropic) && out.s[0] > 0.0f) {
        double Fd[2][2] = {{(double)F[0][0], (double)F[0][1]}, {(double)F[1][0], (double)F[1][1]}};
        Svd2<double> d;
        svd2_impl<double>(Fd, d);
        for (int i = 0; i < 2; ++i) {
            out.s[i] = (float)d.s[i];
            for (int j = 0; j < 2; ++j) {
                out.U[i][j] = (float)d.U[i][j];
                out.V[i][j] = (float)d.V[i][j];
            }
        }
        if (fp64_count) atomicAdd(fp64_count, 1u);
    }
}

}  // namespace slosh
