// Constitutive models of the particle update, in math convention
// (M[i][j] = row i, column j; slosh's Slang code stores the transposes).
//
//  - fixed-corotated: LinearElasticModel::kirchoff_stress
//    (shaders/slosh/models/linear_elasticity.slang:69-82):
//      tau = 2 mu (F - R) F^T + lambda (J - 1) J I
//  - Neo-Hookean: NeoHookeanModel::kirchoff_stress
//    (shaders/slosh/models/neo_hookean_elasticity.slang:16-27):
//      tau = mu F F^T + (lambda ln J - mu) I,  J = max(det F, 1e-10)
//  - Drucker-Prager return mapping: DruckerPragerPlasticity::project
//    (shaders/slosh/models/drucker_prager.slang:46-50, 144-200), followed by
//    the elastic stress of the projected F.  The elastic stress reuses the
//    SVD of the projection (U, projected singular values, V), the
//    factorisation slosh's kirchoff_stress_from_svd takes, instead of a
//    second SVD of the recomposed F.
//  - Tait weakly compressible fluid (extension behind ModelFlags::FLUID):
//      tau = -J p I, p = (K / gamma) (J^-gamma - 1), J = F00.
#pragma once

#include "common.cuh"
#include "svd.cuh"

namespace slosh {

template <int D> struct SvdD;
template <> struct SvdD<3> {
    float U[3][3], V[3][3], s[3];
    __device__ __forceinline__ void compute(const float (&F)[3][3], unsigned *fp64) {
        Svd3<float> r;
        svd3(F, r, fp64);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            s[i] = r.s[i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                U[i][j] = r.U[i][j];
                V[i][j] = r.V[i][j];
            }
        }
    }
};
template <> struct SvdD<2> {
    float U[2][2], V[2][2], s[2];
    __device__ __forceinline__ void compute(const float (&F)[2][2], unsigned *fp64) {
        Svd2<float> r;
        svd2(F, r, fp64);
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            s[i] = r.s[i];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                U[i][j] = r.U[i][j];
                V[i][j] = r.V[i][j];
            }
        }
    }
};

template <int D> __device__ __forceinline__ float det(const float (&F)[D][D]) {
    if constexpr (D == 3) {
        return F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
               F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
    } else {
        return F[0][0] * F[1][1] - F[0][1] * F[1][0];
    }
}

// U diag(s) V^T
template <int D>
__device__ __forceinline__ void recompose(const float (&U)[D][D], const float *s, const float (&V)[D][D],
                                          float (&out)[D][D]) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) acc += (U[i][k] * s[k]) * V[j][k];
            out[i][j] = acc;
        }
}

// With F = U S V^T and R = U V^T, (F - R) F^T = U (S - I) S U^T, so the
// stress needs U and the singular values only: a symmetric product.
template <int D>
__device__ __forceinline__ void fixed_corotated(const SvdD<D> &sv, float lambda, float mu, float (&tau)[D][D]) {
    float j = sv.s[0] * sv.s[1];
    if constexpr (D == 3) j = j * sv.s[2];
    float d[D];
#pragma unroll
    for (int k = 0; k < D; ++k) d[k] = 2.f * mu * (sv.s[k] - 1.f) * sv.s[k];
    const float diag = lambda * (j - 1.f) * j;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = i; k < D; ++k) {
            float acc = 0.f;
#pragma unroll
            for (int l = 0; l < D; ++l) acc += (sv.U[i][l] * d[l]) * sv.U[k][l];
            tau[i][k] = acc;
            tau[k][i] = acc;
        }
#pragma unroll
    for (int i = 0; i < D; ++i) tau[i][i] += diag;
}

template <int D>
__device__ __forceinline__ void neo_hookean(const float (&F)[D][D], float lambda, float mu, float (&tau)[D][D]) {
    const float j = fmaxf(det<D>(F), 1.0e-10f);
    const float diag = lambda * logf(j) - mu;
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
        for (int k = 0; k < D; ++k) {
            float acc = 0.f;
#pragma unroll
            for (int l = 0; l < D; ++l) acc += F[i][l] * F[k][l];
            tau[i][k] = mu * acc;
        }
#pragma unroll
    for (int i = 0; i < D; ++i) tau[i][i] += diag;
}

// Drucker-Prager projection of the singular values.  `st` = (plastic det,
// hardening q, log_vol_gain); `p` = (h0, h1, h2, h3, lambda, mu).  On a
// valid projection updates st, sv.s and F (= U diag(s') V^T).
template <int D>
__device__ __forceinline__ void drucker_prager(float *st, const float *p, SvdD<D> &sv, float (&F)[D][D]) {
    const float ha = p[0], hb = p[1], hc = p[2], hd = p[3], lambda = p[4], mu = p[5];
    const float q = st[1];
    // The friction angle and the cone slope only place the yield surface:
    // the hardware approximations (a few ulp) are used for them; the terms
    // that enter F and the plastic state keep the correctly rounded forms.
    const float angle = ha + (hb * q - hd) * __expf(-hc * q);
    const float s_angle = __sinf(angle);
    const float alpha = __fdividef(sqrtf(2.0f / 3.0f) * (2.0f * s_angle), 3.0f - s_angle);
    const float d = (float)D;
    float strain[D], ls[D], tr = 0.f;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        ls[i] = logf(sv.s[i]);
        strain[i] = ls[i] + st[2] / d;
    }
#pragma unroll
    for (int i = 0; i < D; ++i) tr += strain[i];
    float dev[D];
    bool dev_zero = true;
#pragma unroll
    for (int i = 0; i < D; ++i) {
        dev[i] = strain[i] - tr / d;
        dev_zero = dev_zero && (dev[i] == 0.f);
    }
    // ln of the projected singular values: log(new_det) = sum(hh) and
    // log(prev_det) = sum(ls), so no further log is needed.
    float ns[D], hh[D], dq;
    if (tr > 0.f || dev_zero) {
        float n2 = 0.f;
#pragma unroll
        for (int i = 0; i < D; ++i) n2 += strain[i] * strain[i];
#pragma unroll
        for (int i = 0; i < D; ++i) {
            ns[i] = 1.f;
            hh[i] = 0.f;
        }
        dq = sqrtf(n2);
    } else {
        float n2 = 0.f;
#pragma unroll
        for (int i = 0; i < D; ++i) n2 += dev[i] * dev[i];
        const float devn = sqrtf(n2);
        const float gamma = devn + __fdividef(d * lambda + 2.0f * mu, 2.0f * mu) * tr * alpha;
        if (gamma <= 0.f) return;
        const float g = __fdividef(gamma, devn);
#pragma unroll
        for (int i = 0; i < D; ++i) {
            hh[i] = strain[i] - dev[i] * g;
            ns[i] = expf(hh[i]);
        }
        dq = gamma;
    }
    float prev_det = sv.s[0] * sv.s[1], new_det = ns[0] * ns[1];
    float lprev = ls[0] + ls[1], lnew = hh[0] + hh[1];
    if constexpr (D == 3) {
        prev_det = prev_det * sv.s[2];
        new_det = new_det * ns[2];
        lprev += ls[2];
        lnew += hh[2];
    }
    st[0] = st[0] * prev_det / new_det;
    st[2] = st[2] + lprev - lnew;
    st[1] = q + dq;
#pragma unroll
    for (int i = 0; i < D; ++i) sv.s[i] = ns[i];
    recompose<D>(sv.U, ns, sv.V, F);
}

// DefaultParticleModel::update (shaders/slosh/models/default.slang:51-92)
// plus the Tait fluid.  `st` is the particle's plastic state (sand only).
// `tag` is the material's model tag (a constant when the kernel is
// instantiated for a scene of one model, which leaves the other models out).
template <int D>
__device__ __forceinline__ void model_update(const Material &mat, uint32_t tag, float (&F)[D][D], float *st,
                                             float (&tau)[D][D], unsigned *fp64) {
    switch (tag) {
        case SLOSH_MODEL_ELASTIC_LINEAR: {
            SvdD<D> sv;
            sv.compute(F, fp64);
            fixed_corotated<D>(sv, mat.p[0], mat.p[1], tau);
            break;
        }
        case SLOSH_MODEL_ELASTIC_NEO_HOOKEAN:
            neo_hookean<D>(F, mat.p[0], mat.p[1], tau);
            break;
        case SLOSH_MODEL_SAND_LINEAR: {
            SvdD<D> sv;
            sv.compute(F, fp64);
            if (mat.p[7] != 0.f) drucker_prager<D>(st, mat.p + 3, sv, F);
            fixed_corotated<D>(sv, mat.p[9], mat.p[10], tau);
            break;
        }
        case SLOSH_MODEL_SAND_NEO_HOOKEAN: {
            if (mat.p[7] != 0.f) {
                SvdD<D> sv;
                sv.compute(F, fp64);
                drucker_prager<D>(st, mat.p + 3, sv, F);
            }
            neo_hookean<D>(F, mat.p[9], mat.p[10], tau);
            break;
        }
        case SLOSH_MODEL_FLUID_TAIT: {
            const float J = F[0][0];
            const float pressure = (mat.p[1] / mat.p[2]) * (powf(J, -mat.p[2]) - 1.f);
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int k = 0; k < D; ++k) tau[i][k] = (i == k) ? -J * pressure : 0.f;
            break;
        }
        default:
#pragma unroll
            for (int i = 0; i < D; ++i)
#pragma unroll
                for (int k = 0; k < D; ++k) tau[i][k] = 0.f;
            break;
    }
}

}  // namespace slosh
