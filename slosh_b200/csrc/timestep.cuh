// Timestep bound: the largest dt the particles allow, for adaptive
// substepping.  Replaces WgTimestepBounds (src/solver/timestep_bound.rs:35-101)
// and its shader estimate_timestep_bound
// (shaders/slosh/solver/timestep_bound.slang:37-91).
//
// Per enabled particle: the model's sound-speed bound
// (ElasticitySoundSpeedTimestepBound, shaders/slosh/models/utils.slang:119-136,
// with the bulk and shear moduli of models/utils.slang:22-28) and the
// velocity bound h / |v|; the smaller one is quantised to whole picoseconds,
// floor(dt * 1e12) as a saturating u32, and the minimum over particles is
// taken with an atomic.  Every operation is explicitly rounded (no FMA
// contraction) in the order the shaders write it, so the result can be
// compared bit for bit with the oracle.  The Tait fluid (not in the
// reference, whose default model returns 0 for unknown tags) uses its own
// sound speed c^2 = K J^-gamma / rho with the same CFL factor 0.5.
#pragma once

#include "scene.cuh"

namespace slosh {

constexpr float TIMESTEP_FLOAT_TO_INT = 1.0e12f;  // GpuTimestepBounds::FLOAT_TO_INT
constexpr float TIMESTEP_FLUID_CFL = 0.5f;

// (alpha h) / max(|v|, sound speed) (models/utils.slang:119-136).
__device__ __forceinline__ float sound_speed_bound(float alpha, float bulk, float shear, float density0, float det_f,
                                                   float vlen, float h) {
    const float rho = __fdiv_rn(density0, fmaxf(det_f, 1.0e-6f));
    const float stiff = __fadd_rn(bulk, __fdiv_rn(__fmul_rn(shear, 4.0f), 3.0f));
    const float c = __fsqrt_rn(__fdiv_rn(stiff, rho));
    return __fdiv_rn(__fmul_rn(alpha, h), fmaxf(vlen, c));
}

// ElasticModel::timestep_bound with lambda, mu, cfl (bulk = lambda + 2 mu / 3,
// shear = mu; elastic hardening 1).
__device__ __forceinline__ float elastic_bound(const float *p, float density0, float det_f, float vlen, float h) {
    const float bulk = __fadd_rn(p[0], __fdiv_rn(__fmul_rn(2.0f, p[1]), 3.0f));
    return sound_speed_bound(p[2], bulk, p[1], density0, det_f, vlen, h);
}

// floor(secs * 1e12) as u32, saturating (GpuTimestepBounds::secs_to_int).
__device__ __forceinline__ uint32_t secs_to_int(float secs) {
    const float x = floorf(__fmul_rn(secs, TIMESTEP_FLOAT_TO_INT));
    if (!(x > 0.0f)) return 0u;
    return x >= 4294967296.0f ? 0xffffffffu : (uint32_t)x;
}

template <int D> __device__ __forceinline__ float det_rn(const float (&a)[D][D]) {
    if constexpr (D == 3) {
        const float c0 = __fsub_rn(__fmul_rn(a[1][1], a[2][2]), __fmul_rn(a[1][2], a[2][1]));
        const float c1 = __fsub_rn(__fmul_rn(a[1][0], a[2][2]), __fmul_rn(a[1][2], a[2][0]));
        const float c2 = __fsub_rn(__fmul_rn(a[1][0], a[2][1]), __fmul_rn(a[1][1], a[2][0]));
        return __fadd_rn(__fsub_rn(__fmul_rn(a[0][0], c0), __fmul_rn(a[0][1], c1)), __fmul_rn(a[0][2], c2));
    } else {
        return __fsub_rn(__fmul_rn(a[0][0], a[1][1]), __fmul_rn(a[0][1], a[1][0]));
    }
}

// One thread per stored particle; `out` holds the running minimum (reset to
// 0xffffffff by the caller).  In batches (B) only particles of `scene`, with
// that scene's cell width.
template <int D, bool B = false> __global__ void k_timestep_bound(DevScene s, uint32_t scene, uint32_t *out) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t n = n_particles<B>(s);
    const size_t ps = s.n;
    uint32_t best = 0xffffffffu;
    float h = s.h;
    if constexpr (B) h = s.scenes[scene].h;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint4 fo = s.fo[i];
        const uint32_t fl = fo.x;
        if (!(fl & FLAG_ENABLED)) continue;
        if constexpr (B)
            if (scene_of(fl) != scene) continue;
        const float4 pm = s.pm[i], vv = s.vv[i];
        const float density0 = __fdiv_rn(pm.w, __uint_as_float(fo.z));
        float F[D][D];
        {
            float4 fv[MQ<D>::Q];
#pragma unroll
            for (int q = 0; q < MQ<D>::Q; ++q) fv[q] = s.fq[q * ps + i];
            mat_from<D>(fv, __uint_as_float(fo.w), F);
        }
        const float det_f = det_rn<D>(F);
        const float vel[3] = {vv.x, vv.y, vv.z};
        float v2 = 0.0f;
#pragma unroll
        for (int k = 0; k < D; ++k) v2 = __fadd_rn(v2, __fmul_rn(vel[k], vel[k]));
        const float vlen = __fsqrt_rn(v2);
        const Material &m = s.materials[fl & FLAG_MAT_MASK];
        float dt;
        switch (m.tag) {
            case SLOSH_MODEL_ELASTIC_LINEAR:
            case SLOSH_MODEL_ELASTIC_NEO_HOOKEAN:
                dt = elastic_bound(m.p, density0, det_f, vlen, h);
                break;
            case SLOSH_MODEL_SAND_LINEAR:
            case SLOSH_MODEL_SAND_NEO_HOOKEAN:
                dt = elastic_bound(m.p + 9, density0, det_f, vlen, h);
                break;
            case SLOSH_MODEL_FLUID_TAIT: {
                const float J = F[0][0];
                const float rho = __fdiv_rn(density0, fmaxf(J, 1.0e-6f));
                const float c = __fsqrt_rn(__fdiv_rn(__fmul_rn(m.p[1], powf(fmaxf(J, 1.0e-6f), -m.p[2])), rho));
                dt = __fdiv_rn(__fmul_rn(TIMESTEP_FLUID_CFL, h), fmaxf(vlen, c));
                break;
            }
            default:
                dt = 0.0f;
                break;
        }
        dt = fminf(dt, __fdiv_rn(h, vlen));
        best = min(best, secs_to_int(dt));
    }
    // warp minimum, one atomic per warp
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) best = min(best, __shfl_xor_sync(FULL_MASK, best, off));
    if ((threadIdx.x & 31u) == 0 && best != 0xffffffffu) atomicMin(out, best);
}

}  // namespace slosh
