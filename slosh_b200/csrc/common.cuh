// Device-side constants and helpers shared by the slosh_b200 kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/slosh_b200.h"

namespace slosh {

constexpr uint32_t NONE = 0xffffffffu;
// Flag of a block-map value (a block rank): the block holds no particles
// (a neighbour-only block), so P2G wrote no tile for it.
constexpr uint32_t RANK_EXTRA = 0x80000000u;
__host__ __device__ __forceinline__ uint32_t rank_of(uint32_t v) { return v == NONE ? NONE : (v & ~RANK_EXTRA); }
constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr uint32_t MAX_BODIES = 16;       // collide() unrolls 16 shapes (collide.slang:362-363)
constexpr uint32_t MAX_MATERIALS = 4096;  // distinct particle models per context
constexpr uint32_t MAT_HASH = 8192;       // material hash slots (power of two)
constexpr uint32_t HIST_BINS = 65536;     // top-16-bit bins of the packed block key
constexpr uint32_t HIST_COARSE = 64;      // sums of 1024 consecutive bins (key >> 26)

// Device error bits (accumulated; read by slosh_sync).
constexpr uint32_t ERR_HASH_OVERFLOW = 1u << 0;    // block hash map full
constexpr uint32_t ERR_BLOCK_OVERFLOW = 1u << 1;   // more active blocks than capacity
constexpr uint32_t ERR_MATERIALS = 1u << 2;        // too many distinct materials
constexpr uint32_t ERR_MATERIAL_HASH = 1u << 3;    // two materials share a 32-bit hash
constexpr uint32_t ERR_KEY_RANGE = 1u << 4;        // a block coordinate outside the packed-key range
constexpr uint32_t ERR_BLOCK_PARTICLES = 1u << 6;  // a block holds 2^26 particles or more
constexpr uint32_t ERR_SCENE_BLOCKS = 1u << 5;     // a batch scene has more blocks than the per-scene sort holds
constexpr uint32_t ERR_GRID_REUSE = 1u << 7;       // a kept grid's cell counts and its gathered cells disagree
constexpr uint32_t ERR_BARRIER = 1u << 8;          // a grid barrier of the fused batch substep gave up waiting

// Sparse grid geometry per dimension (shaders/slosh/grid/grid.slang:224-257).
template <int D> struct Geo;
template <> struct Geo<3> {
    static constexpr int BW = 4;         // cells per block edge
    static constexpr int NASSOC = 8;     // primary block + 7 (+1) neighbours
    static constexpr int NPB = 4;        // primary slab buckets (sort.slang:15-21)
    static constexpr int NEB = 6;        // extra slab buckets
    static constexpr int NB = 10;
    static constexpr int MIN_SHIFT = 2;  // stencil spills into the +1 block when a >= 2
    static constexpr int TW = 6;         // halo tile edge: block + 2
    static constexpr int TILE = 216;     // TW^3
    static constexpr int NST = 27;       // stencil size
};
template <> struct Geo<2> {
    static constexpr int BW = 8;
    static constexpr int NASSOC = 4;
    static constexpr int NPB = 8;
    static constexpr int NEB = 10;
    static constexpr int NB = 18;
    static constexpr int MIN_SHIFT = 6;
    static constexpr int TW = 10;
    static constexpr int TILE = 100;
    static constexpr int NST = 9;
};

// Packed block key (grid.slang:77-91): x,z get 11 bits and y 10 bits in 3D,
// 16 bits per axis in 2D.
template <int D> __host__ __device__ __forceinline__ uint32_t pack_key(const int *b) {
    if constexpr (D == 3) {
        return ((uint32_t)(b[0] + 0x3ff) & 0x7ffu) | (((uint32_t)(b[1] + 0x1ff) & 0x3ffu) << 11) |
               (((uint32_t)(b[2] + 0x3ff) & 0x7ffu) << 21);
    } else {
        return ((uint32_t)(b[0] + 0x7fff) & 0xffffu) | (((uint32_t)(b[1] + 0x7fff) & 0xffffu) << 16);
    }
}

template <int D> __host__ __device__ __forceinline__ void unpack_key(uint32_t k, int *b) {
    if constexpr (D == 3) {
        b[0] = (int)(k & 0x7ffu) - 0x3ff;
        b[1] = (int)((k >> 11) & 0x3ffu) - 0x1ff;
        b[2] = (int)((k >> 21) & 0x7ffu) - 0x3ff;
    } else {
        b[0] = (int)(k & 0xffffu) - 0x7fff;
        b[1] = (int)((k >> 16) & 0xffffu) - 0x7fff;
    }
}

// MurmurHash3 mixing step used by slosh's block hash map (grid.slang:93-100).
__host__ __device__ __forceinline__ uint32_t murmur_mix(uint32_t key) {
    key *= 0xcc9e2d51u;
    key = (key << 15) | (key >> 17);
    key *= 0x1b873593u;
    return key;
}

// Offsets of the blocks associated with a block, in slosh's order
// (grid.slang:362-382): index 0 is the block itself.
template <int D> __host__ __device__ __forceinline__ void assoc_offset(int s, int *o) {
    if constexpr (D == 3) {
        o[0] = (s >> 2) & 1;
        o[1] = (s >> 1) & 1;
        o[2] = s & 1;
    } else {
        o[0] = (s >> 1) & 1;
        o[1] = s & 1;
    }
}

// Base cell of a position: round(x/h) - 1 with round-half-to-even (WGSL
// round), its block and its index inside the block
// (grid.slang:346-354; particle.slang:79-87).
template <int D> struct CellLoc {
    int block[D];
    int local[D];
};

// x / h, correctly rounded.  When h is a power of two its reciprocal is
// exact and x * (1/h) is the same correctly rounded quotient, so the IEEE
// division is replaced by a multiplication without changing any bit.
__device__ __forceinline__ float div_h(float x, float h, float inv_h, uint32_t h_pow2) {
    return h_pow2 ? x * inv_h : __fdiv_rn(x, h);
}

// Base cell round(x / h) - 1, its block floor(cell / BW) and its place in
// the block.  One round-to-nearest-even conversion, then integer shifts:
// the same values as rintf / floorf in float for every |x / h| < 2^24.
template <int D>
__device__ __forceinline__ CellLoc<D> locate(const float *x, float h, float inv_h, uint32_t h_pow2) {
    constexpr int SHIFT = Geo<D>::BW == 4 ? 2 : 3;
    static_assert(Geo<D>::BW == (1 << SHIFT), "block width is 4 or 8");
    CellLoc<D> c;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int cell = __float2int_rn(div_h(x[k], h, inv_h, h_pow2)) - 1;
        c.block[k] = cell >> SHIFT;  // arithmetic shift: floor division
        c.local[k] = cell & (Geo<D>::BW - 1);
    }
    return c;
}

// Quadratic B-spline weights of the 3 stencil nodes for fractional offset x
// in [0.5, 1.5) (kernel.slang:62-68).
__device__ __forceinline__ void bspline_weights(float x, float *w) {
    float a = 1.5f - x, b = x - 1.0f, c = x - 0.5f;
    w[0] = 0.5f * a * a;
    w[1] = 0.75f - b * b;
    w[2] = 0.5f * c * c;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Pairs for sm_100's f32x2 arithmetic (__ffma2_rn and friends): one
// instruction computes two FP32 lanes, each rounded as its scalar form.
__device__ __forceinline__ float2 pair(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 lo_pair(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi_pair(const float4 &v) { return make_float2(v.z, v.w); }

// Asynchronous global -> shared copies (cp.async), used to stage the next
// particle's inputs while the current one is computed.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Named CTA barriers (ids 1-15; 0 is __syncthreads) over n threads, a
// multiple of 32: `arrive` signals without waiting, `sync` waits for n.
// Both order the shared-memory accesses made before them for the threads
// that complete the barrier.
__device__ __forceinline__ void named_bar_sync(uint32_t id, uint32_t n) {
    asm volatile("barrier.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ void named_bar_arrive(uint32_t id, uint32_t n) {
    asm volatile("barrier.arrive %0, %1;\n" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// D x D matrices of the particle state (C, F) are stored as MQ<D> float4
// planes holding the row-major elements 0-3 (and 4-7); in 3D element 8 rides
// in the spare fourth lane of another per-particle vector (C22 with the
// velocity, F22 with the flags), so every particle access is a 16-byte one.
template <int D> struct MQ;
template <> struct MQ<3> {
    static constexpr int Q = 2;
};
template <> struct MQ<2> {
    static constexpr int Q = 1;
};

template <int D>
__device__ __forceinline__ void mat_from(const float4 *q, float e8, float (&M)[D][D]) {
    if constexpr (D == 3) {
        M[0][0] = q[0].x, M[0][1] = q[0].y, M[0][2] = q[0].z, M[1][0] = q[0].w;
        M[1][1] = q[1].x, M[1][2] = q[1].y, M[2][0] = q[1].z, M[2][1] = q[1].w;
        M[2][2] = e8;
    } else {
        M[0][0] = q[0].x, M[0][1] = q[0].y, M[1][0] = q[0].z, M[1][1] = q[0].w;
    }
}

// Inverse of mat_from: fills the MQ<D> vectors and returns element 8 (0 in 2D).
template <int D> __device__ __forceinline__ float mat_split(const float (&M)[D][D], float4 *q) {
    if constexpr (D == 3) {
        q[0] = make_float4(M[0][0], M[0][1], M[0][2], M[1][0]);
        q[1] = make_float4(M[1][1], M[1][2], M[2][0], M[2][1]);
        return M[2][2];
    } else {
        q[0] = make_float4(M[0][0], M[0][1], M[1][0], M[1][1]);
        return 0.f;
    }
}

// Material record: GpuParticleModel without the per-particle plastic state.
struct Material {
    uint32_t tag;
    float p[12];
};

// Flags word of a particle: material id, enabled, fixed, and (multi-scene
// batches) the scene slot in the top 14 bits.
constexpr uint32_t FLAG_MAT_MASK = 0xffffu;
constexpr uint32_t FLAG_ENABLED = 1u << 16;
constexpr uint32_t FLAG_FIXED = 1u << 17;
constexpr uint32_t FLAG_SCENE_SHIFT = 18;
constexpr uint32_t MAX_SCENES = 1u << 14;
__host__ __device__ __forceinline__ uint32_t scene_of(uint32_t flags) { return flags >> FLAG_SCENE_SHIFT; }

// Per-scene parameters of a multi-scene batch (the single-scene context
// passes the same values as kernel arguments).
struct SceneRec {
    float h, inv_h, dt;
    float gravity[3];
    uint32_t h_pow2;
    uint32_t body_first, n_bodies;  // the scene's colliders in the body table
    uint32_t live;                  // 0: the slot's particles are dropped at the next substep
    uint32_t g2p_class;             // the G2P launch its blocks go to (G2P_CLASS_*)
};

// A batch's blocks are handed to one G2P launch per class of scene, each
// compiled for one particle model (a scene of one linear-elastic, sand or
// fluid model), or for every model (any other scene).
constexpr uint32_t G2P_CLASSES = 4;
constexpr uint32_t G2P_CLASS_GENERIC = 3;
__host__ __device__ __forceinline__ uint32_t g2p_class_of_tags(uint32_t tags) {
    if (tags == (1u << SLOSH_MODEL_SAND_LINEAR)) return 0u;
    if (tags == (1u << SLOSH_MODEL_ELASTIC_LINEAR)) return 1u;
    if (tags == (1u << SLOSH_MODEL_FLUID_TAIT)) return 2u;
    return G2P_CLASS_GENERIC;
}

// Collider body on the device (slosh_body in device form).
struct DevBody {
    uint32_t shape_type;
    float sa[4];
    float sb[4];
    float rot[4];
    float tra[3];
    float scale;
    float linvel[3];
    float angvel[3];
    float inv_mass[3];
    float local_com[3];
    uint32_t bc_type;
    float friction;
    uint32_t scene;         // owning scene slot (multi-scene batches)
    uint32_t coupling;      // SLOSH_COUPLING_*
    float inv_inertia[9];   // body-frame inverse inertia, row-major (2D: [0])
};

// Two-way coupling impulses: 64-bit fixed point, 2^40 units per N s, six
// sums per body (linear xyz, angular xyz; 2D: linear xy, angular in [3]).
constexpr double IMPULSE_UNITS = 1099511627776.0;  // 2^40

// Rotation matrix of the unit quaternion q = (i, j, k, w).
__host__ __device__ inline void quat_matrix(const float *q, float (&R)[3][3]) {
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    R[0][0] = 1.f - 2.f * (y * y + z * z);
    R[0][1] = 2.f * (x * y - z * w);
    R[0][2] = 2.f * (x * z + y * w);
    R[1][0] = 2.f * (x * y + z * w);
    R[1][1] = 1.f - 2.f * (x * x + z * z);
    R[1][2] = 2.f * (y * z - x * w);
    R[2][0] = 2.f * (x * z - y * w);
    R[2][1] = 2.f * (y * z + x * w);
    R[2][2] = 1.f - 2.f * (x * x + y * y);
}

// out = R M R^T (rot = true) or R^T M R (rot = false) for 3 x 3 M.
__host__ __device__ inline void rotate_tensor(const float (&R)[3][3], const float *M, float *out, bool rot) {
    float T[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float a = 0.f;
            for (int k = 0; k < 3; ++k) a += (rot ? R[i][k] : R[k][i]) * M[k * 3 + j];
            T[i][j] = a;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            float a = 0.f;
            for (int k = 0; k < 3; ++k) a += T[i][k] * (rot ? R[j][k] : R[k][j]);
            out[i * 3 + j] = a;
        }
}

// Per-substep device counters.
struct Counters {
    uint32_t n_primary;      // primary blocks appended by the touch pass
    uint32_t n_extra;        // neighbour-only blocks appended by the neighbour pass
    uint32_t n_blocks;       // active blocks after ranking (min(total, capacity))
    uint32_t n_sorted;       // debug: sorted entries with extras
    uint32_t n_svd_fp64;     // particles whose SVD fell back to FP64 (cumulative)
    uint32_t last_n_blocks;  // n_blocks of the last completed substep
    uint32_t last_n_primary; // n_primary of the last completed substep
    uint32_t p2g_next;       // next block for a P2G warp (reset by k_block_setup or k_reuse_perm)
    uint32_t g2p_next;       // next block for a G2P CTA (reset by k_block_setup or k_reuse_perm)
    uint32_t rebuild[2];     // grid reuse: the substep of this parity runs the full grid build
                             // (set by the host, by G2P for the next substep, by k_grid_reuse)
    uint32_t reuse_done;     // CTAs of k_grid_reuse that finished (the last one decides)
    uint32_t n_rebuilds;     // substeps that ran the full grid build (cumulative)
    uint32_t n_reuses;       // substeps that kept the previous grid (cumulative)
    uint32_t reuse_per_cta;  // blocks each CTA of k_grid_reuse counted (a contiguous range)
    uint32_t n_touched;      // touched cells listed by k_reuse_perm for k_reuse_cells
    uint32_t bar_count;      // fused batch substep: CTAs arrived at the current grid barrier
    uint32_t bar_gen;        // fused batch substep: grid barriers completed (wraps)
    uint32_t pad[2];
};

// The CTA index and CTA count a kernel body runs with: its own launch's
// (blockIdx.x, gridDim.x), or the whole grid of the fused batch substep.
struct Cta {
    uint32_t id, n;
};
__device__ __forceinline__ Cta launch_cta() { return Cta{blockIdx.x, gridDim.x}; }

// Programmatic dependent launch.  A kernel of the substep graph that was
// launched with cudaLaunchAttributeProgrammaticStreamSerialization may be
// scheduled while the kernel before it in the stream still runs; it waits
// here, before its first memory access, until that kernel has completed and
// its writes are visible, then lets its own successor be scheduled.  Every
// stand-alone kernel of the substep enters this way, also those that read
// nothing of their predecessor's output, so that a kernel's completion
// implies the completion of all kernels before it.  Launched without the
// attribute, both instructions return at once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace slosh
