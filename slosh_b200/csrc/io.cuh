// Particle upload/download between slosh's record layout and the device
// structure of arrays, and the debug kernels that rebuild slosh's complete
// sorted-particle layout (primaries + extras).
#pragma once

#include "grid_build.cuh"

namespace slosh {

struct IoBuffers {
    const slosh_particle *in;  // staging, device
    slosh_particle *out;       // staging, device
    uint32_t *mat_hkeys;       // MAT_HASH material-key hashes
    uint32_t *mat_dense;       // MAT_HASH dense material ids
    uint32_t *n_mat;           // device counter
    uint32_t *scene_flags;     // bit0 damping, bit1 force, bit2 sand, bits 8-15 model tags
    float *r0;
    float *phase;
};

constexpr uint32_t SCENE_DAMPING = 1u, SCENE_FORCE = 2u, SCENE_SAND = 4u;
// bits SCENE_MODEL_SHIFT + tag: the model tags present (tags above 6 share bit 7)
constexpr uint32_t SCENE_MODEL_SHIFT = 8;

// Words of the material key: tag + 12 payload words, with the per-particle
// plastic state (payload words 0..2 of the sand models) zeroed.
__device__ __forceinline__ void material_key(const slosh_model &m, uint32_t *w) {
    w[0] = m.tag;
    const bool sand = m.tag == SLOSH_MODEL_SAND_LINEAR || m.tag == SLOSH_MODEL_SAND_NEO_HOOKEAN;
#pragma unroll
    for (int k = 0; k < 12; ++k) w[1 + k] = (sand && k < 3) ? 0u : __float_as_uint(m.data[k]);
}

__device__ __forceinline__ uint32_t material_hash(const uint32_t *w) {
    uint32_t h = 0x9747b28cu;
#pragma unroll
    for (int k = 0; k < 13; ++k) h = murmur_mix(h ^ w[k]) * 5u + 0xe6546b64u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    return h == NONE ? 0x7fffffffu : h;
}

// Pass 1 of the upload: distinct materials of `count` staged records into
// the material table.
__global__ void k_mat_insert(DevScene s, IoBuffers io, uint32_t count) {
    const uint32_t lane = lane_id();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < count; base += stride) {
        const uint32_t i = base + lane;
        const bool valid = i < count;
        const unsigned mask = __ballot_sync(FULL_MASK, valid);
        if (!valid) continue;
        uint32_t w[13];
        material_key(io.in[i].model, w);
        const uint32_t hsh = material_hash(w);
        const unsigned peers = __match_any_sync(mask, hsh);
        if ((int)lane != __ffs(peers) - 1) continue;
        uint32_t slot = hsh & (MAT_HASH - 1u);
        for (uint32_t k = 0; k < MAT_HASH; ++k) {
            const uint32_t old = atomicCAS(&io.mat_hkeys[slot], NONE, hsh);
            if (old == NONE) {
                const uint32_t dense = atomicAdd(io.n_mat, 1u);
                if (dense < MAX_MATERIALS) {
                    Material m;
                    m.tag = w[0];
                    for (int q = 0; q < 12; ++q) m.p[q] = __uint_as_float(w[1 + q]);
                    const_cast<Material *>(s.materials)[dense] = m;
                    io.mat_dense[slot] = dense;
                } else {
                    io.mat_dense[slot] = NONE;
                    atomicOr(s.err, ERR_MATERIALS);
                }
                break;
            }
            if (old == hsh) break;
            slot = (slot + 1u) & (MAT_HASH - 1u);
        }
    }
}

// Pass 2 of the upload: record i -> structure of arrays at storage index
// base + i, original id oid_base + i.  Multi-scene batches (B) tag the
// particle with its scene slot and keep no upload-order side arrays (forces
// are rejected on the host; radius and phase stay with the host).
template <int D, bool B = false>
__global__ void k_ingest(DevScene s, IoBuffers io, uint32_t base, uint32_t count, uint32_t scene,
                         uint32_t oid_base = 0u) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const size_t n = s.n;
    uint32_t sflags = 0;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < count; i0 += stride) {
        const uint32_t i = base + i0;
        const slosh_particle &p = io.in[i0];
        uint32_t w[13];
        material_key(p.model, w);
        const uint32_t hsh = material_hash(w);
        uint32_t slot = hsh & (MAT_HASH - 1u), dense = NONE;
        for (uint32_t k = 0; k < MAT_HASH; ++k) {
            const uint32_t kk = io.mat_hkeys[slot];
            if (kk == hsh) {
                dense = io.mat_dense[slot];
                break;
            }
            if (kk == NONE) break;
            slot = (slot + 1u) & (MAT_HASH - 1u);
        }
        if (dense == NONE || dense >= MAX_MATERIALS) {
            atomicOr(s.err, ERR_MATERIALS);
            dense = 0;
        } else {
            const Material &m = s.materials[dense];
            bool same = m.tag == w[0];
            for (int q = 0; q < 12; ++q) same = same && (__float_as_uint(m.p[q]) == w[1 + q]);
            if (!same) atomicOr(s.err, ERR_MATERIAL_HASH);
        }
        s.pm[i] = make_float4(p.position[0], p.position[1], D == 3 ? p.position[2] : 0.f, p.mass);
        if constexpr (!B) {
            for (int k = 0; k < D; ++k) {
                s.fdt[k * n + i] = p.force_dt[k];
                if (p.force_dt[k] != 0.f) sflags |= SCENE_FORCE;
            }
        }
        float Fm[D][D], Cm[D][D];
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                Fm[r][c] = p.def_grad[c * 3 + r];
                Cm[r][c] = p.affine[c * 3 + r];
            }
        float4 fv[MQ<D>::Q], cv[MQ<D>::Q];
        const float f22 = mat_split<D>(Fm, fv), c22 = mat_split<D>(Cm, cv);
#pragma unroll
        for (int q = 0; q < MQ<D>::Q; ++q) {
            s.fq[q * n + i] = fv[q];
            s.cq[q * n + i] = cv[q];
        }
        s.vv[i] = make_float4(p.velocity[0], p.velocity[1], D == 3 ? p.velocity[2] : 0.f, c22);
        if (p.damping != 0.f) sflags |= SCENE_DAMPING;
        if constexpr (!B) {
            io.r0[oid_base + i0] = p.init_radius;
            io.phase[oid_base + i0] = p.phase;
        }
        const uint32_t flags = (dense & FLAG_MAT_MASK) | (p.enabled ? FLAG_ENABLED : 0u) |
                               (p.fixed ? FLAG_FIXED : 0u) | (scene << FLAG_SCENE_SHIFT);
        s.fo[i] = make_uint4(flags, oid_base + i0, __float_as_uint(p.init_volume), __float_as_uint(f22));
        s.oid[i] = oid_base + i0;
        const bool sand = p.model.tag == SLOSH_MODEL_SAND_LINEAR || p.model.tag == SLOSH_MODEL_SAND_NEO_HOOKEAN;
        s.ps[i] = sand ? make_float4(p.model.data[0], p.model.data[1], p.model.data[2], p.damping)
                       : make_float4(0.f, 0.f, 0.f, p.damping);
        if (sand) sflags |= SCENE_SAND;
        sflags |= 1u << (SCENE_MODEL_SHIFT + min(p.model.tag, 7u));
    }
    sflags = __reduce_or_sync(FULL_MASK, sflags);
    if (lane_id() == 0 && sflags) atomicOr(io.scene_flags, sflags);
}

// Structure of arrays -> records, back in upload order (stored particle i is
// record oid[i]).  Multi-scene batches (B) export the particles of one scene;
// radius and phase are filled in by the host.
template <int D, bool B = false> __global__ void k_egest(DevScene s, IoBuffers io, uint32_t scene) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const size_t n = s.n;
    const uint32_t count = n_particles<B>(s);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint4 fo = s.fo[i];
        if constexpr (B)
            if (scene_of(fo.x) != scene) continue;
        const uint32_t orig = fo.y;
        slosh_particle p;
        const float4 pm = s.pm[i], vv = s.vv[i], ps = s.ps[i];
        p.position[0] = pm.x;
        p.position[1] = pm.y;
        p.position[2] = D == 3 ? pm.z : 0.f;
        p.velocity[0] = vv.x;
        p.velocity[1] = vv.y;
        p.velocity[2] = D == 3 ? vv.z : 0.f;
        for (int k = 0; k < 3; ++k) p.force_dt[k] = (k < D && s.force_pending) ? s.fdt[k * n + i] : 0.f;
        for (int q = 0; q < 9; ++q) {
            p.def_grad[q] = 0.f;
            p.affine[q] = 0.f;
        }
        float Fm[D][D], Cm[D][D];
        {
            float4 fv[MQ<D>::Q], cv[MQ<D>::Q];
#pragma unroll
            for (int q = 0; q < MQ<D>::Q; ++q) {
                fv[q] = s.fq[q * n + i];
                cv[q] = s.cq[q * n + i];
            }
            mat_from<D>(fv, __uint_as_float(fo.w), Fm);
            mat_from<D>(cv, vv.w, Cm);
        }
        for (int r = 0; r < D; ++r)
            for (int c = 0; c < D; ++c) {
                p.def_grad[c * 3 + r] = Fm[r][c];
                p.affine[c * 3 + r] = Cm[r][c];
            }
        p.vel_grad_det = 0.f;
        p.init_volume = __uint_as_float(fo.z);
        p.init_radius = B ? 0.f : io.r0[orig];
        p.mass = pm.w;
        p.damping = s.has_damping ? ps.w : 0.f;
        p.phase = B ? 0.f : io.phase[orig];
        const uint32_t fl = fo.x;
        p.enabled = (fl & FLAG_ENABLED) ? 1u : 0u;
        p.fixed = (fl & FLAG_FIXED) ? 1u : 0u;
        const Material &m = s.materials[fl & FLAG_MAT_MASK];
        p.model.tag = m.tag;
        for (int q = 0; q < 12; ++q) p.model.data[q] = m.p[q];
        if (m.tag == SLOSH_MODEL_SAND_LINEAR || m.tag == SLOSH_MODEL_SAND_NEO_HOOKEAN) {
            p.model.data[0] = ps.x;
            p.model.data[1] = ps.y;
            p.model.data[2] = ps.z;
        }
        io.out[orig] = p;
    }
}

// GpuParticles::shift_remove (src/solver/particle.rs:505-534) of the
// original ids [start, end): every other stored particle is copied from
// storage A to storage B at its new insertion-order index (ids past the
// range move down by end - start), so B holds the survivors in insertion
// order, like right after an upload.  The upload-order side arrays (radius,
// phase) and the pending forces move to the same new indices through
// `tmp` (3 + D floats a particle, plane stride s.n).
template <int D>
__global__ void k_remove(DevScene s, IoBuffers io, uint32_t start, uint32_t end, float *tmp) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const size_t n = s.n;
    const uint32_t removed = end - start;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.count; i += stride) {
        const uint4 fo = s.fo[i];
        const uint32_t o = fo.y;
        if (o >= start && o < end) continue;
        const uint32_t j = o >= end ? o - removed : o;
        s.out_pm[j] = s.pm[i];
        s.out_vv[j] = s.vv[i];
#pragma unroll
        for (int q = 0; q < MQ<D>::Q; ++q) {
            s.out_cq[q * n + j] = s.cq[q * n + i];
            s.out_fq[q * n + j] = s.fq[q * n + i];
        }
        s.out_ps[j] = s.ps[i];
        s.out_fo[j] = make_uint4(fo.x, j, fo.z, fo.w);
        s.out_oid[j] = j;
        tmp[j] = io.r0[o];
        tmp[n + j] = io.phase[o];
#pragma unroll
        for (int k = 0; k < D; ++k) tmp[(2 + k) * n + j] = s.force_pending ? s.fdt[k * n + i] : 0.0f;
    }
}

// Second pass of the removal: the side arrays and forces back from `tmp`.
template <int D> __global__ void k_remove_sides(DevScene s, IoBuffers io, uint32_t count, const float *tmp) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const size_t n = s.n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += stride) {
        io.r0[j] = tmp[j];
        io.phase[j] = tmp[n + j];
#pragma unroll
        for (int k = 0; k < D; ++k) s.fdt[k * n + j] = tmp[(2 + k) * n + j];
    }
}

// Positions as vec4 (x, y, z, 0) in upload order (of one scene in B).
template <bool B = false> __global__ void k_positions(DevScene s, float4 *out, uint32_t scene) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t count = n_particles<B>(s);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint2 fo = make_uint2(s.fo[i].x, s.fo[i].y);
        if constexpr (B)
            if (scene_of(fo.x) != scene) continue;
        const float4 p = s.pm[i];
        out[fo.y] = make_float4(p.x, p.y, p.z, 0.f);
    }
}

// Debug: the hot path's primary permutation in original ids.
__global__ void k_perm_to_oid(DevScene s, uint32_t *out) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < s.count; e += stride) out[e] = s.fo[s.perm[e]].y;
}

// ---------------------------------------------------------------------------
// Debug: slosh's full layout with extras (update_block_particle_count and
// finalize_particles_sort, sort.slang:208-246 and 304-357), in canonical
// order, built from the hot-path block ranks.
// ---------------------------------------------------------------------------
struct DebugBuffers {
    uint32_t *counts;  // nb * NB
    uint32_t *first;   // nb
    uint32_t *npe;     // nb
    uint32_t *np;      // nb
    uint32_t *cursor;  // nb * NB
    uint32_t *sorted;  // entries
    uint32_t *sorted2; // entries (canonicalised)
    uint32_t *total;   // 1
    uint32_t cap_entries;
};

template <int D>
__device__ __forceinline__ bool particle_rank_local(const DevScene &s, uint32_t i, uint32_t &r0, int *a) {
    const float4 p = s.pm[i];
    const float x[3] = {p.x, p.y, p.z};
    const CellLoc<D> c = locate<D>(x, s.h, s.inv_h, s.h_pow2);
    const uint32_t slot = hash_find(s.hkeys, s.hcap, pack_key<D>(c.block));
    if (slot == NONE) return false;
    r0 = rank_of(s.hvals[slot]);
    if (r0 == NONE) return false;
    for (int k = 0; k < D; ++k) a[k] = c.local[k];
    return true;
}

template <int D> __device__ __forceinline__ bool spills(const int *a, const int *o) {
    for (int k = 0; k < D; ++k)
        if (o[k] == 1 && a[k] < Geo<D>::MIN_SHIFT) return false;
    return true;
}

template <int D> __device__ __forceinline__ uint32_t extra_bucket(const int *a, const int *o) {
    const int local = a[D - 1] - o[D - 1] * Geo<D>::BW;
    return (uint32_t)(Geo<D>::NPB + (max(local, -2) + 2));
}

template <int D> __global__ void k_dbg_count(DevScene s, DebugBuffers d) {
    constexpr int NB = Geo<D>::NB, NN = Geo<D>::NASSOC - 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.count; i += stride) {
        uint32_t r0;
        int a[D];
        if (!particle_rank_local<D>(s, i, r0, a)) continue;
        atomicAdd(&d.counts[r0 * NB + a[D - 1]], 1u);
        for (int sidx = 1; sidx <= NN; ++sidx) {
            int o[D];
            assoc_offset<D>(sidx, o);
            if (!spills<D>(a, o)) continue;
            const uint32_t rb = s.bnbh[r0 * NN + sidx - 1];
            if (rb != NONE) atomicAdd(&d.counts[rb * NB + extra_bucket<D>(a, o)], 1u);
        }
    }
}

template <int D, int NT> __global__ void __launch_bounds__(NT) k_dbg_scan(DevScene s, DebugBuffers d) {
    constexpr int NB = Geo<D>::NB, NPB = Geo<D>::NPB;
    __shared__ uint32_t total_sh;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t per = (nb + NT - 1) / NT;
    const uint32_t r0 = threadIdx.x * per, r1 = min(r0 + per, nb);
    uint32_t local = 0;
    for (uint32_t r = r0; r < r1; ++r)
        for (int b = 0; b < NB; ++b) local += d.counts[r * NB + b];
    uint32_t run = block_exclusive_scan<NT>(local, &total_sh);
    for (uint32_t r = r0; r < r1; ++r) {
        d.first[r] = run;
        uint32_t tot = 0;
        for (int b = 0; b < NB; ++b) {
            if (b == NPB) d.np[r] = tot;
            d.cursor[r * NB + b] = run + tot;
            tot += d.counts[r * NB + b];
        }
        d.npe[r] = tot;
        run += tot;
    }
    if (threadIdx.x == 0) *d.total = total_sh;
}

template <int D> __global__ void k_dbg_scatter(DevScene s, DebugBuffers d) {
    constexpr int NB = Geo<D>::NB, NN = Geo<D>::NASSOC - 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.count; i += stride) {
        uint32_t r0;
        int a[D];
        if (!particle_rank_local<D>(s, i, r0, a)) continue;
        uint32_t pos = atomicAdd(&d.cursor[r0 * NB + a[D - 1]], 1u);
        if (pos < d.cap_entries) d.sorted[pos] = i;
        for (int sidx = 1; sidx <= NN; ++sidx) {
            int o[D];
            assoc_offset<D>(sidx, o);
            if (!spills<D>(a, o)) continue;
            const uint32_t rb = s.bnbh[r0 * NN + sidx - 1];
            if (rb == NONE) continue;
            pos = atomicAdd(&d.cursor[rb * NB + extra_bucket<D>(a, o)], 1u);
            if (pos < d.cap_entries) d.sorted[pos] = i;
        }
    }
}

// Canonical order of stored particle j in bucket b: primaries by (cell,
// original id), extras by original id.
template <int D>
__device__ __forceinline__ uint64_t dbg_order_key(const DevScene &s, uint32_t j, uint32_t b) {
    if (b >= (uint32_t)Geo<D>::NPB) return s.fo[j].y;
    const float4 p = s.pm[j];
    const float x[3] = {p.x, p.y, p.z};
    const CellLoc<D> c = locate<D>(x, s.h, s.inv_h, s.h_pow2);
    return ((uint64_t)cell_index<D>(c.local) << 32) | s.fo[j].y;
}

// One thread per (block, bucket) segment: rank each entry by its canonical
// order key inside the segment; the output holds original ids.
template <int D> __global__ void k_dbg_canon(DevScene s, DebugBuffers d) {
    constexpr int NB = Geo<D>::NB;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * NB; t += stride) {
        const uint32_t r = t / NB, b = t % NB;
        uint32_t lo = d.first[r];
        for (uint32_t q = 0; q < b; ++q) lo += d.counts[r * NB + q];
        const uint32_t hi = lo + d.counts[r * NB + b];
        if (hi > d.cap_entries) continue;
        for (uint32_t e = lo; e < hi; ++e) {
            const uint32_t id = d.sorted[e];
            const uint64_t key = dbg_order_key<D>(s, id, b);
            uint32_t rank = 0;
            for (uint32_t j = lo; j < hi; ++j) rank += (dbg_order_key<D>(s, d.sorted[j], b) < key) ? 1u : 0u;
            d.sorted2[lo + rank] = s.fo[id].y;
        }
    }
}

// Generic exclusive scan of n u32 (one CTA), slosh's prefix-sum semantics.
template <int NT> __global__ void __launch_bounds__(NT) k_exclusive_scan(const uint32_t *in, uint32_t *out, uint32_t n) {
    __shared__ uint32_t total_sh;
    const uint32_t per = (n + NT - 1) / NT;
    const uint32_t i0 = threadIdx.x * per, i1 = min(i0 + per, n);
    uint32_t local = 0;
    for (uint32_t i = i0; i < i1; ++i) local += in[i];
    uint32_t run = block_exclusive_scan<NT>(local, &total_sh);
    for (uint32_t i = i0; i < i1; ++i) {
        const uint32_t v = in[i];
        out[i] = run;
        run += v;
    }
}

}  // namespace slosh
