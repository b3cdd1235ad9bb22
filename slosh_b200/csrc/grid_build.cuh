// Sparse hashed grid build: block activation, canonical block ranking and
// the per-block counting sort of particles.
//
// Replaces WgGrid::launch_sort (src/grid/grid.rs:78-238) and the kernels it
// launches (shaders/slosh/grid/grid.slang, shaders/slosh/grid/sort.slang,
// shaders/slosh/grid/prefix_sum.slang).  Differences in design:
//  - one pass per particle both activates its primary block and counts it in
//    its cell, warp-aggregated (__match_any_sync) so that a warp of particles
//    sharing a block issues one hash insert and one atomic per (block, cell);
//  - the hash map stores 4-byte keys and 4-byte values in separate arrays
//    (slosh stores 48-byte entries) with twice the block capacity in slots;
//  - blocks are numbered canonically by ascending packed key (slosh numbers
//    them with an atomic counter), which makes every block index, offset and
//    the sorted permutation a deterministic function of the positions;
//  - particles are counted per cell of their primary block (64 cells) rather
//    than per slab: the canonical primary order is (cell, particle id) with
//    the cell index slab-major (x + BW y + BW^2 z), so slosh's slab buckets
//    are still contiguous ranges, and P2G/G2P get per-cell particle ranges;
//  - the permutation covers primaries only: P2G scatters from each particle
//    to its full stencil, so the "extra" entries slosh keeps for its
//    node-centric P2G are not needed on the hot path.  The debug entry point
//    rebuilds slosh's complete layout (primaries + extras) from the same data.
#pragma once

#include "scene.cuh"

namespace slosh {

constexpr uint32_t CELLS = 64;  // cells (and nodes) per block in 2D and 3D

// Linear-probing insert bounded by the slot count (slosh's insertion_index,
// grid.slang:118-174, probes the same way).  Sets ERR_HASH_OVERFLOW and
// returns NONE when the table is full.
__device__ __forceinline__ uint32_t hash_insert(uint32_t *keys, uint32_t hcap, uint32_t key, bool &inserted,
                                                uint32_t *err) {
    uint32_t slot = murmur_mix(key) & (hcap - 1u);
    for (uint32_t k = 0; k < hcap; ++k) {
        const uint32_t old = atomicCAS(&keys[slot], NONE, key);
        if (old == NONE) {
            inserted = true;
            return slot;
        }
        if (old == key) {
            inserted = false;
            return slot;
        }
        slot = (slot + 1u) & (hcap - 1u);
    }
    atomicOr(err, ERR_HASH_OVERFLOW);
    inserted = false;
    return NONE;
}

__device__ __forceinline__ uint32_t hash_find(const uint32_t *keys, uint32_t hcap, uint32_t key) {
    uint32_t slot = murmur_mix(key) & (hcap - 1u);
    for (uint32_t k = 0; k < hcap; ++k) {
        const uint32_t kk = keys[slot];
        if (kk == key) return slot;
        if (kk == NONE) return NONE;
        slot = (slot + 1u) & (hcap - 1u);
    }
    return NONE;
}

// Multi-scene maps: 64-bit keys (scene << 32 | packed block key), same
// linear probing.  With scene 0 the slot sequence is the single-scene one.
constexpr unsigned long long NONE64 = ~0ull;
__device__ __forceinline__ uint32_t hash64(unsigned long long k) {
    return murmur_mix((uint32_t)k ^ murmur_mix((uint32_t)(k >> 32) * 0x9e3779b1u));
}

__device__ __forceinline__ uint32_t hash_insert64(unsigned long long *keys, uint32_t hcap, unsigned long long key,
                                                  bool &inserted, uint32_t *err) {
    uint32_t slot = hash64(key) & (hcap - 1u);
    for (uint32_t k = 0; k < hcap; ++k) {
        const unsigned long long old = atomicCAS(&keys[slot], NONE64, key);
        if (old == NONE64) {
            inserted = true;
            return slot;
        }
        if (old == key) {
            inserted = false;
            return slot;
        }
        slot = (slot + 1u) & (hcap - 1u);
    }
    atomicOr(err, ERR_HASH_OVERFLOW);
    inserted = false;
    return NONE;
}

__device__ __forceinline__ uint32_t hash_find64(const unsigned long long *keys, uint32_t hcap, unsigned long long key) {
    uint32_t slot = hash64(key) & (hcap - 1u);
    for (uint32_t k = 0; k < hcap; ++k) {
        const unsigned long long kk = keys[slot];
        if (kk == key) return slot;
        if (kk == NONE64) return NONE;
        slot = (slot + 1u) & (hcap - 1u);
    }
    return NONE;
}

// Block map access of the single-scene (B = false: 32-bit keys, scene
// ignored) and the multi-scene (B = true) contexts.
template <bool B>
__device__ __forceinline__ uint32_t map_insert(const DevScene &s, uint32_t key, uint32_t sc, bool &inserted) {
    if constexpr (B) return hash_insert64(s.hkeys64, s.hcap, ((unsigned long long)sc << 32) | key, inserted, s.err);
    else return hash_insert(s.hkeys, s.hcap, key, inserted, s.err);
}
template <bool B> __device__ __forceinline__ uint32_t map_find(const DevScene &s, uint32_t key, uint32_t sc) {
    if constexpr (B) return hash_find64(s.hkeys64, s.hcap, ((unsigned long long)sc << 32) | key);
    else return hash_find(s.hkeys, s.hcap, key);
}
template <bool B> __device__ __forceinline__ uint32_t map_find_prev(const DevScene &s, uint32_t key, uint32_t sc) {
    if constexpr (B) return hash_find64(s.prev_hkeys64, s.hcap, ((unsigned long long)sc << 32) | key);
    else return hash_find(s.prev_hkeys, s.hcap, key);
}
// Particles in storage.
template <bool B> __device__ __forceinline__ uint32_t n_particles(const DevScene &s) {
    if constexpr (B) return *s.n_dev;
    else return s.count;
}

// Cell index of a local cell inside its block: x + BW y (+ BW^2 z).
template <int D> __device__ __forceinline__ uint32_t cell_index(const int *a) {
    if constexpr (D == 3) return (uint32_t)(a[0] + 4 * a[1] + 16 * a[2]);
    else return (uint32_t)(a[0] + 8 * a[1]);
}

// Clears the current hash map, the key histogram and the counters.  Replaces
// reset_hmap (grid.slang:200-218).  The per-slot cell counts are cleared by
// k_block_setup after they are read; after a substep that raised an error
// (blocks left without a rank keep their counts) they are all cleared here.
template <bool B = false> __global__ void k_clear(DevScene s) {
    pdl_enter();
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < s.hcap; i += stride) {
        if constexpr (B) s.hkeys64[i] = NONE64;
        else s.hkeys[i] = NONE;
        s.hvals[i] = NONE;
    }
    if constexpr (B)
        for (uint32_t i = tid; i < s.n_scenes; i += stride) s.scene_nblk[i] = 0u;
    if (*s.err != 0u)
        for (size_t i = tid; i < (size_t)s.hcap * CELLS; i += stride) s.slot_counts[i] = 0u;
    for (uint32_t i = tid; i < HIST_BINS; i += stride) s.hist[i] = 0u;
    if (tid < HIST_COARSE) s.hist_coarse[tid] = 0u;
    if (tid == 0) {
        s.ctr->n_primary = 0u;
        s.ctr->n_extra = 0u;
        s.ctr->n_blocks = 0u;
    }
}

// Per particle: activate the primary block and count the particle in its
// cell.  Replaces touch_primary_blocks (sort.slang:50-67) and the primary
// half of update_block_particle_count (sort.slang:208-246).
// Multi-scene batches (B): the particle's scene comes from its flags, its
// cell width from the scene table, and particles of a dropped scene get no
// block (they leave storage at this substep).
template <int D, bool B = false> __device__ __forceinline__ void touch_body(const DevScene &s, Cta g) {
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    // Each warp takes a contiguous chunk of storage.  Storage is in the
    // previous substep's canonical order (block by block), so successive
    // iterations of a warp mostly hit the block of the last one: the warp
    // remembers its last (key -> slot) and skips the hash CAS round trip.
    const uint32_t lane = lane_id();
    const uint32_t n = n_particles<B>(s);
    const uint32_t warps = g.n * (blockDim.x >> 5);
    const uint32_t wid = g.id * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t chunk = (((n + warps - 1) / warps) + 31u) & ~31u;
    const uint32_t begin = wid * chunk;
    const uint32_t end = min(n, begin + chunk);
    unsigned long long last_key = NONE64;
    uint32_t last_slot = NONE;
    for (uint32_t base = begin; base < end; base += 32) {
        const uint32_t i = base + lane;
        const bool valid = i < end;
        const unsigned mask = __ballot_sync(FULL_MASK, valid);
        if (!valid) break;
        const float4 p = s.pm[i];
        const float x[3] = {p.x, p.y, p.z};
        float h = s.h, inv_h = s.inv_h;
        uint32_t pow2 = s.h_pow2, sc = 0;
        bool live = true;
        if constexpr (B) {
            sc = scene_of(s.fo[i].x);
            const SceneRec &rec = s.scenes[sc];
            h = rec.h;
            inv_h = rec.inv_h;
            pow2 = rec.h_pow2;
            live = rec.live != 0u;
        }
        const CellLoc<D> c = locate<D>(x, h, inv_h, pow2);
        const uint32_t key = pack_key<D>(c.block);
        const uint32_t cell = cell_index<D>(c.local);
        const unsigned long long ckey = live ? (((unsigned long long)sc << 32) | key) : NONE64;
        unsigned peers;
        if constexpr (B) peers = __match_any_sync(mask, ckey);
        else peers = __match_any_sync(mask, key);  // one scene: the 32-bit key is the whole key
        const int leader = __ffs(peers) - 1;
        uint32_t slot = NONE;
        if ((int)lane == leader && live) {
            if (ckey == last_key) {
                slot = last_slot;
            } else {
                bool inserted = false;
                slot = map_insert<B>(s, key, sc, inserted);
                if (inserted) {
                    const uint32_t j = atomicAdd(&s.ctr->n_primary, 1u);
                    if (j < s.cap) {
                        s.blist_key[j] = key;
                        s.blist_slot[j] = slot;
                        if constexpr (B) atomicAdd(&s.scene_nblk[sc], 1u);
                        else atomicAdd(&s.hist[key >> 16], 1u);
                    } else {
                        atomicOr(s.err, ERR_BLOCK_OVERFLOW);
                    }
                }
            }
        }
        slot = __shfl_sync(mask, slot, leader);
        const int top = 31 - __clz(mask);  // last valid lane: its block is the likeliest next
        if constexpr (B) last_key = __shfl_sync(mask, ckey, top);
        else last_key = __shfl_sync(mask, key, top);
        last_slot = __shfl_sync(mask, slot, top);
        const uint32_t bin = (slot == NONE) ? NONE : (slot << 6) | cell;
        const unsigned peers2 = __match_any_sync(mask, bin);
        if (bin != NONE && (int)lane == __ffs(peers2) - 1) atomicAdd(&s.slot_counts[bin], (uint32_t)__popc(peers2));
        s.pslot[i] = bin;
    }
}
template <int D, bool B = false> __global__ void k_touch(DevScene s) {
    pdl_enter();
    touch_body<D, B>(s, launch_cta());
}

// Activates the +1 neighbours of every primary block, one thread per
// (block, neighbour).  Replaces touch_neighbor_blocks (sort.slang:75-92).
// Single scene: also counts the primary and the new blocks in the coarse
// histogram (key >> 26), aggregated over the warp (a compact scene has one
// or two coarse bins, so per-block atomics would all hit one address).
template <int D, bool B = false> __device__ __forceinline__ void neighbors_body(const DevScene &s, Cta g) {
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    constexpr int NN = Geo<D>::NASSOC - 1;
    const uint32_t np = min(s.ctr->n_primary, s.cap);
    const uint32_t stride = g.n * blockDim.x;
    for (uint32_t t = g.id * blockDim.x + threadIdx.x; t < np * NN; t += stride) {
        const uint32_t j = t / NN;
        const int sidx = (int)(t % NN) + 1;
        int b[D], o[D];
        const uint32_t pkey = s.blist_key[j];
        unpack_key<D>(pkey, b);
        assoc_offset<D>(sidx, o);
        for (int k = 0; k < D; ++k) b[k] += o[k];
        const uint32_t key = pack_key<D>(b);
        uint32_t sc = 0;
        if constexpr (B) sc = (uint32_t)(s.hkeys64[s.blist_slot[j]] >> 32);
        bool inserted = false, counted = false;
        const uint32_t slot = map_insert<B>(s, key, sc, inserted);
        if (inserted) {
            const uint32_t jj = atomicAdd(&s.ctr->n_extra, 1u);
            if (jj < s.cap) {
                s.blist2_key[jj] = key;
                s.blist2_slot[jj] = slot;
                if constexpr (B) atomicAdd(&s.scene_nblk[sc], 1u);
                else atomicAdd(&s.hist[key >> 16], 1u);
                counted = true;
            } else {
                atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            }
        }
        if constexpr (!B) {
            const unsigned act = __activemask();
            const uint32_t lane = lane_id();
            const uint32_t cp = sidx == 1 ? pkey >> 26 : NONE, ce = counted ? key >> 26 : NONE;
            const unsigned pp = __match_any_sync(act, cp), pe = __match_any_sync(act, ce);
            if (cp != NONE && (int)lane == __ffs(pp) - 1) atomicAdd(&s.hist_coarse[cp], (uint32_t)__popc(pp));
            if (ce != NONE && (int)lane == __ffs(pe) - 1) atomicAdd(&s.hist_coarse[ce], (uint32_t)__popc(pe));
        }
    }
}
template <int D, bool B = false> __global__ void k_neighbors(DevScene s) {
    pdl_enter();
    neighbors_body<D, B>(s, launch_cta());
}

// Block-wide exclusive scan of one value per thread (blockDim.x == NT,
// NT <= 1024, a multiple of 32).  Writes the block total to *total.
template <int NT> __device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total) {
    constexpr int NW = NT / 32;
    __shared__ uint32_t warp_sums[NW];
    __shared__ uint32_t block_total;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
        if (lane >= (uint32_t)off) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t ws = (lane < (uint32_t)NW) ? warp_sums[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, wi, off);
            if (lane >= (uint32_t)off) wi += y;
        }
        if (lane < (uint32_t)NW) warp_sums[lane] = wi - ws;
        if (lane == 31) block_total = wi;
    }
    __syncthreads();
    const uint32_t res = warp_sums[warp] + incl - v;
    if (total) *total = block_total;
    __syncthreads();
    return res;
}

// Exclusive scan of n u32 by one CTA of NT threads: tiles of NT * PER values
// staged in shared memory with coalesced loads, each thread scanning PER
// consecutive values; `carry` holds the running total.  Returns the total.
template <int NT, int PER>
__device__ __forceinline__ uint32_t cta_exclusive_scan(const uint32_t *in, uint32_t *out, uint32_t n) {
    __shared__ uint32_t tile[NT * PER];
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < n; base += NT * PER) {
        for (uint32_t k = threadIdx.x; k < NT * PER; k += NT) tile[k] = (base + k < n) ? in[base + k] : 0u;
        __syncthreads();
        uint32_t local = 0;
        const uint32_t t0 = threadIdx.x * PER;
#pragma unroll
        for (int k = 0; k < PER; ++k) local += tile[t0 + k];
        uint32_t run = carry + block_exclusive_scan<NT>(local, &tot);
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const uint32_t v = tile[t0 + k];
            tile[t0 + k] = run;
            run += v;
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < NT * PER; k += NT)
            if (base + k < n) out[base + k] = tile[k];
        carry += tot;
        __syncthreads();
    }
    return carry;
}

// Exclusive scan of n u32 by one CTA, each thread owning 16 consecutive
// values read and written as four 16-byte vectors (in and out must be
// 16-byte aligned).  Returns the total.
template <int NT> __device__ __forceinline__ uint32_t cta_scan_vec16(const uint32_t *in, uint32_t *out, uint32_t n) {
    constexpr uint32_t V = 16, TILE = NT * V;
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < n; base += TILE) {
        const uint32_t b = base + threadIdx.x * V;
        uint32_t v[V];
        if (b + V <= n) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint4 u = reinterpret_cast<const uint4 *>(in + b)[q];
                v[4 * q] = u.x;
                v[4 * q + 1] = u.y;
                v[4 * q + 2] = u.z;
                v[4 * q + 3] = u.w;
            }
        } else {
#pragma unroll
            for (uint32_t k = 0; k < V; ++k) v[k] = (b + k < n) ? in[b + k] : 0u;
        }
        uint32_t local = 0;
#pragma unroll
        for (uint32_t k = 0; k < V; ++k) local += v[k];
        uint32_t run = carry + block_exclusive_scan<NT>(local, &tot);
#pragma unroll
        for (uint32_t k = 0; k < V; ++k) {
            const uint32_t x = v[k];
            v[k] = run;
            run += x;
        }
        if (b + V <= n) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                reinterpret_cast<uint4 *>(out + b)[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        } else {
#pragma unroll
            for (uint32_t k = 0; k < V; ++k)
                if (b + k < n) out[b + k] = v[k];
        }
        carry += tot;
    }
    return carry;
}

// Exclusive scan of the key histogram and the final block count.  CTA c
// scans bins [1024 c, 1024 c + 1024), one uint4 a thread, on top of the
// coarse counts of the bins before them.
template <int NT> __global__ void __launch_bounds__(NT) k_hist_scan(DevScene s) {
    pdl_enter();
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    constexpr uint32_t PER = HIST_BINS / HIST_COARSE, NW = NT / 32;
    static_assert(PER == 4 * NT && HIST_COARSE <= 64, "one uint4 of bins a thread");
    __shared__ uint32_t wtot[NW];
    __shared__ uint32_t base;
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5, c = blockIdx.x;
    if (w == 0) {
        uint32_t v = (lane < c ? s.hist_coarse[lane] : 0u) + (lane + 32u < c ? s.hist_coarse[lane + 32u] : 0u);
        v = __reduce_add_sync(FULL_MASK, v);
        if (lane == 0) base = v;
    }
    const uint4 v = reinterpret_cast<const uint4 *>(s.hist + (size_t)c * PER)[threadIdx.x];
    const uint32_t sum = v.x + v.y + v.z + v.w;
    uint32_t incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
        if (lane >= (uint32_t)off) incl += y;
    }
    if (lane == 31) wtot[w] = incl;
    __syncthreads();
    uint32_t pre = base;
    for (uint32_t q = 0; q < w; ++q) pre += wtot[q];
    uint4 o;
    o.x = pre + incl - sum;
    o.y = o.x + v.x;
    o.z = o.y + v.y;
    o.w = o.z + v.z;
    reinterpret_cast<uint4 *>(s.hist_start + (size_t)c * PER)[threadIdx.x] = o;
    if (c == 0 && threadIdx.x == 0) {
        const uint32_t total = min(s.ctr->n_primary, s.cap) + min(s.ctr->n_extra, s.cap);
        if (total > s.cap) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
        s.ctr->n_blocks = min(total, s.cap);
    }
}

// Groups the appended block keys by their top 16 bits.
__global__ void k_bin_scatter(DevScene s) {
    pdl_enter();
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    const uint32_t n1 = min(s.ctr->n_primary, s.cap), n2 = min(s.ctr->n_extra, s.cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n1 + n2; t += stride) {
        const uint32_t key = t < n1 ? s.blist_key[t] : s.blist2_key[t - n1];
        const uint32_t slot = t < n1 ? s.blist_slot[t] : s.blist2_slot[t - n1];
        const uint32_t b = key >> 16;
        const uint32_t pos = atomicAdd(&s.hist_start[b], 1u);
        s.tmp_key[pos] = key;
        s.tmp_slot[pos] = slot | (t < n1 ? 0u : RANK_EXTRA);
    }
}

// Canonical rank = number of active keys smaller than this one.  Keys of one
// top-16-bit bin are compared against each other only, by RANK_LANES lanes
// a key, each counting every RANK_LANES-th key of the bin (a bin holds a
// whole z slab of a compact scene, hundreds of keys).
constexpr uint32_t RANK_LANES = 8;
__global__ void k_rank(DevScene s) {
    pdl_enter();
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    const uint32_t total = min(s.ctr->n_primary, s.cap) + min(s.ctr->n_extra, s.cap);
    const uint32_t g = threadIdx.x % RANK_LANES;
    const unsigned gmask = ((1u << RANK_LANES) - 1u) << (lane_id() & ~(RANK_LANES - 1u));
    const uint32_t stride = gridDim.x * (blockDim.x / RANK_LANES);
    for (uint32_t t = blockIdx.x * (blockDim.x / RANK_LANES) + threadIdx.x / RANK_LANES; t < total; t += stride) {
        const uint32_t key = s.tmp_key[t];
        const uint32_t b = key >> 16;
        const uint32_t end = s.hist_start[b], start = end - s.hist[b];  // advanced by k_bin_scatter
        uint32_t part = 0;
#pragma unroll 4
        for (uint32_t j = start + g; j < end; j += RANK_LANES) part += (s.tmp_key[j] < key) ? 1u : 0u;
#pragma unroll
        for (uint32_t off = RANK_LANES / 2; off > 0; off >>= 1) part += __shfl_xor_sync(gmask, part, off);
        const uint32_t r = start + part;
        if (g == 0 && r < s.cap) {
            const uint32_t ts = s.tmp_slot[t], slot = ts & ~RANK_EXTRA;
            s.bkey[r] = key;
            s.bslot[r] = slot;
            s.hvals[slot] = r | (ts & RANK_EXTRA);
        }
    }
}

// ---- multi-scene block ranking ----------------------------------------------
// Blocks are ranked scene-major and by ascending packed key within a scene,
// so each scene gets the block order (and hence the particle storage order)
// it would have alone.  Per-scene block counts were taken when the blocks
// were inserted; one CTA scans them into per-scene rank bases.
template <int NT> __device__ __forceinline__ void scene_scan_body(const DevScene &s) {
    const uint32_t total = cta_scan_vec16<NT>(s.scene_nblk, s.scene_bbase, s.n_scenes);
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < s.n_scenes; q += NT) s.scene_fill[q] = s.scene_bbase[q];
    if (threadIdx.x == 0) {
        if (total > s.cap) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
        s.ctr->n_blocks = min(total, s.cap);
    }
}
template <int NT> __global__ void __launch_bounds__(NT) k_scene_scan(DevScene s) {
    pdl_enter();
    scene_scan_body<NT>(s);
}

// Groups the appended blocks by scene (unordered within a scene).
__device__ __forceinline__ void scene_scatter_body(const DevScene &s, Cta g) {
    const uint32_t n1 = min(s.ctr->n_primary, s.cap), n2 = min(s.ctr->n_extra, s.cap);
    const uint32_t stride = g.n * blockDim.x;
    for (uint32_t t = g.id * blockDim.x + threadIdx.x; t < n1 + n2; t += stride) {
        const uint32_t key = t < n1 ? s.blist_key[t] : s.blist2_key[t - n1];
        const uint32_t slot = t < n1 ? s.blist_slot[t] : s.blist2_slot[t - n1];
        const uint32_t sc = (uint32_t)(s.hkeys64[slot] >> 32);
        const uint32_t pos = atomicAdd(&s.scene_fill[sc], 1u);
        if (pos < 2u * s.cap) {
            s.tmp_key[pos] = key;
            s.tmp_slot[pos] = slot | (t < n1 ? 0u : RANK_EXTRA);
        }
    }
}
__global__ void k_scene_scatter(DevScene s) { pdl_enter(); scene_scatter_body(s, launch_cta()); }

// Scenes beyond this many active blocks raise ERR_SCENE_BLOCKS (a scene of
// about 7 M particles; larger ones belong in a context of their own).
constexpr uint32_t SCENE_MAX_BLOCKS = 16384;

// Block ranks of a batch: the blocks of each scene (grouped by
// k_scene_scatter) ranked by counting the scene's smaller keys, RANK_LANES
// lanes a block.  Keys are distinct inside a scene, so the rank is the
// block's place in the scene's ascending key order.  Written: the block's
// key, hash slot and scene at its rank, and the rank into the hash map.
__device__ __forceinline__ void scene_rank_body(const DevScene &s, Cta g) {
    const uint32_t total = min(s.ctr->n_primary, s.cap) + min(s.ctr->n_extra, s.cap);
    const uint32_t gl = threadIdx.x % RANK_LANES;
    const unsigned gmask = ((1u << RANK_LANES) - 1u) << (lane_id() & ~(RANK_LANES - 1u));
    const uint32_t stride = g.n * (blockDim.x / RANK_LANES);
    for (uint32_t t = g.id * (blockDim.x / RANK_LANES) + threadIdx.x / RANK_LANES; t < total; t += stride) {
        const uint32_t key = s.tmp_key[t], ts = s.tmp_slot[t], slot = ts & ~RANK_EXTRA;
        const uint32_t sc = (uint32_t)(s.hkeys64[slot] >> 32);
        const uint32_t m = s.scene_nblk[sc], base = s.scene_bbase[sc];
        if (m > SCENE_MAX_BLOCKS) {
            if (gl == 0) atomicOr(s.err, ERR_SCENE_BLOCKS);
            continue;
        }
        if (base + m > 2u * s.cap) continue;  // overflow, already flagged
        uint32_t part = 0;
#pragma unroll 4
        for (uint32_t j = base + gl; j < base + m; j += RANK_LANES) part += (s.tmp_key[j] < key) ? 1u : 0u;
#pragma unroll
        for (uint32_t off = RANK_LANES / 2; off > 0; off >>= 1) part += __shfl_xor_sync(gmask, part, off);
        const uint32_t r = base + part;
        if (gl == 0 && r < s.cap) {
            s.bkey[r] = key;
            s.bslot[r] = slot;
            s.bscene[r] = sc;
            s.hvals[slot] = r | (ts & RANK_EXTRA);
        }
    }
}
__global__ void k_scene_rank(DevScene s) { pdl_enter(); scene_rank_body(s, launch_cta()); }

// One warp per block: per-cell counts (cleared in the hash-slot array once
// read) with their in-block exclusive scan, the block total, the cells in
// decreasing count order for P2G's thread assignment, the +1 and -1
// neighbour ranks (update_nbh_block_ids, sort.slang:100-117), the block's
// rank in the previous substep's map (the grid update's collision cache) and, for the
// atomic P2G variants, zeroed nodes (reset, grid.slang:455-485).
template <int D, bool B = false> __device__ __forceinline__ void block_setup_body(const DevScene &s, Cta g) {
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    constexpr int NN = Geo<D>::NASSOC - 1;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t lane = lane_id();
    const uint32_t warps = g.n * (blockDim.x >> 5);
    if (g.id == 0 && threadIdx.x == 0) {  // the transfer kernels' block queues, read after this kernel
        s.ctr->p2g_next = 0u;
        s.ctr->g2p_next = 0u;
        if constexpr (B)
            if (s.g2p_lists)
                for (uint32_t c = 0; c < G2P_CLASSES; ++c) s.g2p_counts[G2P_CLASSES + c] = 0u;
    }
    for (uint32_t r = g.id * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nb; r += warps) {
        const uint32_t sl = s.bslot[r];
        uint32_t *cnt = s.slot_counts + ((size_t)sl << 6);
        const uint32_t c0 = cnt[2 * lane], c1 = cnt[2 * lane + 1];
        cnt[2 * lane] = 0u;
        cnt[2 * lane + 1] = 0u;
        const uint32_t pair = c0 + c1;
        uint32_t incl = pair;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
            if (lane >= (uint32_t)off) incl += y;
        }
        const uint32_t ex = incl - pair;
        s.bcell[(size_t)r * CELLS + 2 * lane] = ex;
        s.bcell[(size_t)r * CELLS + 2 * lane + 1] = ex + c0;
        s.bcur[(size_t)r * CELLS + 2 * lane] = ex;
        s.bcur[(size_t)r * CELLS + 2 * lane + 1] = ex + c0;
        if (lane == 31) {
            s.bnp[r] = incl;
            if (incl >= (1u << 26)) atomicOr(s.err, ERR_BLOCK_PARTICLES);  // beyond the 26-bit first in bord
            if (s.bsrc) s.bsrc[r] = NONE;  // a full build's permutation is no shifted range
            if constexpr (B)
                if (s.g2p_lists && incl != 0u) {  // the block goes to its scene's G2P launch
                    const uint32_t cls = s.scenes[s.bscene[r]].g2p_class;
                    s.g2p_lists[(size_t)cls * s.cap + atomicAdd(&s.g2p_counts[cls], 1u)] = r;
                }
        }
        {
            // rank of each cell among the 64 by (count desc, cell asc): the
            // number of keys above its own, keys being distinct
            const uint32_t k0 = (min(c0, 0x3ffffffu) << 6) | (63u - 2u * lane);
            const uint32_t k1 = (min(c1, 0x3ffffffu) << 6) | (62u - 2u * lane);
            uint32_t r0 = 0, r1 = 0;
#pragma unroll 8
            for (int q = 0; q < 32; ++q) {
                const uint32_t a = __shfl_sync(FULL_MASK, k0, q), b = __shfl_sync(FULL_MASK, k1, q);
                r0 += (a > k0) + (b > k0);
                r1 += (a > k1) + (b > k1);
            }
            s.bord[(size_t)r * CELLS + r0] = make_uint2((2u * lane) | (ex << 6), c0);
            s.bord[(size_t)r * CELLS + r1] = make_uint2((2u * lane + 1u) | ((ex + c0) << 6), c1);
        }
        if (!s.use_partial) {  // the atomic P2G variants accumulate into the nodes
            s.nodes[(size_t)r * 64 + 2 * lane] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.nodes[(size_t)r * 64 + 2 * lane + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        // lanes [0, NN): the +1 neighbours b + o; lanes [NN, 2 NN): the -1
        // neighbours b - o, whose P2G tiles overlap this block.
        if (lane < (uint32_t)(2 * NN)) {
            const bool fwd = lane < (uint32_t)NN;
            const int q = fwd ? (int)lane : (int)lane - NN;
            int b[D], o[D];
            unpack_key<D>(s.bkey[r], b);
            assoc_offset<D>(q + 1, o);
            for (int k = 0; k < D; ++k) b[k] += fwd ? o[k] : -o[k];
            const uint32_t slot = map_find<B>(s, pack_key<D>(b), B ? s.bscene[r] : 0u);
            const uint32_t v = (slot == NONE) ? NONE : s.hvals[slot];
            // the grid update gathers the tiles of the -1 neighbours that hold particles
            if (fwd) s.bnbh[r * NN + q] = rank_of(v);
            else s.bnbh_rev[r * NN + q] = (v & RANK_EXTRA) ? NONE : v;
        } else if (lane == (uint32_t)(2 * NN)) {
            const uint32_t slot = map_find_prev<B>(s, s.bkey[r], B ? s.bscene[r] : 0u);
            s.bprev[r] = (slot == NONE) ? NONE : rank_of(s.prev_hvals[slot]);
        }
    }
}
template <int D, bool B = false> __global__ void k_block_setup(DevScene s) {
    pdl_enter();
    block_setup_body<D, B>(s, launch_cta());
}

// Exclusive scan of the per-block primary totals into first_particle
// (copy_particles_len_to_scan_value + prefix_sum +
// copy_scan_values_to_first_particles, sort.slang:248-302).  One CTA.
template <int NT> __device__ __forceinline__ void block_scan_body(const DevScene &s) {
    if (build_skipped(s)) return;  // a kept grid's offsets come from k_grid_reuse / k_reuse_perm
    const uint32_t nb = s.ctr->n_blocks;
    cta_scan_vec16<NT>(s.bnp, s.bfirst, nb);
    // P2G's queue order, heaviest blocks first (buckets of 8 particles), so
    // that the last blocks its warps take are light and they finish together.
    // A substep that keeps its grid keeps the order too: the same blocks, and
    // block counts that changed by a few particles at most (the order only
    // balances P2G's load; results do not depend on it).
    if (!s.p2g_heavy_first) return;
    __shared__ uint32_t cnt[64];
    if (threadIdx.x < 64) cnt[threadIdx.x] = 0u;
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < nb; r += NT) atomicAdd(&cnt[min(s.bnp[r] >> 3, 63u)], 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int b = 63; b >= 0; --b) {
            const uint32_t c = cnt[b];
            cnt[b] = run;
            run += c;
        }
    }
    __syncthreads();
    for (uint32_t r = threadIdx.x; r < nb; r += NT) s.qorder[atomicAdd(&cnt[min(s.bnp[r] >> 3, 63u)], 1u)] = r;
}
template <int NT> __global__ void __launch_bounds__(NT) k_block_scan(DevScene s) {
    pdl_enter();
    block_scan_body<NT>(s);
}

// Per particle: claim its slot in the block's cell range (the primary part
// of finalize_particles_sort, sort.slang:304-357), warp-aggregated.
//
// Each warp takes a contiguous chunk of storage and walks it in order; a
// warp's next claim waits for the previous one's result, so a cell's
// particles handled by one warp land in storage order, which is already the
// canonical order for particles that stayed in their cell.  Only cells split
// between two chunks (and cells entered from another cell) need k_canon's
// fix-up.  Like k_touch, a warp remembers the block of its last lane (hash
// slot -> rank, first entry), so most iterations go straight to the claim.
template <bool B = false> __device__ __forceinline__ void scatter_body(const DevScene &s, Cta g) {
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    const uint32_t lane = lane_id();
    const uint32_t n = n_particles<B>(s);
    const uint32_t warps = g.n * (blockDim.x >> 5);
    const uint32_t wid = g.id * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t chunk = (((n + warps - 1) / warps) + 31u) & ~31u;
    const uint32_t begin = wid * chunk;
    const uint32_t end = min(n, begin + chunk);
    uint32_t c_slot = NONE, c_r = NONE, c_first = 0;
    uint32_t bin_next = begin + lane < end ? s.pslot[begin + lane] : NONE;
    for (uint32_t base = begin; base < end; base += 32) {
        const uint32_t i = base + lane;
        const bool valid = i < end;
        const unsigned mask = __ballot_sync(FULL_MASK, valid);
        if (!valid) break;
        const uint32_t bin = bin_next;
        bin_next = i + 32u < end ? s.pslot[i + 32u] : NONE;
        const unsigned peers = __match_any_sync(mask, bin);
        const int leader = __ffs(peers) - 1;
        const uint32_t sl = bin >> 6;
        uint32_t pos = NONE, r = NONE, first = 0;
        if ((int)lane == leader && bin != NONE) {
            if (sl == c_slot) {
                r = c_r;
                first = c_first;
            } else {
                r = rank_of(s.hvals[sl]);
                if (r != NONE) first = s.bfirst[r];
            }
            if (r != NONE) pos = first + atomicAdd(&s.bcur[(size_t)r * CELLS + (bin & 63u)], (uint32_t)__popc(peers));
        }
        pos = __shfl_sync(mask, pos, leader);
        r = __shfl_sync(mask, r, leader);
        first = __shfl_sync(mask, first, leader);
        const int top = 31 - __clz(mask);
        if (__shfl_sync(mask, bin, top) != NONE) {
            c_slot = __shfl_sync(mask, sl, top);
            c_r = __shfl_sync(mask, r, top);
            c_first = __shfl_sync(mask, first, top);
        }
        if (pos != NONE) {
            const uint32_t at = pos + __popc(peers & lanemask_lt());
            if (at < s.n) {
                s.perm[at] = i;
                s.skey[at] = ((unsigned long long)(bin & 63u) << 32) | s.oid[i];
            } else {
                atomicOr(s.err, ERR_BLOCK_OVERFLOW);  // stale counts after an earlier overflow
            }
        }
    }
}
template <bool B = false> __global__ void k_scatter(DevScene s) {
    pdl_enter();
    scatter_body<B>(s, launch_cta());
}

// Canonical order inside each (block, cell) range of the permutation:
// ascending original id.  k_scatter stores beside every permutation entry
// its sort key (cell << 32 | original id).  Storage is already in the
// previous substep's canonical order and the scatter keeps a warp's lanes in
// storage order, so most cells come out sorted; the ones that do not are
// cells whose particles were scattered by two different warps.  One warp per
// block compares neighbouring keys (coalesced loads of the block's
// contiguous entries); each out-of-order cell is then sorted by the whole
// warp: lane l holds entry l, its rank is the number of smaller original ids
// (shuffles), and entries are stored at their ranks.  Cells of more than 32
// entries are insertion-sorted by one lane.
__device__ __forceinline__ void sort_cell_keys(unsigned long long *key, uint32_t *perm, uint32_t m) {
    for (uint32_t j = 1; j < m; ++j) {
        const unsigned long long kj = key[j];
        const uint32_t pj = perm[j];
        int q = (int)j - 1;
        while (q >= 0 && key[q] > kj) {
            key[q + 1] = key[q];
            perm[q + 1] = perm[q];
            --q;
        }
        key[q + 1] = kj;
        perm[q + 1] = pj;
    }
}

__device__ __forceinline__ void canon_body(const DevScene &s, Cta g) {
    if (build_skipped(s)) return;  // this substep keeps the previous grid
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t lane = lane_id();
    const uint32_t warps = g.n * (blockDim.x >> 5);
    // With few blocks (a small scene) G warps share a block, warp `part`
    // sorting the cells c with c % G == part, so that a block's out-of-order
    // cells are sorted side by side instead of one after another.  Cells
    // are disjoint, so the result does not depend on G.
    uint32_t G = 1u;
    while (G < 8u && (size_t)nb * G * 2u <= warps) G <<= 1;
    for (uint32_t t = g.id * (blockDim.x >> 5) + (threadIdx.x >> 5); t < nb * G; t += warps) {
        const uint32_t r = t / G, part = t % G;
        const uint32_t first = s.bfirst[r], np = s.bnp[r];
        if (np < 2) continue;
        if ((size_t)first + np > s.n) {  // only after an earlier overflow left stale counts
            if (lane == 0 && part == 0) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            continue;
        }
        const unsigned long long *k = s.skey + first;
        unsigned long long bad = 0ull;  // cells holding an inversion
        for (uint32_t e = lane; e + 1 < np; e += 32) {
            const unsigned long long k0 = k[e], k1 = k[e + 1];
            if (k0 > k1 && (k0 >> 32) == (k1 >> 32)) bad |= 1ull << (uint32_t)(k0 >> 32);
        }
        if (G > 1u) {
            unsigned long long mine = 0ull;
            for (uint32_t c = part; c < CELLS; c += G) mine |= 1ull << c;
            bad &= mine;
        }
        const uint32_t lo = __reduce_or_sync(FULL_MASK, (uint32_t)bad);
        const uint32_t hi = __reduce_or_sync(FULL_MASK, (uint32_t)(bad >> 32));
        if ((lo | hi) == 0u) continue;
        unsigned long long cells = ((unsigned long long)hi << 32) | lo;
        while (cells != 0ull) {
            const uint32_t c = (uint32_t)__ffsll((long long)cells) - 1u;
            cells &= cells - 1ull;
            const uint32_t b0 = s.bcell[(size_t)r * CELLS + c];
            const uint32_t b1 = (c < CELLS - 1) ? s.bcell[(size_t)r * CELLS + c + 1] : np;
            if (b1 <= b0 + 1 || b1 > np) continue;
            const uint32_t m = b1 - b0;
            unsigned long long *ck = s.skey + first + b0;
            uint32_t *cp = s.perm + first + b0;
            if (m > 32u) {
                if (lane == 0) sort_cell_keys(ck, cp, m);
                __syncwarp();
                continue;
            }
            const unsigned long long kl = lane < m ? ck[lane] : ~0ull;
            const uint32_t pl = lane < m ? cp[lane] : 0u;
            const uint32_t id = (uint32_t)kl;  // the cell part of the keys is equal
            uint32_t rank = 0;
            for (uint32_t j = 0; j < m; ++j) rank += __shfl_sync(FULL_MASK, id, j) < id ? 1u : 0u;
            __syncwarp();  // every lane has read its entry
            if (lane < m) {
                ck[rank] = kl;
                cp[rank] = pl;
            }
            __syncwarp();
        }
    }
}
__global__ void k_canon(DevScene s) { pdl_enter(); canon_body(s, launch_cta()); }

}  // namespace slosh
