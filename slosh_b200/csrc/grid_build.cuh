// Sparse hashed grid build: block activation, canonical block ranking and
// the per-block counting sort of particles.
//
// Replaces WgGrid::launch_sort (src/grid/grid.rs:78-238) and the kernels it
// launches (shaders/slosh/grid/grid.slang, shaders/slosh/grid/sort.slang,
// shaders/slosh/grid/prefix_sum.slang).  Differences in design:
//  - one pass per particle both activates its primary block and counts it in
//    its slab bucket, warp-aggregated (__match_any_sync) so that a warp of
//    particles sharing a block issues one hash insert and one atomic per
//    (block, bucket) instead of one per particle;
//  - the hash map stores 4-byte keys and 4-byte values in separate arrays
//    (slosh stores 48-byte entries) with twice the block capacity in slots;
//  - blocks are numbered canonically by ascending packed key (slosh numbers
//    them with an atomic counter), which makes every block index, offset and
//    the sorted permutation a deterministic function of the positions;
//  - the particle permutation covers primaries only: P2G scatters from each
//    particle to its full 27-node stencil, so the "extra" entries slosh keeps
//    for its node-centric P2G are not needed on the hot path.  The debug
//    entry point rebuilds slosh's complete layout (primaries + extras) from
//    the same data for the bit-exactness checks.
#pragma once

#include "scene.cuh"

namespace slosh {

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

// Clears the current hash map, the per-slot counts, the key histogram and
// the counters.  Replaces reset_hmap (grid.slang:200-218).
template <int D> __global__ void k_clear(DevScene s) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < s.hcap; i += stride) {
        s.hkeys[i] = NONE;
        s.hvals[i] = NONE;
    }
    for (uint32_t i = tid; i < s.hcap * Geo<D>::NPB; i += stride) s.slot_counts[i] = 0u;
    for (uint32_t i = tid; i < HIST_BINS; i += stride) {
        s.hist[i] = 0u;
        s.hist_fill[i] = 0u;
    }
    if (tid == 0) {
        s.ctr->n_primary = 0u;
        s.ctr->n_extra = 0u;
        s.ctr->n_blocks = 0u;
    }
}

// Per particle: activate the primary block and count the particle in its slab
// bucket.  Replaces touch_primary_blocks (sort.slang:50-67) and the primary
// half of update_block_particle_count (sort.slang:208-246).
template <int D> __global__ void k_touch(DevScene s) {
    const uint32_t lane = lane_id();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < s.n; base += stride) {
        const uint32_t i = base + lane;
        const bool valid = i < s.n;
        const unsigned mask = __ballot_sync(FULL_MASK, valid);
        if (!valid) continue;
        const float4 p = s.pm[i];
        const float x[3] = {p.x, p.y, p.z};
        const CellLoc<D> c = locate<D>(x, s.h);
        const uint32_t key = pack_key<D>(c.block);
        const uint32_t bucket = (uint32_t)c.local[D - 1];
        const unsigned peers = __match_any_sync(mask, key);
        const int leader = __ffs(peers) - 1;
        uint32_t slot = NONE;
        if ((int)lane == leader) {
            bool inserted = false;
            slot = hash_insert(s.hkeys, s.hcap, key, inserted, s.err);
            if (inserted) {
                const uint32_t j = atomicAdd(&s.ctr->n_primary, 1u);
                if (j < s.cap) {
                    s.blist_key[j] = key;
                    s.blist_slot[j] = slot;
                    atomicAdd(&s.hist[key >> 16], 1u);
                } else {
                    atomicOr(s.err, ERR_BLOCK_OVERFLOW);
                }
            }
        }
        slot = __shfl_sync(mask, slot, leader);
        const uint32_t bin = (slot == NONE) ? NONE : slot * Geo<D>::NPB + bucket;
        const unsigned peers2 = __match_any_sync(mask, bin);
        if (bin != NONE && (int)lane == __ffs(peers2) - 1) atomicAdd(&s.slot_counts[bin], (uint32_t)__popc(peers2));
        s.pslot[i] = bin;
    }
}

// Activates the +1 neighbours of every primary block, one thread per
// (block, neighbour).  Replaces touch_neighbor_blocks (sort.slang:75-92).
template <int D> __global__ void k_neighbors(DevScene s) {
    constexpr int NN = Geo<D>::NASSOC - 1;
    const uint32_t np = min(s.ctr->n_primary, s.cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < np * NN; t += stride) {
        const uint32_t j = t / NN;
        const int sidx = (int)(t % NN) + 1;
        int b[D], o[D];
        unpack_key<D>(s.blist_key[j], b);
        assoc_offset<D>(sidx, o);
        for (int k = 0; k < D; ++k) b[k] += o[k];
        const uint32_t key = pack_key<D>(b);
        bool inserted = false;
        const uint32_t slot = hash_insert(s.hkeys, s.hcap, key, inserted, s.err);
        if (inserted) {
            const uint32_t jj = atomicAdd(&s.ctr->n_extra, 1u);
            if (jj < s.cap) {
                s.blist2_key[jj] = key;
                s.blist2_slot[jj] = slot;
                atomicAdd(&s.hist[key >> 16], 1u);
            } else {
                atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            }
        }
    }
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

// Exclusive scan of the key histogram (one CTA) and the final block count.
template <int NT> __global__ void __launch_bounds__(NT) k_hist_scan(DevScene s) {
    __shared__ uint32_t total_sh;
    constexpr uint32_t PER = HIST_BINS / NT;
    uint32_t local = 0;
    const uint32_t b0 = threadIdx.x * PER;
    for (uint32_t k = 0; k < PER; ++k) local += s.hist[b0 + k];
    const uint32_t off = block_exclusive_scan<NT>(local, &total_sh);
    uint32_t run = off;
    for (uint32_t k = 0; k < PER; ++k) {
        s.hist_start[b0 + k] = run;
        run += s.hist[b0 + k];
    }
    if (threadIdx.x == 0) {
        const uint32_t total = min(s.ctr->n_primary, s.cap) + min(s.ctr->n_extra, s.cap);
        if (total > s.cap) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
        s.ctr->n_blocks = min(total, s.cap);
    }
}

// Groups the appended block keys by their top 16 bits.
__global__ void k_bin_scatter(DevScene s) {
    const uint32_t n1 = min(s.ctr->n_primary, s.cap), n2 = min(s.ctr->n_extra, s.cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n1 + n2; t += stride) {
        const uint32_t key = t < n1 ? s.blist_key[t] : s.blist2_key[t - n1];
        const uint32_t slot = t < n1 ? s.blist_slot[t] : s.blist2_slot[t - n1];
        const uint32_t b = key >> 16;
        const uint32_t pos = s.hist_start[b] + atomicAdd(&s.hist_fill[b], 1u);
        s.tmp_key[pos] = key;
        s.tmp_slot[pos] = slot;
    }
}

// Canonical rank = number of active keys smaller than this one.  Keys of one
// top-16-bit bin are compared against each other only.
__global__ void k_rank(DevScene s) {
    const uint32_t total = min(s.ctr->n_primary, s.cap) + min(s.ctr->n_extra, s.cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint32_t key = s.tmp_key[t];
        const uint32_t b = key >> 16;
        const uint32_t start = s.hist_start[b], cnt = s.hist[b];
        uint32_t r = start;
        for (uint32_t j = start; j < start + cnt; ++j) r += (s.tmp_key[j] < key) ? 1u : 0u;
        if (r < s.cap) {
            const uint32_t slot = s.tmp_slot[t];
            s.bkey[r] = key;
            s.bslot[r] = slot;
            s.hvals[slot] = r;
        }
    }
}

// Per block: neighbour ranks (update_nbh_block_ids, sort.slang:100-117) and
// zeroed nodes (reset, grid.slang:455-485).  Four blocks per 256 threads.
template <int D> __global__ void k_block_setup(DevScene s) {
    constexpr int NN = Geo<D>::NASSOC - 1;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nb * 64u; t += stride) {
        const uint32_t r = t >> 6, node = t & 63u;
        s.nodes[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (node < (uint32_t)NN) {
            int b[D], o[D];
            unpack_key<D>(s.bkey[r], b);
            assoc_offset<D>((int)node + 1, o);
            for (int k = 0; k < D; ++k) b[k] += o[k];
            const uint32_t slot = hash_find(s.hkeys, s.hcap, pack_key<D>(b));
            s.bnbh[r * NN + node] = (slot == NONE) ? NONE : s.hvals[slot];
        }
    }
}

// Exclusive scan of per-block primary totals into first_particle and the
// per-bucket insertion cursors (copy_particles_len_to_scan_value,
// prefix_sum, copy_scan_values_to_first_particles_and_prepare_for_finalize:
// sort.slang:248-302, prefix_sum.slang).  One CTA.
template <int D, int NT> __global__ void __launch_bounds__(NT) k_block_scan(DevScene s) {
    constexpr int NPB = Geo<D>::NPB;
    __shared__ uint32_t total_sh;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t per = (nb + NT - 1) / NT;
    const uint32_t r0 = threadIdx.x * per, r1 = min(r0 + per, nb);
    uint32_t local = 0;
    for (uint32_t r = r0; r < r1; ++r) {
        const uint32_t sl = s.bslot[r];
        for (int b = 0; b < NPB; ++b) local += s.slot_counts[sl * NPB + b];
    }
    uint32_t run = block_exclusive_scan<NT>(local, &total_sh);
    for (uint32_t r = r0; r < r1; ++r) {
        const uint32_t sl = s.bslot[r];
        s.bfirst[r] = run;
        uint32_t tot = 0;
        for (int b = 0; b < NPB; ++b) {
            s.bcur[r * NPB + b] = run + tot;
            tot += s.slot_counts[sl * NPB + b];
        }
        s.bnp[r] = tot;
        run += tot;
    }
}

// Per particle: claim its slot in the block's bucket (finalize_particles_sort,
// sort.slang:304-357, primaries only), warp-aggregated.
template <int D> __global__ void k_scatter(DevScene s) {
    const uint32_t lane = lane_id();
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < s.n; base += stride) {
        const uint32_t i = base + lane;
        const bool valid = i < s.n;
        const unsigned mask = __ballot_sync(FULL_MASK, valid);
        if (!valid) continue;
        const uint32_t bin = s.pslot[i];
        const unsigned peers = __match_any_sync(mask, bin);
        const int leader = __ffs(peers) - 1;
        uint32_t pos = NONE;
        if ((int)lane == leader && bin != NONE) {
            const uint32_t r = s.hvals[bin / Geo<D>::NPB];
            if (r != NONE) pos = atomicAdd(&s.bcur[r * Geo<D>::NPB + bin % Geo<D>::NPB], (uint32_t)__popc(peers));
        }
        pos = __shfl_sync(mask, pos, leader);
        if (pos != NONE) s.perm_tmp[pos + __popc(peers & lanemask_lt())] = i;
    }
}

// Orders each (block, bucket) range of the permutation by particle id: the
// canonical order.  Each element's position is its rank among the ids of its
// bucket (ids are unique).  Ranges up to CANON_SMEM ids are staged in shared
// memory; larger ones are ranked from global memory.
constexpr uint32_t CANON_SMEM = 4096;
template <int D, int NT> __global__ void __launch_bounds__(NT) k_canon(DevScene s) {
    constexpr int NPB = Geo<D>::NPB;
    __shared__ uint32_t ids[CANON_SMEM];
    __shared__ uint32_t bstart[NPB + 1];
    const uint32_t nb = s.ctr->n_blocks;
    for (uint32_t r = blockIdx.x; r < nb; r += gridDim.x) {
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        const uint32_t first = s.bfirst[r];
        if (threadIdx.x == 0) {
            const uint32_t sl = s.bslot[r];
            uint32_t run = 0;
            for (int b = 0; b < NPB; ++b) {
                bstart[b] = run;
                run += s.slot_counts[sl * NPB + b];
            }
            bstart[NPB] = run;
        }
        const bool in_smem = np <= CANON_SMEM;
        if (in_smem)
            for (uint32_t e = threadIdx.x; e < np; e += NT) ids[e] = s.perm_tmp[first + e];
        __syncthreads();
        const uint32_t *src = in_smem ? ids : s.perm_tmp + first;
        for (uint32_t e = threadIdx.x; e < np; e += NT) {
            int b = 0;
            while (b + 1 < NPB && e >= bstart[b + 1]) ++b;
            const uint32_t lo = bstart[b], hi = bstart[b + 1];
            const uint32_t id = src[e];
            uint32_t rank = 0;
            for (uint32_t j = lo; j < hi; ++j) rank += (src[j] < id) ? 1u : 0u;
            s.perm[first + lo + rank] = id;
        }
        __syncthreads();
    }
}

}  // namespace slosh
