// Grid reuse between substeps (single-scene context).
//
// The fused G2P/update writes every particle at its canonical position, so
// the next substep's storage is already sorted by the grid the particle was
// gathered from.  A particle moves at most one cell a substep (|v| <= h/dt),
// and in a typical substep only a small fraction of the particles changes
// cell.  G2P records each change as a per-cell count delta and a
// touched-cell bit, in the old and the new block (k_g2p_update).  The next
// substep keeps the grid -- block keys, ranks, neighbour ranks, hash map --
// when the set of active blocks cannot have changed:
//  - every particle that changed block landed in a block holding particles
//    (not in a neighbour-only block, not outside the grid),
//  - no block lost its last particle,
//  - no particle moved further than one cell on an axis.
// Otherwise the full build of grid_build.cuh runs (slosh's WgGrid::launch_sort,
// src/grid/grid.rs:78-238, rebuilds every substep).  When the grid is kept,
// only the per-cell counts, the offsets and the primary permutation change:
//   k_grid_reuse:  per block, the new per-cell counts (old + delta), their
//                  scan, the cells by decreasing count (touched blocks only),
//                  the identity previous rank; decides reuse or rebuild;
//                  the block offsets are scanned by CTA ranges here and
//                  completed in k_reuse_perm;
//   k_reuse_perm:  the permutation.  A cell no particle entered or left is a
//                  shifted range of storage; the touched cells are listed;
//   k_reuse_cells: a warp per touched cell gathers it from its own old range
//                  and the touched cells around it, ordered by original index.
// The result is the layout the full build produces from the same positions,
// bit for bit: blocks by key, cells slab-major, particles of a cell by
// original index.
#pragma once

#include "grid_build.cuh"

namespace slosh {

// Cell coordinates (inside its block) of cell index c: x + BW y (+ BW^2 z).
template <int D> __device__ __forceinline__ void cell_coords(uint32_t c, int *l) {
    if constexpr (D == 3) {
        l[0] = (int)(c & 3u);
        l[1] = (int)((c >> 2) & 3u);
        l[2] = (int)(c >> 4);
    } else {
        l[0] = (int)(c & 7u);
        l[1] = (int)(c >> 3);
    }
}

// CTAs of k_grid_reuse (at most): each counts a contiguous range of blocks.
constexpr uint32_t REUSE_MAX_CTAS = 4096;

// Warp per block of the previous substep, each CTA a contiguous range of
// blocks: new per-cell counts from G2P's deltas (clearing them), their
// in-block scan, the block total, the cells by decreasing count for P2G
// (touched blocks; the others keep theirs, which are relative to the
// block's first entry), the block's previous rank (the collision cache:
// itself).  Sets the rebuild flag when a block lost its last particle.
// The block offsets come out in two parts: each CTA scans its blocks'
// totals into offsets relative to its range (left in bfirst) and the last
// CTA to finish scans the CTAs' totals; k_reuse_perm adds the two.  That
// last CTA also reads the decision and, inside the substep graph, sets the
// conditional node that picks the full build or the reuse.
template <int D> __global__ void k_grid_reuse(DevScene s) {
    pdl_enter();
    __shared__ uint32_t cta_total;
    __shared__ bool last;
    const uint32_t nbp = min(s.ctr->last_n_blocks, s.cap);
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t per = (nbp + gridDim.x - 1) / gridDim.x;
    const uint32_t lo = min(blockIdx.x * per, nbp), hi = min(lo + per, nbp);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s.ctr->n_blocks = nbp;  // a full build recounts
        s.ctr->reuse_per_cta = per;
        s.ctr->n_touched = 0u;
    }
    for (uint32_t r = lo + warp; r < hi; r += nwarps) {
        const unsigned long long mask = s.touch[r];
        const size_t cb = (size_t)r * CELLS;
        const uint32_t q0 = s.prev_bcell[cb + 2 * lane], q1 = s.prev_bcell[cb + 2 * lane + 1];
        const uint32_t q2 = lane < 31 ? s.prev_bcell[cb + 2 * lane + 2] : s.prev_bnp[r];
        int c0 = (int)(q1 - q0), c1 = (int)(q2 - q1);
        if (mask != 0ull) {
            if ((mask >> (2 * lane)) & 1ull) {
                c0 += s.cell_delta[cb + 2 * lane];
                s.cell_delta[cb + 2 * lane] = 0;
            }
            if ((mask >> (2 * lane + 1)) & 1ull) {
                c1 += s.cell_delta[cb + 2 * lane + 1];
                s.cell_delta[cb + 2 * lane + 1] = 0;
            }
        }
        if (c0 < 0 || c1 < 0) {  // not a layout this grid can hold: rebuild
            s.ctr->rebuild[s.par] = 1u;
            c0 = max(c0, 0);
            c1 = max(c1, 0);
        }
        const uint32_t u0 = (uint32_t)c0, u1 = (uint32_t)c1, pair = u0 + u1;
        uint32_t incl = pair;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
            if (lane >= (uint32_t)off) incl += y;
        }
        const uint32_t ex = incl - pair;
        s.bcell[cb + 2 * lane] = ex;
        s.bcell[cb + 2 * lane + 1] = ex + u0;
        const uint32_t total = __shfl_sync(FULL_MASK, incl, 31);
        if (!s.use_partial) {  // the float-atomic P2G variant accumulates into zeroed nodes
            s.nodes[(size_t)r * 64 + 2 * lane] = make_float4(0.f, 0.f, 0.f, 0.f);
            s.nodes[(size_t)r * 64 + 2 * lane + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (lane == 0) {
            s.bnp[r] = total;
            s.cur_touch[r] = mask;
            s.bprev[r] = r;
            if (total == 0u && s.prev_bnp[r] != 0u) s.ctr->rebuild[s.par] = 1u;
        }
        if (mask != 0ull) {
            // cells by (count desc, cell asc), as k_block_setup orders them
            const uint32_t k0 = (min(u0, 0x3ffffffu) << 6) | (63u - 2u * lane);
            const uint32_t k1 = (min(u1, 0x3ffffffu) << 6) | (62u - 2u * lane);
            uint32_t r0 = 0, r1 = 0;
#pragma unroll 8
            for (int q = 0; q < 32; ++q) {
                const uint32_t a = __shfl_sync(FULL_MASK, k0, q), b = __shfl_sync(FULL_MASK, k1, q);
                r0 += (a > k0) + (b > k0);
                r1 += (a > k1) + (b > k1);
            }
            s.bord[cb + r0] = make_uint2((2u * lane) | (ex << 6), u0);
            s.bord[cb + r1] = make_uint2((2u * lane + 1u) | ((ex + u0) << 6), u1);
            if (lane == 0) s.touch[r] = 0ull;
        }
    }
    __syncthreads();  // the range's block totals are written
    if (warp == 0) {
        // offsets of the range's blocks relative to the range, and its total
        uint32_t carry = 0;
        for (uint32_t b0 = lo; b0 < hi; b0 += 32) {
            const uint32_t r = b0 + lane;
            const uint32_t v = r < hi ? s.bnp[r] : 0u;
            uint32_t incl = v;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
                if (lane >= (uint32_t)off) incl += y;
            }
            if (r < hi) s.bfirst[r] = carry + incl - v;
            carry += __shfl_sync(FULL_MASK, incl, 31);
        }
        if (lane == 0) {
            s.reuse_cta[blockIdx.x] = carry;
            cta_total = carry;
        }
    }
    // the decision, once every block is counted: each thread's stores are
    // made visible device-wide before its CTA counts itself done
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&s.ctr->reuse_done, 1u) == gridDim.x - 1u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: exclusive scan of the CTAs' totals, each thread a run of
    // consecutive CTAs (their loads independent, one round trip)
    {
        __shared__ uint32_t wsum[32];
        constexpr uint32_t RUN = 16;  // REUSE_MAX_CTAS / 256
        const uint32_t c0 = threadIdx.x * RUN;
        uint32_t v[RUN], sum = 0;
#pragma unroll
        for (uint32_t k = 0; k < RUN; ++k) {
            v[k] = c0 + k < gridDim.x ? *(volatile uint32_t *)&s.reuse_cta[c0 + k] : 0u;
            sum += v[k];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL_MASK, incl, off);
            if (lane >= (uint32_t)off) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t run = incl - sum;
        for (uint32_t w = 0; w < warp; ++w) run += wsum[w];
#pragma unroll
        for (uint32_t k = 0; k < RUN; ++k) {
            if (c0 + k < gridDim.x) s.reuse_cta[REUSE_MAX_CTAS + c0 + k] = run;
            run += v[k];
        }
    }
    if (threadIdx.x == 0) {
        const uint32_t rb = *(volatile uint32_t *)&s.ctr->rebuild[s.par];
        if (rb) s.ctr->n_rebuilds += 1u;
        else s.ctr->n_reuses += 1u;
        s.ctr->reuse_done = 0u;
        if (s.use_cond) cudaGraphSetConditional(s.cond, rb ? 1u : 0u);
    }
}

// The particles of touched cell c of block r in the reused grid: the old
// entries of the cell itself and of the touched cells around it (a particle
// moves at most one cell) whose stored position now lies in (r, c), written
// to the permutation at the cell's new range in original-index order.
// Candidates are evaluated 32 at a time, one per lane; ranks come from
// comparing original indices over all candidate chunks.  Writes at most
// `room` entries (the cell's new count) and returns the number of particles
// found.
template <int D>
__device__ uint32_t gather_touched_cell(const DevScene &s, uint32_t r, uint32_t c, const int (&bv)[D],
                                        uint32_t dst, uint32_t room) {
    constexpr int BW = Geo<D>::BW, NC = (D == 3) ? 27 : 9;
    const uint32_t lane = lane_id();
    const uint32_t key = s.bkey[r];
    int lc[D];
    cell_coords<D>(c, lc);
    // lane t < NC: neighbour cell t of (r, c), its old range when it can hold
    // a particle of (r, c) now: the cell itself, or a touched cell
    uint32_t os = 0, oc = 0;
    if (lane < (uint32_t)NC) {
        int g[D], nbk[D], nl[D];
        const int o[3] = {(int)(lane % 3u) - 1, (int)((lane / 3u) % 3u) - 1, (int)(lane / 9u) - 1};
        bool same = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            g[k] = bv[k] * BW + lc[k] + o[k];
            nbk[k] = g[k] >> (BW == 4 ? 2 : 3);
            nl[k] = g[k] & (BW - 1);
            same = same && nbk[k] == bv[k];
        }
        uint32_t rn = r;
        if (!same) {
            const uint32_t slot = hash_find(s.prev_hkeys, s.hcap, pack_key<D>(nbk));
            rn = slot == NONE ? NONE : rank_of(s.prev_hvals[slot]);
        }
        const uint32_t cn = cell_index<D>(nl);
        const bool centre = lane == (uint32_t)(NC / 2);
        if (rn != NONE && rn < s.cap && (centre || ((s.cur_touch[rn] >> cn) & 1ull))) {
            const size_t cb = (size_t)rn * CELLS;
            const uint32_t lo = s.prev_bcell[cb + cn];
            const uint32_t hi = cn < CELLS - 1 ? s.prev_bcell[cb + cn + 1] : s.prev_bnp[rn];
            os = s.prev_bfirst[rn] + lo;
            oc = hi > lo ? hi - lo : 0u;
        }
    }
    uint32_t start = oc;  // exclusive scan of the candidate counts
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL_MASK, start, off);
        if (lane >= (uint32_t)off) start += y;
    }
    const uint32_t total = __shfl_sync(FULL_MASK, start, 31);
    start -= oc;
    // candidate t: storage index, and whether it is a particle of (r, c)
    auto candidate = [&](uint32_t t, uint32_t &i, uint32_t &oid) -> bool {
        uint32_t j = 0;
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (__shfl_sync(FULL_MASK, start, q) <= t) j = (uint32_t)q;
        const uint32_t sj = __shfl_sync(FULL_MASK, start, (int)j), oj = __shfl_sync(FULL_MASK, os, (int)j);
        if (t >= total) return false;
        i = oj + (t - sj);
        if (i >= s.count) return false;
        const float4 p = s.pm[i];
        const float x[3] = {p.x, p.y, p.z};
        const CellLoc<D> cl = locate<D>(x, s.h, s.inv_h, s.h_pow2);
        oid = s.oid[i];
        return pack_key<D>(cl.block) == key && cell_index<D>(cl.local) == c;
    };
    uint32_t found = 0;
    for (uint32_t a0 = 0; a0 < total; a0 += 32) {
        uint32_t i = 0, oid = 0;
        const bool mine = candidate(a0 + lane, i, oid);
        uint32_t rank = 0;
        for (uint32_t b0 = 0; b0 < total; b0 += 32) {
            uint32_t ib = 0, ob = 0;
            const bool mb = (b0 == a0) ? mine : candidate(b0 + lane, ib, ob);
            if (b0 == a0) ob = oid;
            const unsigned mm = __ballot_sync(FULL_MASK, mb);
#pragma unroll 8
            for (int q = 0; q < 32; ++q) {
                const uint32_t oq = __shfl_sync(FULL_MASK, ob, q);
                rank += ((mm >> q) & 1u) && oq < oid ? 1u : 0u;
            }
        }
        if (mine && rank < room) s.perm[dst + rank] = i;
        found += (uint32_t)__popc(__ballot_sync(FULL_MASK, mine));
    }
    return found;
}

// The reused grid's primary permutation (warp per block): each block's
// offset completed from k_grid_reuse's two partial scans, its untouched
// cells written as shifted ranges and its touched cells listed for
// k_reuse_cells; the previous map becomes this substep's; the transfer
// kernels' block queues restart.
template <int D> __global__ void k_reuse_perm(DevScene s) {
    pdl_enter();
    if (s.ctr->rebuild[s.par]) return;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    for (uint32_t q = tid; q < s.hcap; q += stride) {
        s.hkeys[q] = s.prev_hkeys[q];
        s.hvals[q] = s.prev_hvals[q];
    }
    if (tid == 0) {
        s.ctr->p2g_next = 0u;
        s.ctr->g2p_next = 0u;
    }
    const uint32_t nb = s.ctr->n_blocks, per = max(s.ctr->reuse_per_cta, 1u);
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nb; r += warps) {
        // the block's offset: k_grid_reuse's range-relative offset plus its range's base
        const uint32_t first = s.bfirst[r] + s.reuse_cta[REUSE_MAX_CTAS + r / per];
        const uint32_t pf = s.prev_bfirst[r], np = s.bnp[r];
        __syncwarp();  // every lane has read the relative offset
        const unsigned long long mask = s.cur_touch[r];
        // the transfer kernels index an untouched block's particles from
        // its storage start instead of loading the permutation
        if (lane == 0) {
            s.bfirst[r] = first;
            s.bsrc[r] = (mask == 0ull && (size_t)pf + np <= s.count) ? pf : NONE;
        }
        if ((size_t)first + np > s.count) {
            if (lane == 0) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            continue;
        }
        if (mask == 0ull) {  // the block's particles are a shifted range
            for (uint32_t e = lane; e < np; e += 32) s.perm[first + e] = pf + e;
            continue;
        }
        const size_t cb = (size_t)r * CELLS;
        // untouched cells: shifted ranges, two cells a lane
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t c = 2u * lane + (uint32_t)hh;
            if ((mask >> c) & 1ull) continue;
            const uint32_t lo = s.bcell[cb + c], hi = c < CELLS - 1 ? s.bcell[cb + c + 1] : np;
            const uint32_t plo = pf + s.prev_bcell[cb + c];
            for (uint32_t k = lo; k < hi; ++k) s.perm[first + k] = plo + (k - lo);
        }
        // touched cells: listed for k_reuse_cells, which gathers them a warp each
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&s.ctr->n_touched, (uint32_t)__popcll(mask));
        base = __shfl_sync(FULL_MASK, base, 0);
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const uint32_t c = 2u * lane + (uint32_t)hh;
            if ((mask >> c) & 1ull)
                s.touched_cells[base + (uint32_t)__popcll(mask & ((1ull << c) - 1ull))] = (r << 6) | c;
        }
    }
}

// The touched cells of a kept grid, one warp each (their gathers are chains
// of dependent loads, so they run side by side rather than block by block).
template <int D> __global__ void k_reuse_cells(DevScene s) {
    pdl_enter();
    if (s.ctr->rebuild[s.par]) return;
    const uint32_t nt = s.ctr->n_touched;
    const uint32_t lane = lane_id();
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < nt; t += warps) {
        const uint32_t e = s.touched_cells[t];
        const uint32_t r = e >> 6, c = e & 63u;
        const uint32_t first = s.bfirst[r], np = s.bnp[r];
        const size_t cb = (size_t)r * CELLS;
        const uint32_t lo = s.bcell[cb + c], hi = c < CELLS - 1 ? s.bcell[cb + c + 1] : np;
        if ((size_t)first + np > s.count || hi < lo || hi > np) {
            if (lane == 0) atomicOr(s.err, ERR_GRID_REUSE);
            continue;
        }
        int bv[D];
        unpack_key<D>(s.bkey[r], bv);
        const uint32_t got = gather_touched_cell<D>(s, r, c, bv, first + lo, hi - lo);
        if (got != hi - lo && lane == 0) atomicOr(s.err, ERR_GRID_REUSE);
    }
}

}  // namespace slosh
