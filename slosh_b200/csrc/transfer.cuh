// Particle/grid transfer kernels of one substep:
//   k_p2g          APIC/MLS particle-to-grid scatter
//   k_grid_update  momentum -> velocity, gravity, clamping, collider BCs
//   k_g2p_update   grid-to-particle gather fused with the particle update
//   k_rigid        rigid-body pose integration
#pragma once

#include "grid_build.cuh"
#include "models.cuh"
#include "scene.cuh"
#include "trimesh.cuh"

namespace slosh {

// Coordinates of tile node t (tile edge TW) and the rank + local node id of
// the grid block that owns it (the block itself or one of its +1
// neighbours, in slosh's associated-block order).
template <int D>
__device__ __forceinline__ bool tile_node_owner(const DevScene &s, uint32_t r, int t, uint32_t &rank, uint32_t &local) {
    constexpr int TW = Geo<D>::TW, BW = Geo<D>::BW, NN = Geo<D>::NASSOC - 1;
    int c[D];
    c[0] = t % TW;
    if constexpr (D == 3) {
        c[1] = (t / TW) % TW;
        c[2] = t / (TW * TW);
    } else {
        c[1] = t / TW;
    }
    int oct = 0;
    uint32_t loc = 0, mul = 1;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int o = c[k] >= BW ? 1 : 0;
        oct = oct * 2 + o;
        loc += (uint32_t)(c[k] - o * BW) * mul;
        mul *= BW;
    }
    rank = (oct == 0) ? r : s.bnbh[r * NN + oct - 1];
    local = loc;
    return rank != NONE;
}

// Adds one particle to a thread's stencil sums.  The thread owns cell `assoc`
// (its base node, in cells) and one slab of the 3^D stencil: 3D the nodes
// (sx, sy, slab), 2D (sx, slab).  p = (x, m), vv = (v, C22), cq = C rows,
// fdt = the pending force impulse (zeros when none).  The weights use
// -d0 / h = -d0 * (1/h) like slosh's p2g (dpt * inv_cell_width) with
// d0 = assoc h - x exact from the sorted cell.  Returns false for a
// particle outside the cell (packed-key aliasing far outside the key range).
template <int D>
__device__ __forceinline__ bool p2g_particle(const float4 p, const float4 vv, const float4 *cq, const float (&fdt)[3],
                                             const float (&assoc)[D], float h, float inv_h, int slab,
                                             float4 (&acc)[D == 3 ? 9 : 3]) {
    const float x[3] = {p.x, p.y, p.z};
    const float m = p.w;
    float d0[D], w[D][3], fs = 0.f;
    bool in_cell = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        d0[k] = assoc[k] * h - x[k];
        const float f = -d0[k] * inv_h;
        in_cell = in_cell && f >= 0.49f && f <= 1.51f;
        if (k < D - 1) bspline_weights(f, w[k]);
        else fs = f;
    }
    if (!in_cell) return false;
    // Along the slab axis the lane needs its own slab's weight only, in
    // bspline_weights' arithmetic: (0.5 t) t with t = f - 1.5 (= -(1.5 - f)
    // exactly) or t = f - 0.5, and 0.75 - t t with t = f - 1.  The
    // coefficients depend on the slab alone, so they stay out of the loop.
    const float sb = slab == 0 ? 1.5f : (slab == 1 ? 1.0f : 0.5f);
    const float sa = slab == 1 ? -1.0f : 0.5f, sc = slab == 1 ? 0.75f : 0.0f;
    const float ts = fs - sb;
    const float wsl = fmaf(sa * ts, ts, sc);
    float bm[D], hc[D][D], Cm[D][D];
    mat_from<D>(cq, vv.w, Cm);
    const float vel[3] = {vv.x, vv.y, vv.z};
#pragma unroll
    for (int jj = 0; jj < D; ++jj) {
        float q = vel[jj] * m + fdt[jj];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float c = Cm[jj][k];
            q += c * d0[k];
            hc[k][jj] = h * c;
        }
        bm[jj] = q;
    }
    const float fsl = (float)slab;
    if constexpr (D == 3) {
        // Paired FP32 arithmetic (sm_100 f32x2 FMA): the node value
        // (b + s h C, m) is carried as the pairs (x, y) and (z, m); the m
        // lane's offsets are zero, so it stays m exactly.  Offset 0 adds
        // nothing to a finite value and is skipped.
        const float wz = wsl;
        const float2 hx01 = make_float2(hc[0][0], hc[0][1]), hx2 = make_float2(hc[0][2], 0.f);
        const float2 hy01 = make_float2(hc[1][0], hc[1][1]), hy2 = make_float2(hc[1][2], 0.f);
        const float2 fs2 = make_float2(fsl, fsl);
        const float2 mz01 = __ffma2_rn(fs2, make_float2(hc[2][0], hc[2][1]), make_float2(bm[0], bm[1]));
        const float2 mz2 = __ffma2_rn(fs2, make_float2(hc[2][2], 0.f), make_float2(bm[2], m));
#pragma unroll
        for (int sy = 0; sy < 3; ++sy) {
            const float wyz = w[1][sy] * wz;
            float2 my01 = mz01, my2 = mz2;
            if (sy > 0) {
                const float2 sy2 = make_float2((float)sy, (float)sy);
                my01 = __ffma2_rn(sy2, hy01, mz01);
                my2 = __ffma2_rn(sy2, hy2, mz2);
            }
#pragma unroll
            for (int sx = 0; sx < 3; ++sx) {
                float2 t01 = my01, t2 = my2;
                if (sx > 0) {
                    const float2 sx2 = make_float2((float)sx, (float)sx);
                    t01 = __ffma2_rn(sx2, hx01, my01);
                    t2 = __ffma2_rn(sx2, hx2, my2);
                }
                const float wt = w[0][sx] * wyz;
                const float2 wt2 = make_float2(wt, wt);
                float4 &a = acc[sx + 3 * sy];
                const float2 axy = __ffma2_rn(wt2, t01, make_float2(a.x, a.y));
                const float2 azw = __ffma2_rn(wt2, t2, make_float2(a.z, a.w));
                a = make_float4(axy.x, axy.y, azw.x, azw.y);
            }
        }
    } else {
        const float wy = wsl;
        const float my0 = bm[0] + fsl * hc[1][0], my1 = bm[1] + fsl * hc[1][1];
#pragma unroll
        for (int sx = 0; sx < 3; ++sx) {
            const float wt = w[0][sx] * wy;
            float4 &a = acc[sx];
            a.x += wt * (my0 + (float)sx * hc[0][0]);
            a.y += wt * (my1 + (float)sx * hc[0][1]);
            a.w += wt * m;
        }
    }
    return true;
}

// Particle-to-grid, one warp per active block (P2G_WARPS warps a CTA, each
// on its own blocks, no CTA barrier).
//
// The block's 64 cells x 3 stencil slabs are 192 (cell, slab) items, taken
// in bord's order (cells by decreasing particle count) in 6 passes of 32:
// the lanes of a pass hold cells of similar count, so they finish their
// particle loops together, and a pass whose first (largest) cell is empty
// ends the block.  A lane owns cell c and the 9 (3D) or 3 (2D) stencil nodes
// of one slab, reads the particles of c -- contiguous in the canonical order
// -- double-buffered through cp.async, and sums its nodes in registers.
//
// Reduction, fixed order (the substep is bit-reproducible): each slab has a
// tile of the nodes its cells reach (3D: 6 x 6 x 4, z relative to the slab;
// 2D: 10 x 8).  After each pass the lanes add their 9 (3) sums, one stencil
// offset at a time; for a fixed offset the lanes of a pass hit distinct
// nodes (one item per (cell, slab)), so only __syncwarp is needed.  The
// slab tiles are then summed in slab order into the block's (block + 2)^D
// tile, stored to its own `partial` slot; k_grid_update adds the (up to 2^D)
// tiles overlapping each node in a fixed order.
constexpr int P2G_WARPS = 4;
template <int D> struct SlabTile;
template <> struct SlabTile<3> {
    static constexpr int PY = 6, PZ = 36, SIZE = 144;  // x 6, y 6, z 4
};
template <> struct SlabTile<2> {
    static constexpr int PY = 10, PZ = 0, SIZE = 80;  // x 10, y 8
};

// FORCE: the substep adds the particles' pending force impulses (the first
// substep after they were set); the other substeps compile without them.
// NBUF: particles of a cell staged ahead through cp.async (batches tune it;
// the results do not depend on it).
// Shared memory of k_p2g's CTA (P2G_WARPS warps): each warp's three slab
// tiles and its staged particles.  Staging: the particles of a pass's cells
// (at most CS = 12: 32 lanes, 3 slab lanes a cell, the first and last cell
// possibly shared with the neighbouring passes) in NBUF buffers; particle
// k + NBUF - 1 of every cell is copied while particle k is summed.
template <int D, int NBUF, int W = P2G_WARPS> struct P2gSmem {
    static constexpr int CS = 12;
    float4 stile[W][3 * SlabTile<D>::SIZE];
    float4 sp_pm[W][NBUF][CS];
    float4 sp_vv[W][NBUF][CS];
    float4 sp_cq[W][NBUF][MQ<D>::Q][CS];
};

template <int D, bool B = false, bool FORCE = false, int NBUF = 3, int W = P2G_WARPS>
__device__ __forceinline__ void p2g_body(const DevScene &s, P2gSmem<D, NBUF, W> &sm) {
    constexpr int TW = Geo<D>::TW, TILE = Geo<D>::TILE, BW = Geo<D>::BW;
    constexpr int NACC = (D == 3) ? 9 : 3;
    constexpr int PY = SlabTile<D>::PY, PZ = SlabTile<D>::PZ, SSZ = SlabTile<D>::SIZE;
    constexpr int Q = MQ<D>::Q;
    constexpr int CS = P2gSmem<D, NBUF, W>::CS;
    static_assert(NBUF >= 2 && NBUF <= 4, "staging depth 2 to 4");
    auto &stile = sm.stile;
    auto &sp_pm = sm.sp_pm;
    auto &sp_vv = sm.sp_vv;
    auto &sp_cq = sm.sp_cq;
    // storage index of the current block's first particle when its
    // particles are one shifted range of storage, else NONE (the
    // permutation is read)
    uint32_t src = NONE;
    const bool use_src = !B && s.reuse && s.bsrc != nullptr;
    const uint32_t nb = s.ctr->n_blocks;
    const size_t n = s.n;
    const uint32_t lane = lane_id(), wl = threadIdx.x >> 5;
    float4 *tiles = stile[wl];
    // One pass of block r: 32 (cell, slab) items (`ord` their cells)
    // summed into this warp's slab tiles.  Returns false when the pass's
    // cells are empty (and so are the later passes').  With `next`, `ord`
    // is reloaded with the next pass's cells once this pass's are read.
    auto run_pass = [&](uint32_t r, uint32_t first, const int (&bv)[D], float h, float inv_h, uint32_t pass,
                        uint2 &ord, bool next) -> bool {
        const uint32_t item = 32u * pass + lane;
        const int slab = (int)(item % 3u);
        const uint32_t lo = ord.x >> 6, hi = lo + ord.y;
        const int cell = (int)(ord.x & 63u);
        if (__shfl_sync(FULL_MASK, ord.y, 0) == 0u) return false;
        if (next) ord = s.bord[(size_t)r * CELLS + (item + 32u) / 3u];
        int ca[D];
        if constexpr (D == 3) {
            ca[0] = cell & 3;
            ca[1] = (cell >> 2) & 3;
            ca[2] = cell >> 4;
        } else {
            ca[0] = cell & 7;
            ca[1] = cell >> 3;
        }
        float assoc[D];
#pragma unroll
        for (int k = 0; k < D; ++k) assoc[k] = (float)(bv[k] * BW + ca[k]);
        float4 acc[NACC];
#pragma unroll
        for (int k = 0; k < NACC; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        // The first lane of each cell in this pass (its slab-0 lane, or lane
        // 0 for a cell begun in the previous pass) copies the cell's
        // particles into the cell's staging slot; the three slab lanes of a
        // cell read the same slot.  The lanes step through particle k
        // together (k up to the pass's largest count, lane 0's), so the warp
        // can sync around the copies.
        const uint32_t cnt = hi - lo, kmax = __shfl_sync(FULL_MASK, cnt, 0);
        const uint32_t cs = item / 3u - (32u * pass) / 3u;
        const bool loader = slab == 0 || lane == 0;
        auto stage = [&](uint32_t k, uint32_t i) {
            if (loader && k < cnt) {
                const int b = (int)(k % NBUF);
                cp_async16(&sp_pm[wl][b][cs], &s.pm[i]);
                cp_async16(&sp_vv[wl][b][cs], &s.vv[i]);
#pragma unroll
                for (int q = 0; q < Q; ++q) cp_async16(&sp_cq[wl][b][q][cs], &s.cq[q * n + i]);
            }
            cp_async_commit();
        };
        auto index = [&](uint32_t k) {
            return (loader && k < cnt) ? (src != NONE ? src + lo + k : s.perm[first + lo + k]) : 0u;
        };
#pragma unroll
        for (uint32_t k = 0; k + 1 < (uint32_t)NBUF; ++k) stage(k, index(k));
        uint32_t i_next = index(NBUF - 1u);  // loaded one iteration before its copies
        for (uint32_t k = 0; k < kmax; ++k) {
            stage(k + NBUF - 1u, i_next);
            i_next = index(k + NBUF);
            cp_async_wait<NBUF - 1>();
            __syncwarp();  // the loaders' copies of particle k have landed
            if (k < cnt) {
                const int b = (int)(k % NBUF);
                float fdt[3] = {0.f, 0.f, 0.f};
                if constexpr (FORCE) {
                    const uint32_t i = src != NONE ? src + lo + k : s.perm[first + lo + k];
#pragma unroll
                    for (int d = 0; d < D; ++d) fdt[d] = s.fdt[d * n + i];
                }
                float4 cv[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) cv[q] = sp_cq[wl][b][q][cs];
                if (!p2g_particle<D>(sp_pm[wl][b][cs], sp_vv[wl][b][cs], cv, fdt, assoc, h, inv_h, slab, acc))
                    atomicOr(s.err, ERR_KEY_RANGE);
            }
            __syncwarp();  // slot k % NBUF is refilled by the next iteration's copies
        }
        cp_async_wait<0>();
        __syncwarp();
        // node (cell + stencil offset) in the slab's tile, whose slab-axis
        // coordinate is relative to the slab: 3D z - slab = ca[2], 2D
        // y - slab = ca[1]
        float4 *pt = tiles + slab * SSZ;
#pragma unroll
        for (int k = 0; k < NACC; ++k) {
            const int sx = k % 3;
            int idx;
            if constexpr (D == 3) idx = (ca[0] + sx) + PY * (ca[1] + k / 3) + PZ * ca[2];
            else idx = (ca[0] + sx) + PY * ca[1];
            float4 v = pt[idx];
            v.x += acc[k].x;
            v.y += acc[k].y;
            v.z += acc[k].z;
            v.w += acc[k].w;
            pt[idx] = v;
            __syncwarp();
        }
        return true;
    };
    // Node t of the block's (block + 2)^D tile: the sum of the slab tiles of
    // warps [w0, w1) in warp then slab order.
    auto tile_node = [&](int t, uint32_t w0, uint32_t w1) {
        int tc[D];
        tc[0] = t % TW;
        if constexpr (D == 3) {
            tc[1] = (t / TW) % TW;
            tc[2] = t / (TW * TW);
        } else {
            tc[1] = t / TW;
        }
        const int along = tc[D - 1];  // slab axis: z in 3D, y in 2D
        float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t w = w0; w < w1; ++w)
#pragma unroll
            for (int sl = 0; sl < 3; ++sl) {
                const int rel = along - sl;  // node plane within slab sl's tile
                if (rel < 0 || rel >= BW) continue;
                const int lay = (D == 3) ? tc[0] + PY * tc[1] + PZ * rel : tc[0] + PY * rel;
                const float4 v = stile[w][sl * SSZ + lay];
                sum.x += v.x;
                sum.y += v.y;
                sum.z += v.z;
                sum.w += v.w;
            }
        return sum;
    };
    auto block_setup = [&](uint32_t r, float &h, float &inv_h, int (&bv)[D]) {
        if constexpr (B) {
            h = s.scenes[s.bscene[r]].h;
            inv_h = 1.0f / h;
        }
        unpack_key<D>(s.bkey[r], bv);
        for (uint32_t q = lane; q < 3u * SSZ; q += 32u) tiles[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    };
    if (!B && nb < s.p2g_coop_below) {
        // Few blocks (a small scene): the CTA's W warps share a block, warp w
        // taking passes w, w + W, ..., and the block's tile sums the warps'
        // slab tiles in warp order.
        __shared__ uint32_t coop_r;
        for (;;) {
            __syncthreads();  // the previous block's tile sum has read the slab tiles
            if (threadIdx.x == 0) {
                const uint32_t q = atomicAdd(&s.ctr->p2g_next, 1u);
                coop_r = q < nb ? (s.p2g_heavy_first ? s.qorder[q] : q) : nb;
            }
            __syncthreads();
            const uint32_t r = coop_r;
            if (r >= nb) break;
            const uint32_t np = s.bnp[r];
            if (np == 0) continue;
            const uint32_t first = s.bfirst[r];
            if (first + np > s.n) {
                if (threadIdx.x == 0) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
                continue;
            }
            float h = s.h, inv_h = 1.0f / s.h;
            int bv[D];
            block_setup(r, h, inv_h, bv);
            src = use_src ? s.bsrc[r] : NONE;
            for (uint32_t pass = wl; pass < 6u; pass += W) {
                uint2 ord = s.bord[(size_t)r * CELLS + (32u * pass + lane) / 3u];
                if (!run_pass(r, first, bv, h, inv_h, pass, ord, false)) break;
            }
            __syncthreads();
            for (int t = (int)threadIdx.x; t < TILE; t += 32 * W)
                s.partial[(size_t)r * TILE + t] = tile_node(t, 0, W);
        }
        return;
    }
    // One warp a block.  Blocks are taken from a queue (one atomic a
    // block), so warps that get light blocks take more of them.
    auto next_block = [&]() {
        uint32_t r = 0;
        if (lane == 0) {
            const uint32_t q = atomicAdd(&s.ctr->p2g_next, 1u);
            r = q < nb ? (s.p2g_heavy_first ? s.qorder[q] : q) : nb;
        }
        return __shfl_sync(FULL_MASK, r, 0);
    };
    for (uint32_t r = next_block(); r < nb; r = next_block()) {
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        const uint32_t first = s.bfirst[r];
        if (first + np > s.n) {  // only after an earlier overflow left stale counts
            if (lane == 0) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            continue;
        }
        float h = s.h, inv_h = 1.0f / s.h;
        int bv[D];
        block_setup(r, h, inv_h, bv);
        src = use_src ? s.bsrc[r] : NONE;
        uint2 ord = s.bord[(size_t)r * CELLS + lane / 3u];
        for (uint32_t pass = 0; pass < 6u; ++pass)
            if (!run_pass(r, first, bv, h, inv_h, pass, ord, pass < 5u)) break;  // later passes hold empty cells
        __syncwarp();
        for (int t = (int)lane; t < TILE; t += 32) s.partial[(size_t)r * TILE + t] = tile_node(t, wl, wl + 1);
        __syncwarp();
    }
}
template <int D, bool B = false, bool FORCE = false, int NBUF = 3>
__global__ void __launch_bounds__(32 * P2G_WARPS, 5) k_p2g(DevScene s) {
    pdl_enter();
    __shared__ P2gSmem<D, NBUF> sm;
    p2g_body<D, B, FORCE, NBUF>(s, sm);
}

// Small scenes: CTAs of P2G_WIDE_WARPS warps, which take one pass each of a
// shared block (3 CTAs an SM by registers); their shared memory (54 KB in
// 3D) is dynamic.
constexpr int P2G_WIDE_WARPS = 6;
template <int D, bool FORCE>
__global__ void __launch_bounds__(32 * P2G_WIDE_WARPS, 3) k_p2g_wide(DevScene s) {
    pdl_enter();
    extern __shared__ __align__(16) unsigned char psm[];
    p2g_body<D, false, FORCE, 3, P2G_WIDE_WARPS>(s, *reinterpret_cast<P2gSmem<D, 3, P2G_WIDE_WARPS> *>(psm));
}

// Particle-to-grid with float atomics, kept for comparison (SLOSH_P2G=direct):
// one CTA of 192 threads a block, thread (cell, slab) sums its nodes like
// k_p2g and adds them through shared-memory atomics into the block's tile,
// then 16-byte global atomics into the nodes.  Not bit-reproducible.
constexpr int P2G_ATOMIC_THREADS = 192;
template <int D> __global__ void __launch_bounds__(P2G_ATOMIC_THREADS, 4) k_p2g_atomic(DevScene s) {
    pdl_enter();
    constexpr int TW = Geo<D>::TW, TILE = Geo<D>::TILE, BW = Geo<D>::BW;
    constexpr int NACC = (D == 3) ? 9 : 3;
    constexpr int NT = P2G_ATOMIC_THREADS;
    constexpr int Q = MQ<D>::Q;
    __shared__ float tile[4][TILE];
    __shared__ float4 sp_pm[2][NT];
    __shared__ float4 sp_vv[2][NT];
    __shared__ float4 sp_cq[2][Q][NT];
    const uint32_t nb = s.ctr->n_blocks;
    const float h = s.h, inv_h = 1.0f / s.h;
    const size_t n = s.n;
    const uint32_t tid = threadIdx.x;
    const int mycell = (int)(tid & 63u), myslab = (int)(tid >> 6);
    int ca[D];
    if constexpr (D == 3) {
        ca[0] = mycell & 3;
        ca[1] = (mycell >> 2) & 3;
        ca[2] = mycell >> 4;
    } else {
        ca[0] = mycell & 7;
        ca[1] = mycell >> 3;
    }
    for (uint32_t r = blockIdx.x; r < nb; r += gridDim.x) {
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        const uint32_t first = s.bfirst[r];
        if (first + np > s.n) {
            if (tid == 0) atomicOr(s.err, ERR_BLOCK_OVERFLOW);
            continue;
        }
        for (int t = tid; t < 4 * TILE; t += NT) (&tile[0][0])[t] = 0.f;
        int bv[D];
        unpack_key<D>(s.bkey[r], bv);
        const uint32_t lo = s.bcell[(size_t)r * CELLS + mycell];
        const uint32_t hi = (mycell < 63) ? s.bcell[(size_t)r * CELLS + mycell + 1] : np;
        float assoc[D];
#pragma unroll
        for (int k = 0; k < D; ++k) assoc[k] = (float)(bv[k] * BW + ca[k]);
        float4 acc[NACC];
#pragma unroll
        for (int k = 0; k < NACC; ++k) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        auto stage = [&](int b, uint32_t j) {
            if (j < hi) {
                const uint32_t i = s.perm[first + j];
                cp_async16(&sp_pm[b][tid], &s.pm[i]);
                cp_async16(&sp_vv[b][tid], &s.vv[i]);
#pragma unroll
                for (int q = 0; q < Q; ++q) cp_async16(&sp_cq[b][q][tid], &s.cq[q * n + i]);
            }
            cp_async_commit();
        };
        stage(0, lo);
        __syncthreads();
        int buf = 0;
        for (uint32_t j = lo; j < hi; ++j, buf ^= 1) {
            stage(buf ^ 1, j + 1);
            cp_async_wait<1>();
            float fdt[3] = {0.f, 0.f, 0.f};
            if (s.force_pending) {
                const uint32_t i = s.perm[first + j];
#pragma unroll
                for (int k = 0; k < D; ++k) fdt[k] = s.fdt[k * n + i];
            }
            float4 cv[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) cv[q] = sp_cq[buf][q][tid];
            if (!p2g_particle<D>(sp_pm[buf][tid], sp_vv[buf][tid], cv, fdt, assoc, h, inv_h, myslab, acc))
                atomicOr(s.err, ERR_KEY_RANGE);
        }
        cp_async_wait<0>();
        if (hi > lo) {
#pragma unroll
            for (int k = 0; k < NACC; ++k) {
                const int sx = k % 3, sy = (D == 3) ? k / 3 : myslab, sz = (D == 3) ? myslab : 0;
                int idx = (ca[0] + sx) + TW * (ca[1] + sy);
                if constexpr (D == 3) idx += TW * TW * (ca[2] + sz);
                atomicAdd(&tile[0][idx], acc[k].x);
                atomicAdd(&tile[1][idx], acc[k].y);
                if constexpr (D == 3) atomicAdd(&tile[2][idx], acc[k].z);
                atomicAdd(&tile[3][idx], acc[k].w);
            }
        }
        __syncthreads();
        for (int t = tid; t < TILE; t += NT) {
            const float4 val = make_float4(tile[0][t], tile[1][t], tile[2][t], tile[3][t]);
            if (val.x == 0.f && val.y == 0.f && val.z == 0.f && val.w == 0.f) continue;
            uint32_t rank, local;
            if (!tile_node_owner<D>(s, r, t, rank, local)) continue;
            atomicAdd(&s.nodes[(size_t)rank * 64u + local], val);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Colliders: Sim3/Sim2 poses, ball and cuboid projections, collide() and the
// boundary-condition projection.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void quat_rotate(const float *q, const float *v, float *out) {
    const float t0 = 2.f * (q[1] * v[2] - q[2] * v[1]);
    const float t1 = 2.f * (q[2] * v[0] - q[0] * v[2]);
    const float t2 = 2.f * (q[0] * v[1] - q[1] * v[0]);
    out[0] = v[0] + q[3] * t0 + (q[1] * t2 - q[2] * t1);
    out[1] = v[1] + q[3] * t1 + (q[2] * t0 - q[0] * t2);
    out[2] = v[2] + q[3] * t2 + (q[0] * t1 - q[1] * t0);
}

template <int D> __device__ __forceinline__ void pose_mul_pt(const DevBody &b, const float *p, float *out) {
    if constexpr (D == 3) {
        const float sp[3] = {p[0] * b.scale, p[1] * b.scale, p[2] * b.scale};
        float r[3];
        quat_rotate(b.rot, sp, r);
        for (int i = 0; i < 3; ++i) out[i] = r[i] + b.tra[i];
    } else {
        const float sp0 = p[0] * b.scale, sp1 = p[1] * b.scale;
        out[0] = b.rot[0] * sp0 - b.rot[1] * sp1 + b.tra[0];
        out[1] = b.rot[1] * sp0 + b.rot[0] * sp1 + b.tra[1];
    }
}

template <int D> __device__ __forceinline__ void pose_inv_mul_pt(const DevBody &b, const float *p, float *out) {
    if constexpr (D == 3) {
        const float d[3] = {p[0] - b.tra[0], p[1] - b.tra[1], p[2] - b.tra[2]};
        const float qi[4] = {-b.rot[0], -b.rot[1], -b.rot[2], b.rot[3]};
        float r[3];
        quat_rotate(qi, d, r);
        for (int i = 0; i < 3; ++i) out[i] = r[i] / b.scale;
    } else {
        const float d0 = p[0] - b.tra[0], d1 = p[1] - b.tra[1];
        out[0] = (b.rot[0] * d0 + b.rot[1] * d1) / b.scale;
        out[1] = (-b.rot[1] * d0 + b.rot[0] * d1) / b.scale;
    }
}

// Closest point of the segment a-b (shaders/slosh/rbd/shapes/segment.slang:9-28):
// an end point in its Voronoi region, else the orthogonal projection.
template <int D> __device__ __forceinline__ void segment_closest(const float *a, const float *b, const float *p,
                                                                 float *q) {
    float ab[D], ap_ab = 0.f, ab2 = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        ab[k] = b[k] - a[k];
        ap_ab += ab[k] * (p[k] - a[k]);
        ab2 += ab[k] * ab[k];
    }
    if (ap_ab <= 0.f) {
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = a[k];
    } else if (ap_ab >= ab2) {
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = b[k];
    } else {
        const float u = ap_ab / ab2;
#pragma unroll
        for (int k = 0; k < D; ++k) q[k] = a[k] + ab[k] * u;
    }
}

// Capsule = segment a-b inflated by `radius` (capsule.slang:38-55): the
// closest axis point pushed out by the radius.  A point exactly on the axis
// goes out along a fixed unit vector orthogonal to the axis: in 3D the first
// vector of the branchless orthonormal basis of Duff et al., "Building an
// Orthonormal Basis, Revisited" (JCGT 2017).  Returns "inside".
template <int D>
__device__ __forceinline__ bool capsule_boundary(const float *a, const float *b, float radius, const float *p,
                                                 float *out) {
    float q[D], d[D], n2 = 0.f;
    segment_closest<D>(a, b, p, q);
#pragma unroll
    for (int k = 0; k < D; ++k) {
        d[k] = p[k] - q[k];
        n2 += d[k] * d[k];
    }
    const float dist = sqrtf(n2);
    if (dist > 0.f) {
#pragma unroll
        for (int k = 0; k < D; ++k) out[k] = q[k] + d[k] * (radius / dist);
        return dist <= radius;
    }
    float ax[D], l2 = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        ax[k] = b[k] - a[k];
        l2 += ax[k] * ax[k];
    }
    const float len = sqrtf(l2);
#pragma unroll
    for (int k = 0; k < D; ++k) ax[k] /= len;
    float o[D];
    if constexpr (D == 2) {
        o[0] = ax[1];
        o[1] = -ax[0];
    } else {
        const float sg = ax[2] >= 0.f ? 1.f : -1.f;
        const float aa = -1.0f / (sg + ax[2]);
        const float bb = ax[0] * ax[1] * aa;
        o[0] = 1.0f + sg * ax[0] * ax[0] * aa;
        o[1] = sg * bb;
        o[2] = -sg * ax[0];
    }
#pragma unroll
    for (int k = 0; k < D; ++k) out[k] = q[k] + o[k] * radius;
    return true;
}

// Cylinder of half height hh and radius r around the local y axis
// (cylinder.slang:72-125): inside, the nearest of the two caps and the
// side; outside, the cap disc, the cap rim or the side.  Returns "inside".
__device__ __forceinline__ bool cylinder_boundary(float hh, float r, const float *p, float *out) {
    const float rxz = sqrtf(p[0] * p[0] + p[2] * p[2]);
    const float dx = rxz > 0.f ? p[0] / rxz : 1.f, dz = rxz > 0.f ? p[2] / rxz : 0.f;
    const float sx = dx * r, sz = dz * r;
    if (p[1] >= -hh && p[1] <= hh && rxz <= r) {
        const float to_top = hh - p[1], to_bottom = p[1] + hh, to_side = r - rxz;
        if (to_top < to_bottom && to_top < to_side) {
            out[0] = p[0], out[1] = hh, out[2] = p[2];
        } else if (to_bottom < to_top && to_bottom < to_side) {
            out[0] = p[0], out[1] = -hh, out[2] = p[2];
        } else {
            out[0] = sx, out[1] = p[1], out[2] = sz;
        }
        return true;
    }
    if (p[1] > hh || p[1] < -hh) {
        const float y = p[1] > hh ? hh : -hh;
        if (rxz <= r) out[0] = p[0], out[1] = y, out[2] = p[2];
        else out[0] = sx, out[1] = y, out[2] = sz;
    } else {
        out[0] = sx, out[1] = p[1], out[2] = sz;
    }
    return false;
}

// Cone of half height hh and base radius r, apex at +hh on the local y axis
// (cone.slang:82-131): below the base disc, the disc; otherwise the closest
// point of the generatrix through the point's azimuth, or (inside) the base
// when that is nearer.  Returns "inside".
__device__ __forceinline__ bool cone_boundary(float hh, float r, const float *p, float *out) {
    const float rxz = sqrtf(p[0] * p[0] + p[2] * p[2]);
    const float dx = rxz > 0.f ? p[0] / rxz : 1.f, dz = rxz > 0.f ? p[2] / rxz : 0.f;
    const float base[3] = {p[0], -hh, p[2]};
    if (p[1] < -hh && rxz <= r) {
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k] = base[k];
        return false;
    }
    const float rim[3] = {dx * r, -hh, dz * r};
    const float apex[3] = {0.f, hh, 0.f};
    float proj[3];
    segment_closest<3>(apex, rim, p, proj);
    const float gen[3] = {rim[0] - apex[0], rim[1] - apex[1], rim[2] - apex[2]};
    const float ap[3] = {p[0] - apex[0], p[1] - apex[1], p[2] - apex[2]};
    const float axis[3] = {0.f, -2.0f * hh, 0.f};
    const float c1[3] = {gen[1] * ap[2] - gen[2] * ap[1], gen[2] * ap[0] - gen[0] * ap[2], gen[0] * ap[1] - gen[1] * ap[0]};
    const float c2[3] = {gen[1] * axis[2] - gen[2] * axis[1], gen[2] * axis[0] - gen[0] * axis[2],
                         gen[0] * axis[1] - gen[1] * axis[0]};
    const bool in = p[1] >= -hh && p[1] <= hh && (c1[0] * c2[0] + c1[1] * c2[1] + c1[2] * c2[2]) >= 0.f;
    if (in) {
        float d_side = 0.f, d_base = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            d_side += (proj[k] - p[k]) * (proj[k] - p[k]);
            d_base += (base[k] - p[k]) * (base[k] - p[k]);
        }
        const float *src = d_side > d_base ? base : proj;
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k] = src[k];
        return true;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = proj[k];
    return false;
}

// Shape::project_point_on_boundary for balls, cuboids, capsules, cylinders
// and cones (shaders/slosh/rbd/shapes/shape.slang:152-175; ball.slang:39-52,
// cuboid.slang:14-63, capsule.slang, cylinder.slang, cone.slang), and the
// triangle-mesh query of collide (collision/collide.slang:124-134): a mesh
// point is returned only within `cap` of the surface.
template <int D>
__device__ __forceinline__ bool project_on_boundary(const DevBody &b, const float *pt, float *proj, bool &inside,
                                                    const float4 *mvtx, const uint32_t *midx, float cap) {
    float local[D], lp[D];
    pose_inv_mul_pt<D>(b, pt, local);
    if (b.shape_type == SLOSH_SHAPE_CUBOID) {
        float outp[D], sgn[D], diff[D], inp[D];
        bool in = true;
#pragma unroll
        for (int i = 0; i < D; ++i) {
            const float shift = fmaxf(-b.sa[i] - local[i], 0.f) - fmaxf(local[i] - b.sa[i], 0.f);
            outp[i] = local[i] + shift;
            const float sw = (local[i] > 0.f) ? 1.f : ((local[i] < 0.f) ? -1.f : 0.f);
            sgn[i] = sw + (fabsf(sw) - 1.f);
            diff[i] = b.sa[i] - sgn[i] * local[i];
            inp[i] = local[i];
            in = in && (local[i] == outp[i]);
        }
        if constexpr (D == 3) {
            const bool px = diff[0] <= diff[1] && diff[0] <= diff[2];
            const bool py = diff[1] <= diff[0] && diff[1] <= diff[2];
            if (px) inp[0] = local[0] + diff[0] * sgn[0];
            else if (py) inp[1] = local[1] + diff[1] * sgn[1];
            else inp[2] = local[2] + diff[2] * sgn[2];
        } else {
            if (diff[0] <= diff[1]) inp[0] = local[0] + diff[0] * sgn[0];
            else inp[1] = local[1] + diff[1] * sgn[1];
        }
#pragma unroll
        for (int i = 0; i < D; ++i) lp[i] = in ? inp[i] : outp[i];
        inside = in;
    } else if (b.shape_type == SLOSH_SHAPE_BALL) {
        float n2 = 0.f;
#pragma unroll
        for (int i = 0; i < D; ++i) n2 += local[i] * local[i];
        const float dist = sqrtf(n2), rad = b.sa[0];
#pragma unroll
        for (int i = 0; i < D; ++i) lp[i] = (dist != 0.f) ? local[i] * (rad / dist) : 0.f;
        if (dist == 0.f) lp[1] = rad;
        inside = dist <= rad;
    } else if (b.shape_type == SLOSH_SHAPE_CAPSULE) {
        inside = capsule_boundary<D>(b.sa, b.sb, b.sb[3], local, lp);
    } else if constexpr (D == 3) {
        if (b.shape_type == SLOSH_SHAPE_CYLINDER) inside = cylinder_boundary(b.sa[0], b.sa[1], local, lp);
        else if (b.shape_type == SLOSH_SHAPE_CONE) inside = cone_boundary(b.sa[0], b.sa[1], local, lp);
        else if (b.shape_type == SLOSH_SHAPE_TRIMESH && mvtx) {
            if (!trimesh_project(trimesh_ref(b.sa, b.sb), mvtx, midx, local, cap, lp, inside)) return false;
        } else
            return false;
    } else {
        return false;
    }
    pose_mul_pt<D>(b, lp, proj);
    return true;
}

// collide (shaders/slosh/collision/collide.slang:87-153).  Returns the
// collider id or NONE; `nd` = (normal, dot(point_node - proj, normal)).
template <int D>
__device__ __forceinline__ uint32_t collide(const DevBody *bodies, uint32_t n_bodies, float h, const float *pt,
                                            float4 &nd, const float4 *mvtx, const uint32_t *midx) {
    const float cap = h * 1.5f;
    float best = 1.0e10f;
    uint32_t id = NONE;
    float bn[D] = {}, bp[D] = {};
    for (uint32_t i = 0; i < n_bodies && i < MAX_BODIES; ++i) {
        float proj[D];
        bool inside = false;
        if (!project_on_boundary<D>(bodies[i], pt, proj, inside, mvtx, midx, cap)) continue;
        float dpt[D], n2 = 0.f;
        bool within = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
            dpt[k] = proj[k] - pt[k];
            within = within && (fabsf(dpt[k]) <= cap);
            n2 += dpt[k] * dpt[k];
        }
        if (inside || within) {
            const float sign = inside ? -1.f : 1.f;
            const float dist = sqrtf(n2);
            if (sign * dist < best && dist != 0.f) {
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    bn[k] = dpt[k] / (dist * -sign);
                    bp[k] = proj[k];
                }
                id = i;
                best = dist;
            }
        }
    }
    float dd = 0.f;
#pragma unroll
    for (int k = 0; k < D; ++k) dd += (pt[k] - bp[k]) * bn[k];
    nd = make_float4(bn[0], bn[1], D == 3 ? bn[D - 1] : 0.f, dd);
    return id;
}

// BoundaryCondition::project_velocity (boundary_condition.slang:31-89),
// keeping slosh's use of the collider friction for FrictionZUp.
template <int D>
__device__ __forceinline__ void project_velocity(uint32_t type, float friction, float *vel, const float *n, float dist,
                                                 float dt) {
    if (type == SLOSH_BC_STICK) {
        if (dist <= 0.f)
#pragma unroll
            for (int k = 0; k < D; ++k) vel[k] = 0.f;
    } else if (type == SLOSH_BC_SLIP) {
        if (dist <= 0.f) {
            float nv = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
#pragma unroll
            for (int k = 0; k < D; ++k) vel[k] = vel[k] - n[k] * nv;
        }
    } else if (type == SLOSH_BC_SEPARATE || type == SLOSH_BC_FRICTION_Z_UP) {
        float nv = 0.f;
#pragma unroll
        for (int k = 0; k < D; ++k) nv += vel[k] * n[k];
        if (nv < 0.f) {
            if (dist <= 0.f) {
                float tv[D], tl2 = 0.f;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    tv[k] = vel[k] - n[k] * nv;
                    tl2 += tv[k] * tv[k];
                }
                const float tl = sqrtf(tl2);
                const float sc = fmaxf(0.f, tl + friction * nv);
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = ((tl > 1.0e-8f) ? tv[k] / tl : 0.f) * sc;
            } else if (-nv * dt > dist) {
                const float a = dist / dt + nv;
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = vel[k] - a * n[k];
            }
        }
    }
}

// Grid update (shaders/slosh/solver/grid_update.slang:38-163), one thread per
// node.  The collision of a node is reused from the previous substep when
// its block was active there (slosh's cache, which assumes static colliders),
// otherwise collide() runs; both are recorded for the next substep.
// 8 CTAs of 256 per SM (64 warps): the node gather is a chain of dependent
// loads, so occupancy pays; the register cap (32) leaves the rare collision
// queries (nodes without a cached collision) to spill, not the common path.
template <int D, bool B = false> __device__ __forceinline__ void grid_update_body(const DevScene &s, Cta g) {
    constexpr int BW = Geo<D>::BW;
    const uint32_t nb = s.ctr->n_blocks;
    const uint32_t stride = g.n * blockDim.x;
    float h = s.h, dt = s.dt, grav[3] = {s.gravity[0], s.gravity[1], s.gravity[2]};
    const DevBody *bodies = s.bodies;
    uint32_t n_bodies = s.n_bodies, sc = 0;
    for (uint32_t t = g.id * blockDim.x + threadIdx.x; t < nb * 64u; t += stride) {
        const uint32_t r = t >> 6, node = t & 63u;
        if constexpr (B) {
            sc = s.bscene[r];
            const SceneRec &rec = s.scenes[sc];
            h = rec.h;
            dt = rec.dt;
            for (int k = 0; k < 3; ++k) grav[k] = rec.gravity[k];
            bodies = s.bodies + rec.body_first;
            n_bodies = rec.n_bodies;
        }
        const float vlim = h / dt;
        const uint32_t key = s.bkey[r];
        int bv[D], lc[D];
        unpack_key<D>(key, bv);
        if constexpr (D == 3) {
            lc[0] = node & 3;
            lc[1] = (node >> 2) & 3;
            lc[2] = node >> 4;
        } else {
            lc[0] = node & 7;
            lc[1] = node >> 3;
        }
        float cell_pos[D];
#pragma unroll
        for (int k = 0; k < D; ++k) cell_pos[k] = (float)(bv[k] * BW + lc[k]) * h;
        float4 nv;
        if (s.use_partial) {
            // Node sums of the deterministic P2G: the tiles of this block and
            // of its -1 neighbours b - o that cover the node (local
            // coordinate + BW o inside the tile), added in the fixed order
            // of o.
            constexpr int TW = Geo<D>::TW, NN = Geo<D>::NASSOC - 1;
            nv = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int q = 0; q < Geo<D>::NASSOC; ++q) {
                int o[D];
                assoc_offset<D>(q, o);
                bool inside = true;
                int tix = 0, mul = 1;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const int tc = lc[k] + BW * o[k];
                    inside = inside && tc < TW;
                    tix += tc * mul;
                    mul *= TW;
                }
                if (!inside) continue;
                // blocks without particles have no tile (their -1
                // neighbour ranks are NONE)
                const uint32_t ra = (q == 0) ? (s.bnp[r] != 0u ? r : NONE) : s.bnbh_rev[r * NN + q - 1];
                if (ra >= nb) continue;
                const float4 v = s.partial[(size_t)ra * Geo<D>::TILE + tix];
                nv.x += v.x;
                nv.y += v.y;
                nv.z += v.z;
                nv.w += v.w;
            }
            if (s.gather_only) {
                s.nodes[t] = nv;
                continue;
            }
        } else {
            nv = s.nodes[t];
        }
        const float pm[3] = {nv.x, nv.y, nv.z};
        const float mass = nv.w;
        const float inv_mass = mass > 0.f ? 1.0f / mass : 0.f;
        float vel[D];
#pragma unroll
        for (int k = 0; k < D; ++k) {
            const float v = (pm[k] + mass * grav[k] * dt) * inv_mass;
            vel[k] = fminf(fmaxf(v, -vlim), vlim);
        }
        // The cached normal and distance are read, and recorded, only for a
        // node that has a collision (cid != NONE), their only readers.
        float4 cn = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t cid;
        const uint32_t prank = s.bprev[r];
        if (prank != NONE && !s.coll_dynamic) {
            cid = s.prev_coll_id[(size_t)prank * 64u + node];
            if (cid != NONE) cn = s.prev_coll[(size_t)prank * 64u + node];
        } else {
            cid = collide<D>(bodies, n_bodies, h, cell_pos, cn, s.mesh_vtx, s.mesh_idx);
        }
        if (cid != NONE) s.coll[t] = cn;
        s.coll_id[t] = cid;
        if (cid != NONE) {
            const DevBody &bd = bodies[cid];
            const float n[3] = {cn.x, cn.y, cn.z};
            if (bd.coupling == SLOSH_COUPLING_TWO_WAY) {
                // project in the body's frame; the momentum the node loses
                // goes to the body as an impulse at the node
                float com[3] = {0.f, 0.f, 0.f}, r[3] = {0.f, 0.f, 0.f}, vb[3] = {0.f, 0.f, 0.f};
                pose_mul_pt<D>(bd, bd.local_com, com);
#pragma unroll
                for (int k = 0; k < D; ++k) r[k] = cell_pos[k] - com[k];
                if constexpr (D == 3) {
                    vb[0] = bd.linvel[0] + bd.angvel[1] * r[2] - bd.angvel[2] * r[1];
                    vb[1] = bd.linvel[1] + bd.angvel[2] * r[0] - bd.angvel[0] * r[2];
                    vb[2] = bd.linvel[2] + bd.angvel[0] * r[1] - bd.angvel[1] * r[0];
                } else {
                    vb[0] = bd.linvel[0] - bd.angvel[0] * r[1];
                    vb[1] = bd.linvel[1] + bd.angvel[0] * r[0];
                }
                float rel[D];
#pragma unroll
                for (int k = 0; k < D; ++k) rel[k] = vel[k] - vb[k];
                project_velocity<D>(bd.bc_type, bd.friction, rel, n, cn.w - h, dt);
                float J[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const float nvk = rel[k] + vb[k];
                    J[k] = mass * (vel[k] - nvk);
                    vel[k] = nvk;
                }
                if (mass > 0.f) {
                    float A[3];
                    int na;
                    if constexpr (D == 3) {
                        A[0] = r[1] * J[2] - r[2] * J[1];
                        A[1] = r[2] * J[0] - r[0] * J[2];
                        A[2] = r[0] * J[1] - r[1] * J[0];
                        na = 3;
                    } else {
                        A[0] = r[0] * J[1] - r[1] * J[0];
                        na = 1;
                    }
                    unsigned long long *acc = s.body_imp + (size_t)(&bd - s.bodies) * 6u;
#pragma unroll
                    for (int k = 0; k < D; ++k)
                        if (J[k] != 0.f) atomicAdd(acc + k, (unsigned long long)__double2ll_rn((double)J[k] * IMPULSE_UNITS));
                    for (int k = 0; k < na; ++k)
                        if (A[k] != 0.f)
                            atomicAdd(acc + 3 + k, (unsigned long long)__double2ll_rn((double)A[k] * IMPULSE_UNITS));
                }
            } else {
                project_velocity<D>(bd.bc_type, bd.friction, vel, n, cn.w - h, dt);
            }
        }
        s.nodes[t] = make_float4(vel[0], vel[1], D == 3 ? vel[D - 1] : 0.f, mass);
    }
}
template <int D, bool B = false> __global__ void __launch_bounds__(256, 8) k_grid_update(DevScene s) {
    pdl_enter();
    grid_update_body<D, B>(s, launch_cta());
}

// Clears the next substep's hash map and the key histogram / per-scene
// block counts (their readers in this substep have all run), thread g0 of
// gs.  Done by the fused G2P / particle update, or by k_clear_next when a
// stage hook replaced it.
template <bool B> __device__ __forceinline__ void clear_next_map(const DevScene &s, uint32_t g0, uint32_t gs) {
    for (uint32_t q = g0; q < s.hcap; q += gs) {
        if constexpr (B) s.clr_hkeys64[q] = NONE64;
        else s.clr_hkeys[q] = NONE;
        s.clr_hvals[q] = NONE;
    }
    if constexpr (B) {
        for (uint32_t q = g0; q < s.n_scenes; q += gs) s.scene_nblk[q] = 0u;
    } else {
        for (uint32_t q = g0; q < HIST_BINS; q += gs) s.hist[q] = 0u;
        if (g0 < HIST_COARSE) s.hist_coarse[g0] = 0u;
    }
    if (*s.err != 0u)
        for (size_t q = g0; q < (size_t)s.hcap * CELLS; q += gs) s.slot_counts[q] = 0u;
}

// After a stage hook replaced the fused G2P / particle update: the next
// map cleared as G2P would, and the original-index plane of the next
// storage taken from its flags plane.
__global__ void k_after_replaced_g2p(DevScene s) {
    pdl_enter();
    const uint32_t g0 = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    clear_next_map<false>(s, g0, gs);
    for (uint32_t i = g0; i < s.count; i += gs) s.out_oid[i] = s.out_fo[i].y;
}

// Grid-reuse bookkeeping of one particle that G2P has just moved from xo to
// xn (storage position in block r of this substep's grid): when its base
// cell changed, the per-cell count deltas and touched-cell bits of the old
// and new blocks, which the next substep's k_grid_reuse applies; when the
// change is one the kept grid cannot hold (a move of more than one cell, or
// into a block without particles or outside the grid), the next substep's
// full build.  The cells are the ones k_touch would compute from the stored
// positions.
template <int D, bool POW2>
__device__ __forceinline__ void note_cell_change(const DevScene &s, uint32_t r, const float4 &xo4, const float4 &xn4,
                                                 float h, float inv_h, uint32_t h_pow2) {
    const float xo[3] = {xo4.x, xo4.y, xo4.z}, xn[3] = {xn4.x, xn4.y, xn4.z};
    // round(x / h) per axis, as locate() computes it (the base cell is one less)
    int co[D], cn[D];
    bool moved = false;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        co[k] = __float2int_rn(POW2 ? xo[k] * inv_h : div_h(xo[k], h, inv_h, h_pow2));
        cn[k] = __float2int_rn(POW2 ? xn[k] * inv_h : div_h(xn[k], h, inv_h, h_pow2));
        moved = moved || co[k] != cn[k];
    }
    if (!moved) return;
    constexpr int SHIFT = Geo<D>::BW == 4 ? 2 : 3, BW = Geo<D>::BW;
    int bo[D], bn[D], lo[D], ln[D];
    bool far = false, same_block = true;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int dc = cn[k] - co[k];
        far = far || dc > 1 || dc < -1;
        bo[k] = (co[k] - 1) >> SHIFT;
        bn[k] = (cn[k] - 1) >> SHIFT;
        lo[k] = (co[k] - 1) & (BW - 1);
        ln[k] = (cn[k] - 1) & (BW - 1);
        same_block = same_block && bo[k] == bn[k];
    }
    uint32_t r2 = r;
    bool ok = !far;
    if (ok && !same_block) {
        const uint32_t slot = hash_find(s.hkeys, s.hcap, pack_key<D>(bn));
        const uint32_t v = slot == NONE ? NONE : s.hvals[slot];
        ok = v != NONE && (v & RANK_EXTRA) == 0u;
        r2 = v;
    }
    if (!ok) {
        s.ctr->rebuild[s.par ^ 1u] = 1u;
        return;
    }
    const uint32_t c_old = cell_index<D>(lo), c_new = cell_index<D>(ln);
    atomicAdd(&s.cell_delta[(size_t)r * CELLS + c_old], -1);
    atomicAdd(&s.cell_delta[(size_t)r2 * CELLS + c_new], 1);
    atomicOr(&s.touch[r], 1ull << c_old);
    atomicOr(&s.touch[r2], 1ull << c_new);
}

// G2P fused with the particle update.  One CTA per active block with
// primaries: the block's (block + 2)^D tile of node velocities is staged in
// shared memory, then each thread gathers v, grad v and div v for its
// particles (g2p.slang:150-265) and applies the particle update of
// particle_update.slang:48-159 with the constitutive model, writing the new
// position, velocity, APIC matrix C and F.  The inputs of a thread's next
// particle (x, m, F, V0, flags, original id, plastic state, damping) are
// staged into shared memory with cp.async while the current particle is
// computed; each thread consumes only its own staged slot, so the particle
// loop has no barrier.
// POW2: the cell width is a power of two (known at launch), so x / h is
// exactly x * (1/h) and no division is compiled in.  MODEL >= 0: every
// particle of the scene uses that model tag (known at upload), so only its
// constitutive code is compiled in; MODEL < 0 reads each particle's tag.
// Shared memory of k_g2p_update's CTA (NT threads): the block's node tile
// (velocity, mass: one 16-byte load a node) and two buffers of staged
// particles, one particle a thread.
template <int D, int NT> struct G2pSmem {
    float4 tv[Geo<D>::TILE];
    float4 st_pm[2][NT];
    float4 st_fq[2][MQ<D>::Q][NT];
    uint4 st_fo[2][NT];
    float4 st_ps[2][NT];
    uint32_t next_r;
};

template <int D, int NT, bool B = false, bool POW2 = false, int MODEL = -1>
__device__ __forceinline__ void g2p_update_body(const DevScene &s, Cta g, G2pSmem<D, NT> &sm) {
    constexpr int TW = Geo<D>::TW, TILE = Geo<D>::TILE, BW = Geo<D>::BW;
    constexpr int Q = MQ<D>::Q;
    auto &tv = sm.tv;
    auto &st_pm = sm.st_pm;
    auto &st_fq = sm.st_fq;
    auto &st_fo = sm.st_fo;
    auto &st_ps = sm.st_ps;
    const uint32_t nb = s.ctr->n_blocks;
    float h = s.h, dt = s.dt, inv_h = s.inv_h;
    uint32_t h_pow2 = s.h_pow2;
    float inv_d = 4.0f / (h * h);
    float vmax = h / dt;
    const size_t n = s.n;
    const uint32_t tid = threadIdx.x;
    if (s.clear_tail) clear_next_map<B>(s, g.id * NT + tid, g.n * NT);
    // Issues the copies of sorted entry e (storage index i) of the block into
    // buffer b (an empty group when e is past the block's particles).  The
    // storage index is loaded one iteration before the copies that need it.
    auto stage = [&](int b, uint32_t e, uint32_t np, uint32_t i) {
        if (e < np) {
            cp_async16(&st_pm[b][tid], &s.pm[i]);
#pragma unroll
            for (int q = 0; q < Q; ++q) cp_async16(&st_fq[b][q][tid], &s.fq[q * n + i]);
            cp_async16(&st_fo[b][tid], &s.fo[i]);
            if (s.has_sand | s.has_damping) cp_async16(&st_ps[b][tid], &s.ps[i]);
        }
        cp_async_commit();
    };
    // blocks are taken from a queue, one atomic a block
    uint32_t &next_r = sm.next_r;
    for (;;) {
        __syncthreads();  // every thread has read next_r
        if (tid == 0) {
            if (B && s.g2p_class >= 0) {  // this launch's class of the batch's blocks
                const uint32_t cls = (uint32_t)s.g2p_class;
                const uint32_t q = atomicAdd(&s.g2p_counts[G2P_CLASSES + cls], 1u);
                next_r = q < s.g2p_counts[cls] ? s.g2p_lists[(size_t)cls * s.cap + q] : nb;
            } else {
                next_r = atomicAdd(&s.ctr->g2p_next, 1u);
            }
        }
        __syncthreads();
        const uint32_t r = next_r;
        if (r >= nb) break;
        const uint32_t np = s.bnp[r];
        if (np == 0) continue;
        const uint32_t first = s.bfirst[r];
        // storage index of entry e: from the block's storage start when its
        // particles are one shifted range of storage, else the permutation
        const uint32_t src = (!B && s.reuse && s.bsrc != nullptr) ? s.bsrc[r] : NONE;
        auto pidx = [&](uint32_t e) { return src != NONE ? src + e : s.perm[first + e]; };
        stage(0, tid, np, tid < np ? pidx(tid) : 0u);
        uint32_t i_next = tid + NT < np ? pidx(tid + NT) : 0u;
        if constexpr (B) {
            const SceneRec &rec = s.scenes[s.bscene[r]];
            h = rec.h;
            dt = rec.dt;
            inv_h = rec.inv_h;
            h_pow2 = rec.h_pow2;
            inv_d = 4.0f / (h * h);
            vmax = h / dt;
        }
        for (int t = threadIdx.x; t < TILE; t += NT) {
            uint32_t rank, local;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (tile_node_owner<D>(s, r, t, rank, local)) v = s.nodes[(size_t)rank * 64u + local];
            tv[t] = v;
        }
        __syncthreads();
        int bv[D];
        unpack_key<D>(s.bkey[r], bv);
        int buf = 0;
        for (uint32_t e = tid; e < np; e += NT, buf ^= 1) {
            stage(buf ^ 1, e + NT, np, i_next);
            i_next = e + 2 * NT < np ? pidx(e + 2 * NT) : 0u;
            cp_async_wait<1>();
            const float4 p = st_pm[buf][tid];
            const float x[3] = {p.x, p.y, p.z};
            float m = p.w;
            const uint4 fo = st_fo[buf][tid];
            uint32_t fl = fo.x;
            // ---- G2P ----
            float vel[D], grad[D][D], div = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) {
                vel[k] = 0.f;
#pragma unroll
                for (int l = 0; l < D; ++l) grad[k][l] = 0.f;
            }
            if (fl & FLAG_ENABLED) {
                float d0[D], w[D][3];
                int a[D];
                bool in_block = true;
#pragma unroll
                for (int k = 0; k < D; ++k) {
                    const float assoc = rintf(POW2 ? x[k] * inv_h : div_h(x[k], h, inv_h, h_pow2)) - 1.0f;
                    a[k] = (int)assoc - bv[k] * BW;
                    in_block = in_block && a[k] >= 0 && a[k] < BW;
                    d0[k] = assoc * h - x[k];
                    bspline_weights(POW2 ? -d0[k] * inv_h : div_h(-d0[k], h, inv_h, h_pow2), w[k]);
                }
                if (!in_block) {  // packed-key aliasing: gather nothing
                    atomicOr(s.err, ERR_KEY_RANGE);
#pragma unroll
                    for (int k = 0; k < D; ++k) a[k] = 0, w[k][0] = w[k][1] = w[k][2] = 0.f;
                }
                // Separable gather.  With w_s = wx[sx] wy[sy] wz[sz] and
                // dpt_s = d0 + s h, the sums of g2p.slang:196-244 are
                //   v = M0,  grad v[c][r] = inv_d (d0_r M0_c + h M_r,c),
                //   vel_grad_det = trace(grad v),
                // with M0 = sum_s w_s v_s and M_r = sum_s w_s s_r v_s,
                // accumulated axis by axis.
                // Separable gather in paired FP32 arithmetic: the node
                // velocity (x, y, z, mass) is read as the pairs (x, y) and
                // (z, mass); the mass lane is carried along unused.  Terms
                // with offset 0 (s_r = 0) add nothing and are skipped.
                constexpr int NP = (D == 3) ? 2 : 1;
                float2 M0p[NP], Mrp[D][NP];
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    M0p[q] = make_float2(0.f, 0.f);
#pragma unroll
                    for (int k = 0; k < D; ++k) Mrp[k][q] = make_float2(0.f, 0.f);
                }
                const float2 wx0p = pair(w[0][0]), wx1p = pair(w[0][1]), wx2p = pair(w[0][2]),
                             wx2bp = pair(2.f * w[0][2]);
                auto row = [&](const float4 &n0, const float4 &n1, const float4 &n2, int q, float2 &R0, float2 &Rx) {
                    const float2 v0 = q ? hi_pair(n0) : lo_pair(n0), v1 = q ? hi_pair(n1) : lo_pair(n1),
                                 v2 = q ? hi_pair(n2) : lo_pair(n2);
                    R0 = __ffma2_rn(wx2p, v2, __ffma2_rn(wx1p, v1, __fmul2_rn(wx0p, v0)));
                    Rx = __ffma2_rn(wx2bp, v2, __fmul2_rn(wx1p, v1));
                };
                if constexpr (D == 3) {
#pragma unroll
                    for (int sz = 0; sz < 3; ++sz) {
                        float2 S0[2], Sx[2], Sy[2];
#pragma unroll
                        for (int q = 0; q < 2; ++q) S0[q] = Sx[q] = Sy[q] = make_float2(0.f, 0.f);
#pragma unroll
                        for (int sy = 0; sy < 3; ++sy) {
                            const int idx = a[0] + TW * ((a[1] + sy) + TW * (a[2] + sz));
                            const float2 wyp = pair(w[1][sy]), wysp = pair((float)sy * w[1][sy]);
                            const float4 n0 = tv[idx], n1 = tv[idx + 1], n2 = tv[idx + 2];
#pragma unroll
                            for (int q = 0; q < 2; ++q) {
                                float2 R0, Rx;
                                row(n0, n1, n2, q, R0, Rx);
                                S0[q] = __ffma2_rn(wyp, R0, S0[q]);
                                Sx[q] = __ffma2_rn(wyp, Rx, Sx[q]);
                                if (sy > 0) Sy[q] = __ffma2_rn(wysp, R0, Sy[q]);
                            }
                        }
                        const float2 wzp = pair(w[2][sz]), wzsp = pair((float)sz * w[2][sz]);
#pragma unroll
                        for (int q = 0; q < 2; ++q) {
                            M0p[q] = __ffma2_rn(wzp, S0[q], M0p[q]);
                            Mrp[0][q] = __ffma2_rn(wzp, Sx[q], Mrp[0][q]);
                            Mrp[1][q] = __ffma2_rn(wzp, Sy[q], Mrp[1][q]);
                            if (sz > 0) Mrp[2][q] = __ffma2_rn(wzsp, S0[q], Mrp[2][q]);
                        }
                    }
                } else {
#pragma unroll
                    for (int sy = 0; sy < 3; ++sy) {
                        const int idx = a[0] + TW * (a[1] + sy);
                        const float2 wyp = pair(w[1][sy]), wysp = pair((float)sy * w[1][sy]);
                        float2 R0, Rx;
                        row(tv[idx], tv[idx + 1], tv[idx + 2], 0, R0, Rx);
                        M0p[0] = __ffma2_rn(wyp, R0, M0p[0]);
                        Mrp[0][0] = __ffma2_rn(wyp, Rx, Mrp[0][0]);
                        if (sy > 0) Mrp[1][0] = __ffma2_rn(wysp, R0, Mrp[1][0]);
                    }
                }
                // v = M0, grad v[c][r] = inv_d (d0_r M0_c + h M_r,c), pairs over c
                const float2 hp = pair(h), invdp = pair(inv_d);
#pragma unroll
                for (int rr = 0; rr < D; ++rr) {
                    const float2 d0p = pair(d0[rr]);
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        const float2 g = __fmul2_rn(invdp, __ffma2_rn(d0p, M0p[q], __fmul2_rn(hp, Mrp[rr][q])));
                        grad[2 * q][rr] = g.x;
                        if (2 * q + 1 < D) grad[2 * q + 1][rr] = g.y;
                    }
                }
                vel[0] = M0p[0].x;
                vel[1] = M0p[0].y;
                if constexpr (D == 3) vel[2] = M0p[1].x;
                div = grad[0][0] + grad[1][1];
                if constexpr (D == 3) div += grad[2][2];
            }
            // ---- particle update ----
            const Material &mat = s.materials[fl & FLAG_MAT_MASK];
            const uint32_t tag = MODEL >= 0 ? (uint32_t)MODEL : mat.tag;
            const bool fluid = tag == SLOSH_MODEL_FLUID_TAIT;
            const bool sand = tag == SLOSH_MODEL_SAND_LINEAR || tag == SLOSH_MODEL_SAND_NEO_HOOKEAN;
            float len2 = 0.f;
#pragma unroll
            for (int k = 0; k < D; ++k) len2 += vel[k] * vel[k];
            // |v| > h / dt, tested on the squares first (sqrt is monotone; the
            // square root is taken only for a particle near the clamp).  When
            // (h / dt)^2 overflows, every particle takes the exact test.
            const float vclamp2 = vmax * vmax * (1.0f - 4e-7f);
            if (len2 > vclamp2 || isinf(vclamp2)) {
                const float len = sqrtf(len2);
                if (len > vmax)
#pragma unroll
                    for (int k = 0; k < D; ++k) vel[k] = vel[k] / len * h / dt;
            }
            const float4 ps = (s.has_sand | s.has_damping) ? st_ps[buf][tid] : make_float4(0.f, 0.f, 0.f, 0.f);
            if (s.has_damping) {
                const float dmp = 1.0f + ps.w * dt;
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = vel[k] / dmp;
            }
            const bool fixed = (fl & FLAG_FIXED) != 0;
            if (fixed)
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = 0.f;
            float nx[D];
#pragma unroll
            for (int k = 0; k < D; ++k) nx[k] = x[k] + vel[k] * dt;
            float F[D][D];
            {
                float4 fv[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) fv[q] = st_fq[buf][q][tid];
                mat_from<D>(fv, __uint_as_float(fo.w), F);
            }
            if (!fluid) {
                // F <- F + (dt grad v) F, row by row in column pairs (c, c + 1)
                float Fn[D][D];
#pragma unroll
                for (int rr = 0; rr < D; ++rr) {
                    float2 g[D];
#pragma unroll
                    for (int k = 0; k < D; ++k) g[k] = pair(grad[rr][k] * dt);
#pragma unroll
                    for (int c = 0; c < D; c += 2) {
                        const bool two = c + 1 < D;
                        auto col = [&](int k) { return make_float2(F[k][c], two ? F[k][c + 1] : 0.f); };
                        float2 acc = __fmul2_rn(col(0), g[0]);
#pragma unroll
                        for (int k = 1; k < D; ++k) acc = __ffma2_rn(col(k), g[k], acc);
                        const float2 r = __fadd2_rn(make_float2(F[rr][c], two ? F[rr][c + 1] : 0.f), acc);
                        Fn[rr][c] = r.x;
                        if (two) Fn[rr][c + 1] = r.y;
                    }
                }
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) F[rr][c] = Fn[rr][c];
            } else {
                const float f0 = F[0][0];
                const float nf = f0 + f0 * div * dt;
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) F[rr][c] = (rr == c) ? nf : 0.f;
            }
            if (fixed)
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) grad[rr][c] = 0.f;
            float st[3] = {0.f, 0.f, 0.f};
            if (sand) {
                st[0] = ps.x;
                st[1] = ps.y;
                st[2] = ps.z;
            }
            float tau[D][D];
            model_update<D>(mat, tag, F, st, tau, &s.ctr->n_svd_fp64);
            const float v0 = __uint_as_float(fo.z);
            const float coef = v0 * inv_d * dt;
            bool finite = true;
#pragma unroll
            for (int k = 0; k < D; ++k) finite = finite && (nx[k] == nx[k]);
            // The particle is stored at its canonical position o in the
            // output buffers (contiguous, coalesced writes).
            const size_t o = (size_t)first + e;
            float Cn[D][D];
            float4 np4 = p;
            if (finite && det<D>(F) > 0.f) {
                np4.x = nx[0];
                np4.y = nx[1];
                if constexpr (D == 3) np4.z = nx[2];
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) Cn[rr][c] = grad[rr][c] * m - tau[rr][c] * coef;
            } else {
                fl &= ~FLAG_ENABLED;
                m = 0.f;
                np4.w = 0.f;
#pragma unroll
                for (int rr = 0; rr < D; ++rr)
#pragma unroll
                    for (int c = 0; c < D; ++c) {
                        F[rr][c] = (rr == c) ? 1.f : 0.f;
                        Cn[rr][c] = 0.f;
                    }
#pragma unroll
                for (int k = 0; k < D; ++k) vel[k] = 0.f;
            }
            float4 cv[Q], fv[Q];
            const float c22 = mat_split<D>(Cn, cv), f22 = mat_split<D>(F, fv);
            s.out_pm[o] = np4;
            if constexpr (!B) {
                if (s.reuse && (st_fo[buf][tid].x & FLAG_ENABLED)) note_cell_change<D, POW2>(s, r, st_pm[buf][tid], np4, h, inv_h, h_pow2);
            }
            s.out_vv[o] = make_float4(vel[0], vel[1], D == 3 ? vel[D - 1] : 0.f, c22);
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                s.out_cq[q * n + o] = cv[q];
                s.out_fq[q * n + o] = fv[q];
            }
            s.out_fo[o] = make_uint4(fl, fo.y, fo.z, __float_as_uint(f22));
            s.out_oid[o] = fo.y;
            if (s.has_sand | s.has_damping) s.out_ps[o] = make_float4(st[0], st[1], st[2], ps.w);
        }
        cp_async_wait<0>();
        __syncthreads();
    }
}
template <int D, int NT, bool B = false, bool POW2 = false, int MODEL = -1>
__global__ void __launch_bounds__(NT, 512 / NT) k_g2p_update(DevScene s) {
    pdl_enter();
    __shared__ G2pSmem<D, NT> sm;
    g2p_update_body<D, NT, B, POW2, MODEL>(s, launch_cta(), sm);
}

// Rigid-body update (shaders/slosh/solver/rigid_impulses.slang:72-121) with
// integrate_velocity (shaders/slosh/rbd/dynamics/body.slang:117-130).  The
// incremental impulse slosh applies here is never written by any of its
// kernels, so velocity capping (guarded by a non-zero impulse) never runs.
// The last kernel of the substep: it also resets the grid-build counters for
// the next substep.
// Multi-scene batches (B): bodies of all scenes in one table, each with its
// scene's dt and gravity (bodies of dropped scenes are left alone), and the
// particle count in storage becomes this substep's sorted count.
template <int D, bool B = false> __device__ __forceinline__ void rigid_body(const DevScene &s, uint32_t id) {
    if (id == 0 && s.clear_tail) {
        const uint32_t nb = s.ctr->n_blocks;
        s.ctr->last_n_blocks = nb;
        if (!build_skipped(s)) s.ctr->last_n_primary = min(s.ctr->n_primary, s.cap);
        if (s.reuse) s.ctr->rebuild[s.par] = 0u;  // read by this substep only; G2P set the next one's
        if constexpr (B)
            if (s.g2p_lists)
                for (uint32_t c = 0; c < G2P_CLASSES; ++c) s.g2p_counts[c] = 0u;  // the next block setup's lists
        s.ctr->n_primary = 0u;
        s.ctr->n_extra = 0u;
        s.ctr->n_blocks = 0u;
        if constexpr (B) *s.n_dev = nb ? s.bfirst[nb - 1] + s.bnp[nb - 1] : 0u;
    }
    if (id >= s.n_bodies) return;
    DevBody b = s.bodies[id];
    float dt = s.dt, grav[3] = {s.gravity[0], s.gravity[1], s.gravity[2]};
    if constexpr (B) {
        const SceneRec &rec = s.scenes[b.scene];
        if (!rec.live) return;
        dt = rec.dt;
        for (int k = 0; k < 3; ++k) grav[k] = rec.gravity[k];
    }
    if (b.coupling == SLOSH_COUPLING_TWO_WAY) {
        // apply_impulse (shaders/slosh/rbd/dynamics/body.slang:62-70) of the
        // impulse the grid gave this substep, and the velocity caps of
        // rigid_impulses.slang:99-111; the sums restart at zero
        float h = s.h;
        if constexpr (B) h = s.scenes[b.scene].h;
        unsigned long long *acc = s.body_imp + (size_t)id * 6u;
        float jl[3] = {0.f, 0.f, 0.f}, ja[3] = {0.f, 0.f, 0.f};
        for (int k = 0; k < 3; ++k) {
            jl[k] = (float)((double)(long long)acc[k] / IMPULSE_UNITS);
            ja[k] = (float)((double)(long long)acc[3 + k] / IMPULSE_UNITS);
            acc[k] = 0ull;
            acc[3 + k] = 0ull;
        }
        for (int k = 0; k < D; ++k) b.linvel[k] += b.inv_mass[k] * jl[k];
        if constexpr (D == 3) {
            float R[3][3], Iw[9];
            quat_matrix(b.rot, R);
            rotate_tensor(R, b.inv_inertia, Iw, true);
            for (int i = 0; i < 3; ++i) b.angvel[i] += Iw[i * 3] * ja[0] + Iw[i * 3 + 1] * ja[1] + Iw[i * 3 + 2] * ja[2];
        } else {
            b.angvel[0] += b.inv_inertia[0] * ja[0];
        }
        const bool pushed = jl[0] != 0.f || jl[1] != 0.f || jl[2] != 0.f || ja[0] != 0.f || ja[1] != 0.f || ja[2] != 0.f;
        if (pushed) {
            const float lin_limit = 0.1f * h / dt, ang_limit = 1.0f;
            float l2 = 0.f, a2 = 0.f;
            for (int k = 0; k < D; ++k) l2 += b.linvel[k] * b.linvel[k];
            for (int k = 0; k < (D == 3 ? 3 : 1); ++k) a2 += b.angvel[k] * b.angvel[k];
            const float ln = sqrtf(l2), an = sqrtf(a2);
            if (ln > lin_limit)
                for (int k = 0; k < D; ++k) b.linvel[k] = b.linvel[k] * (lin_limit / ln);
            if (an > ang_limit)
                for (int k = 0; k < (D == 3 ? 3 : 1); ++k) b.angvel[k] = b.angvel[k] * (ang_limit / an);
        }
    }
    float init_com[3] = {0.f, 0.f, 0.f};
    pose_mul_pt<D>(b, b.local_com, init_com);
    if constexpr (D == 3) {
        const float sa[3] = {b.angvel[0] * dt, b.angvel[1] * dt, b.angvel[2] * dt};
        const float ang = sqrtf(sa[0] * sa[0] + sa[1] * sa[1] + sa[2] * sa[2]);
        float dq[4] = {0.f, 0.f, 0.f, 1.f};
        if (ang > 0.f) {
            const float sc = sinf(ang * 0.5f) / ang;
            dq[0] = sa[0] * sc;
            dq[1] = sa[1] * sc;
            dq[2] = sa[2] * sc;
            dq[3] = cosf(ang * 0.5f);
        }
        const float rel[3] = {b.tra[0] - init_com[0], b.tra[1] - init_com[1], b.tra[2] - init_com[2]};
        float rr[3];
        quat_rotate(dq, rel, rr);
        for (int k = 0; k < 3; ++k) b.tra[k] = init_com[k] + rr[k] * b.scale + b.linvel[k] * dt;
        const float *q = b.rot;
        float nq[4];
        nq[0] = dq[3] * q[0] + dq[0] * q[3] + dq[1] * q[2] - dq[2] * q[1];
        nq[1] = dq[3] * q[1] - dq[0] * q[2] + dq[1] * q[3] + dq[2] * q[0];
        nq[2] = dq[3] * q[2] + dq[0] * q[1] - dq[1] * q[0] + dq[2] * q[3];
        nq[3] = dq[3] * q[3] - dq[0] * q[0] - dq[1] * q[1] - dq[2] * q[2];
        const float n2 = nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3];
        const float f = 0.5f * (3.0f - n2);
        for (int k = 0; k < 4; ++k) b.rot[k] = nq[k] * f;
    } else {
        const float a = b.angvel[0] * dt;
        const float c = cosf(a), sn = sinf(a);
        const float rel0 = b.tra[0] - init_com[0], rel1 = b.tra[1] - init_com[1];
        const float r0 = c * rel0 - sn * rel1, r1 = sn * rel0 + c * rel1;
        b.tra[0] = init_com[0] + r0 * b.scale + b.linvel[0] * dt;
        b.tra[1] = init_com[1] + r1 * b.scale + b.linvel[1] * dt;
        const float nc = c * b.rot[0] - sn * b.rot[1], ns = sn * b.rot[0] + c * b.rot[1];
        b.rot[0] = nc;
        b.rot[1] = ns;
    }
    for (int k = 0; k < D; ++k) b.linvel[k] = b.linvel[k] + grav[k] * ((b.inv_mass[k] != 0.f) ? 1.f : 0.f) * dt;
    s.bodies[id] = b;
}
template <int D, bool B = false> __global__ void k_rigid(DevScene s) {
    pdl_enter();
    rigid_body<D, B>(s, blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace slosh
