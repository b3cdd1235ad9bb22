// Device view of one scene: every pointer the substep kernels read or
// write, passed by value to each kernel.
#pragma once

#include "common.cuh"

namespace slosh {

struct DevScene {
    // ---- particles (structure of arrays, math convention) -------------------
    // Storage is double-buffered: the substep reads the arrays below (in the
    // canonical order of the previous substep) and the fused G2P/update
    // writes the `out_*` arrays in this substep's canonical order.
    uint32_t n;            // plane stride of the particle arrays (pool capacity)
    uint32_t count;        // particles in storage (single-scene context; batches read *n_dev)
    float h;               // cell width
    float inv_h;           // 1 / h (exact when h_pow2)
    uint32_t h_pow2;       // h is a power of two
    float dt;
    float gravity[3];
    float4 *pm;            // (x, y, z, mass); 2D: (x, y, 0, mass)
    float4 *vv;            // (vx, vy, vz, C22); 2D: (vx, vy, 0, 0)
    float4 *cq;            // APIC matrix C, row-major elements 0-7 (0-3): MQ<D> float4 planes
    float4 *fq;            // deformation gradient F, same layout
    uint4 *fo;             // (flags: material id | enabled | fixed | scene slot, original index,
                           //  V0 bits, F22 bits (3D))
    float4 *ps;            // (plastic det, hardening q, log_vol_gain, damping)
    uint32_t *oid;         // copy of fo.y as its own plane for the grid build's sort keys
    float4 *out_pm, *out_vv, *out_cq, *out_fq, *out_ps;
    uint4 *out_fo;
    uint32_t *out_oid;
    float *fdt;            // D planes of force*dt in upload order, read by P2G while force_pending
    uint32_t has_damping;
    uint32_t has_sand;
    uint32_t force_pending;
    const Material *materials;

    // ---- sparse grid --------------------------------------------------------
    uint32_t cap;          // block capacity (power of two)
    uint32_t hcap;         // hash slots = 2 * cap
    uint32_t *hkeys;       // current substep hash map: packed keys
    uint32_t *hvals;       // current substep hash map: canonical block rank
    const uint32_t *prev_hkeys;
    const uint32_t *prev_hvals;
    // The previous substep's map is the next substep's current map: the
    // fused G2P/update clears it (and the key histogram) once k_grid_update,
    // its last reader, has run.
    uint32_t *clr_hkeys;
    uint32_t *clr_hvals;
    uint32_t clear_tail;
    uint32_t *slot_counts; // hcap * 64 per-cell particle counts per hash slot
    uint32_t *blist_key;   // primary blocks in append order [cap]
    uint32_t *blist_slot;
    uint32_t *blist2_key;  // neighbour-only blocks in append order [cap]
    uint32_t *blist2_slot;
    uint32_t *hist;        // HIST_BINS counts of key >> 16
    uint32_t *hist_start;  // their exclusive scan; k_bin_scatter advances it to the bins' ends
    uint32_t *hist_coarse; // HIST_COARSE counts of key >> 26
    uint32_t *tmp_key;     // [2 cap] keys grouped by key >> 16
    uint32_t *tmp_slot;
    uint32_t *bkey;        // canonical block order: packed key [cap]
    uint32_t *bslot;       // hash slot of the block
    uint32_t *bfirst;      // first primary entry in perm
    uint32_t *bnp;         // number of primary particles
    uint32_t *bcell;       // 64 per block: first entry of each cell, relative to bfirst
    uint32_t *bcur;        // 64 per block: insertion cursors, relative to bfirst
    uint32_t *qorder;      // ranks of the blocks, heaviest first: P2G's queue order
    uint2 *bord;           // 64 per block: cells by decreasing particle count (ties: cell index),
                           // each (cell | first << 6, count) with first relative to bfirst
    uint32_t *bnbh;        // (NASSOC - 1) neighbour ranks per block, NONE if inactive
    uint32_t *pslot;       // per particle: (hash slot << 6) | cell
    uint32_t *perm;        // primary order: scatter output, canonicalised in place
    unsigned long long *skey;  // beside perm: (cell << 32 | original id), the canonical sort key
    uint32_t *bnbh_rev;    // (NASSOC - 1) ranks of the blocks b - o (the -1 neighbours), NONE if inactive
    uint32_t *bprev;       // rank of the block in the previous substep's map (its collision cache), NONE if new
    float4 *nodes;         // 64 nodes per block: (momentum | velocity, mass)
    float4 *partial;       // TILE nodes per block: the block's own P2G sums over its (block + 2)^D tile
    uint32_t use_partial;  // P2G wrote `partial` (deterministic path); grid update gathers it
    uint32_t p2g_coop_below;  // P2G shares a block between a CTA's warps below this many blocks
    uint32_t p2g_heavy_first; // P2G takes blocks in `qorder` (heaviest first), else in rank order
    uint32_t gather_only;  // grid update stops after the gather (P2G node sums, debug)
    float4 *coll;          // node collision cache of this substep: (normal, d0)
    uint32_t *coll_id;     // collider id or NONE
    const float4 *prev_coll;
    const uint32_t *prev_coll_id;

    // ---- bodies -------------------------------------------------------------
    DevBody *bodies;
    uint32_t n_bodies;
    const float4 *mesh_vtx;        // triangle-mesh colliders: packed vertex and index buffers
    const uint32_t *mesh_idx;
    unsigned long long *body_imp;  // 6 fixed-point impulse sums per body (two-way coupling)
    uint32_t coll_dynamic;         // a two-way body moves: no collision cache

    Counters *ctr;
    uint32_t *err;

    // ---- grid reuse between substeps (single-scene context) -----------------
    // bfirst, bnp and bcell are double-buffered by substep parity: the prev_*
    // arrays hold the previous substep's, whose canonical order storage is in.
    uint32_t reuse;            // keep the previous grid when no particle changed it (else: full build)
    uint32_t par;              // parity of this substep (its rebuild flag)
    const uint32_t *prev_bfirst;
    const uint32_t *prev_bnp;
    const uint32_t *prev_bcell;
    int *cell_delta;           // 64 per block: particles gained - lost per cell, written by G2P
    unsigned long long *touch; // per block: cells a particle entered or left in G2P
    unsigned long long *cur_touch;  // per block: the touched cells this substep's reuse applies
    uint32_t *reuse_cta;       // [2 * REUSE_MAX_CTAS]: k_grid_reuse's per-CTA particle totals, then their scan
    uint32_t *touched_cells;   // [cap * 64]: (block << 6 | cell) of the cells a kept grid re-gathers
    uint32_t *bsrc;            // per block: storage index of its first particle when its particles are
                               // one shifted range of storage (a kept grid's untouched block), else NONE
    cudaGraphConditionalHandle cond;  // inside the substep graph: full build (1) or reuse (0)
    uint32_t use_cond;

    // ---- multi-scene batch (unused by the single-scene context) -------------
    // `n` is then the plane stride (pool capacity) and the particle count in
    // storage is *n_dev; blocks are hashed by (scene << 32 | key) in 64-bit
    // maps and ranked scene-major, ascending key within a scene.
    const SceneRec *scenes;
    uint32_t n_scenes;               // scene slots
    uint32_t *n_dev;
    unsigned long long *hkeys64;
    const unsigned long long *prev_hkeys64;
    unsigned long long *clr_hkeys64;
    uint32_t *bscene;                // scene of each ranked block
    uint32_t *scene_nblk;            // blocks per scene this substep
    uint32_t *scene_bbase;           // first block rank of each scene
    uint32_t *scene_fill;            // scatter cursors
    // fused substep's grid barrier: arrivals expected beyond the launch's
    // CTAs (0; a test sets more to make the wait run out) and its time
    // limit in ns (0: the default)
    uint32_t bar_extra;
    unsigned long long bar_ns;
    // G2P by scene class: the blocks of each class (G2P_CLASSES lists of
    // `cap`, appended by k_block_setup), g2p_counts[c] their number and
    // g2p_counts[G2P_CLASSES + c] the queue of class c's launch.  g2p_class:
    // the class this G2P launch takes (-1: every block, in rank order).
    uint32_t *g2p_lists;
    uint32_t *g2p_counts;
    int32_t g2p_class;
};

// This substep keeps the previous grid: the full build's kernels return at
// once (they also run under the conditional graph node that skips them).
__device__ __forceinline__ bool build_skipped(const DevScene &s) {
    return s.reuse != 0u && s.ctr->rebuild[s.par] == 0u;
}

}  // namespace slosh
