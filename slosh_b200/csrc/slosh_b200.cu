// C ABI of the B200-native slosh MPM substep: context lifetime, uploads and
// downloads, the substep launch sequence (captured once per parity as a CUDA
// graph) and the debug entry points used by the parity tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "grid_build.cuh"
#include "grid_reuse.cuh"
#include "io.cuh"
#include "transfer.cuh"
#include "timestep.cuh"
#include "fused.cuh"

using namespace slosh;

struct slosh_ctx {
    int dim = 3;
    float h = 0.f;
    uint32_t cap = 0, hcap = 0, max_n = 0, n = 0;
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    slosh_params params{};

    // particles: double-buffered storage in canonical order (buffer `parity`
    // holds the state the next substep reads) + upload-order side arrays
    struct Storage {
        float4 *pm = nullptr, *vv = nullptr, *cq = nullptr, *fq = nullptr, *ps = nullptr;
        uint4 *fo = nullptr;
        uint32_t *oid = nullptr;
    } pb[2];
    float *fdt = nullptr, *r0 = nullptr, *phase = nullptr;
    Material *materials = nullptr;
    uint32_t *mat_hkeys = nullptr, *mat_dense = nullptr;
    uint32_t has_damping = 0, force_pending = 0, has_sand = 0, n_materials = 0;
    uint32_t model_mask = 0;  // model tags present among the particles (bit = tag)

    // grid
    uint32_t *hkeys[2] = {nullptr, nullptr}, *hvals[2] = {nullptr, nullptr};
    uint32_t *slot_counts = nullptr, *blist_key = nullptr, *blist_slot = nullptr, *blist2_key = nullptr,
             *blist2_slot = nullptr, *hist = nullptr, *hist_start = nullptr, *hist_coarse = nullptr, *tmp_key = nullptr,
             *tmp_slot = nullptr, *bkey = nullptr, *bslot = nullptr, *bfirst = nullptr, *bnp = nullptr,
             *bcell = nullptr, *bcur = nullptr, *bnbh = nullptr, *bnbh_rev = nullptr;
    uint2 *bord = nullptr;
    uint32_t *qorder = nullptr, *bprev = nullptr;
    // grid reuse (single-scene contexts): the second parity's block arrays
    // and G2P's per-cell bookkeeping; reuse = 0 in batches and when the
    // environment sets SLOSH_GRID_REUSE=0
    uint32_t *bfirst2 = nullptr, *bnp2 = nullptr, *bcell2 = nullptr;
    int *cell_delta = nullptr;
    unsigned long long *touch = nullptr, *cur_touch = nullptr;
    uint32_t *reuse_cta = nullptr, *touched_cells = nullptr;
    uint32_t *bsrc = nullptr;  // per block: storage start of a shifted-range block, else NONE
    uint32_t reuse = 0;
    uint32_t reuse_mode = 2;  // SLOSH_GRID_REUSE: 0 off, 1 on, 2 (unset) on from REUSE_MIN_PARTICLES
    bool cond_graphs = false;  // the substep graphs pick the build through a conditional node
    // stage hooks (slosh's MpmPipelineHooks); while one is set, substeps are
    // launched kernel by kernel with the hooks called between the stages
    slosh_hook_fn hooks[SLOSH_HOOK_COUNT] = {};
    void *hook_user[SLOSH_HOOK_COUNT] = {};
    uint32_t n_hooks = 0;
    bool in_hook = false;
    uint32_t hook_point = 0;
    DevScene hook_scene{};  // the substep a hook runs in
    // P2G reduction (environment SLOSH_P2G at creation): 0 fixed-order,
    // bit-reproducible (default); 3 "direct": the same cell-owner kernel with
    // shared-memory and global float atomics, kept for A/B comparison.
    int p2g_variant = 0;
    uint32_t g2p_threads = 0;  // G2P CTA size, 0: chosen by the scene size (SLOSH_G2P_THREADS)
    // Programmatic dependent launch inside the substep graphs (SLOSH_PDL=0
    // turns it off).  pdl_capture: a substep graph is being captured;
    // pdl_link: the previous operation captured on the stream is a kernel.
    bool pdl = true, pdl_capture = false, pdl_link = false;
    uint32_t *pslot = nullptr, *perm = nullptr;
    unsigned long long *skey = nullptr;
    float4 *nodes = nullptr, *partial = nullptr, *coll[2] = {nullptr, nullptr};
    uint32_t *coll_id[2] = {nullptr, nullptr};

    DevBody *bodies = nullptr;
    uint32_t n_bodies = 0;
    unsigned long long *body_imp = nullptr;  // two-way coupling impulse sums, 6 per body slot
    uint32_t coll_dynamic = 0;               // some body is coupled two-way
    // triangle-mesh colliders: host copies of the packed buffers and their
    // device copies, re-uploaded whole when a mesh is added
    std::vector<float4> mesh_vtx_host;
    std::vector<uint32_t> mesh_idx_host;
    float4 *mesh_vtx = nullptr;
    uint32_t *mesh_idx = nullptr;
    uint32_t n_meshes = 0;
    Counters *ctr = nullptr;
    uint32_t *err = nullptr;
    uint32_t *small = nullptr;  // [0] n_mat, [1] scene flags, [2] debug total
    uint32_t parity = 0;

    slosh_particle *staging = nullptr;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graphs_valid = false;

    std::string last_error;
    std::vector<void *> allocs;
};

namespace {

int fail(slosh_ctx *c, int code, const char *fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        c->last_error = buf;
    }
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(c, SLOSH_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Launches one kernel of the substep.  While a substep graph is captured and
// the previous operation captured on the stream is a kernel, the launch
// carries cudaLaunchAttributeProgrammaticStreamSerialization: the graph edge
// between the two becomes programmatic, and the kernel's CTAs are scheduled
// once all of its predecessor's CTAs have started, instead of after the
// predecessor has drained and the graph has processed its completion.  The
// kernel itself waits in pdl_enter() for that completion, so the results are
// the same bits.
template <typename... P, typename... A>
void launch_k(slosh_ctx *c, uint32_t grid, uint32_t block, size_t smem, cudaStream_t st, void (*k)(P...), A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = c->pdl_capture && c->pdl_link ? 1u : 0u;
    cudaLaunchKernelEx(&cfg, k, args...);
    c->pdl_link = c->pdl_capture;
}

template <typename T> int dalloc(slosh_ctx *c, T **p, size_t count) {
    void *q = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, SLOSH_E_NOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    c->allocs.push_back(q);
    *p = (T *)q;
    return SLOSH_OK;
}

// One particle storage buffer (128 bytes a particle in 3D).
int alloc_storage(slosh_ctx *c, slosh_ctx::Storage &S, size_t N, int D) {
    const size_t Q = D == 3 ? 2 : 1;
    int st;
    if ((st = dalloc(c, &S.pm, N)) || (st = dalloc(c, &S.vv, N)) || (st = dalloc(c, &S.cq, N * Q)) ||
        (st = dalloc(c, &S.fq, N * Q)) || (st = dalloc(c, &S.ps, N)) || (st = dalloc(c, &S.fo, N)) ||
        (st = dalloc(c, &S.oid, N)))
        return st;
    cudaMemset(S.ps, 0, N * sizeof(float4));
    return SLOSH_OK;
}

uint32_t next_pow2(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

int nnb(int dim) { return dim == 3 ? Geo<3>::NASSOC - 1 : Geo<2>::NASSOC - 1; }
int nbk(int dim) { return dim == 3 ? Geo<3>::NB : Geo<2>::NB; }

// Scenes below this many particles have too few blocks to fill the transfer
// kernels' persistent grids: G2P then runs CTAs of 256 (a block in one
// round) and P2G takes blocks in rank order (with no more blocks than warps
// the heaviest-first order balances nothing and its bucket sort is saved).
constexpr uint32_t G2P_SMALL_PARTICLES = 262144;
constexpr uint32_t P2G_WIDE_PARTICLES = 1048576;  // P2G in CTAs of six warps below this

DevScene make_scene(slosh_ctx *c, uint32_t parity, bool force) {
    DevScene s{};
    s.n = c->max_n;
    s.count = c->n;
    s.h = c->h;
    s.inv_h = 1.0f / c->h;
    {
        int ex = 0;
        s.h_pow2 = (std::frexp(c->h, &ex) == 0.5f) ? 1u : 0u;
    }
    s.dt = c->params.dt;
    for (int k = 0; k < 3; ++k) s.gravity[k] = c->params.gravity[k];
    const slosh_ctx::Storage &A = c->pb[parity & 1u], &B = c->pb[(parity & 1u) ^ 1u];
    s.pm = A.pm;
    s.vv = A.vv;
    s.cq = A.cq;
    s.fq = A.fq;
    s.ps = A.ps;
    s.fo = A.fo;
    s.oid = A.oid;
    s.out_pm = B.pm;
    s.out_vv = B.vv;
    s.out_cq = B.cq;
    s.out_fq = B.fq;
    s.out_ps = B.ps;
    s.out_fo = B.fo;
    s.out_oid = B.oid;
    s.fdt = c->fdt;
    s.has_damping = c->has_damping;
    s.has_sand = c->has_sand;
    s.force_pending = force ? 1u : 0u;
    s.materials = c->materials;
    s.cap = c->cap;
    s.hcap = c->hcap;
    const uint32_t cur = parity & 1u, prv = cur ^ 1u;
    s.hkeys = c->hkeys[cur];
    s.hvals = c->hvals[cur];
    s.prev_hkeys = c->hkeys[prv];
    s.prev_hvals = c->hvals[prv];
    s.slot_counts = c->slot_counts;
    s.blist_key = c->blist_key;
    s.blist_slot = c->blist_slot;
    s.blist2_key = c->blist2_key;
    s.blist2_slot = c->blist2_slot;
    s.hist = c->hist;
    s.hist_start = c->hist_start;
    s.hist_coarse = c->hist_coarse;
    s.tmp_key = c->tmp_key;
    s.tmp_slot = c->tmp_slot;
    s.bkey = c->bkey;
    s.bslot = c->bslot;
    {
        // block arrays of this parity and of the previous substep
        const uint32_t pc = parity & 1u;
        uint32_t *bf[2] = {c->bfirst, c->bfirst2 ? c->bfirst2 : c->bfirst};
        uint32_t *bn[2] = {c->bnp, c->bnp2 ? c->bnp2 : c->bnp};
        uint32_t *bc[2] = {c->bcell, c->bcell2 ? c->bcell2 : c->bcell};
        s.bfirst = bf[pc];
        s.bnp = bn[pc];
        s.bcell = bc[pc];
        s.prev_bfirst = bf[pc ^ 1u];
        s.prev_bnp = bn[pc ^ 1u];
        s.prev_bcell = bc[pc ^ 1u];
        s.reuse = c->reuse;
        s.par = pc;
        s.cell_delta = c->cell_delta;
        s.touch = c->touch;
        s.cur_touch = c->cur_touch;
        s.reuse_cta = c->reuse_cta;
        s.touched_cells = c->touched_cells;
        s.bsrc = c->bsrc;
        s.cond = 0;
        s.use_cond = 0u;
    }
    s.bord = c->bord;
    s.qorder = c->qorder;
    s.bcur = c->bcur;
    s.bnbh = c->bnbh;
    s.bnbh_rev = c->bnbh_rev;
    s.bprev = c->bprev;
    s.pslot = c->pslot;
    s.perm = c->perm;
    s.skey = c->skey;
    s.nodes = c->nodes;
    s.partial = c->partial;
    s.use_partial = (c->p2g_variant == 0) ? 1u : 0u;
    s.gather_only = 0u;
    // P2G: one warp a block fills the GPU from about 10 blocks an SM; below
    // that a CTA's warps share each block.  Scenes below P2G_WIDE_PARTICLES
    // run CTAs of six warps (3 an SM), which share blocks up to about 5
    // blocks a CTA (16 an SM): one pass a warp beats six passes a warp there
    s.p2g_coop_below = c->n < P2G_WIDE_PARTICLES ? (uint32_t)c->sm_count * 16u : (uint32_t)c->sm_count * 10u;
    s.p2g_heavy_first = c->n >= G2P_SMALL_PARTICLES ? 1u : 0u;
    s.coll = c->coll[cur];
    s.coll_id = c->coll_id[cur];
    s.prev_coll = c->coll[prv];
    s.prev_coll_id = c->coll_id[prv];
    s.bodies = c->bodies;
    s.n_bodies = c->n_bodies;
    s.body_imp = c->body_imp;
    s.coll_dynamic = c->coll_dynamic;
    s.mesh_vtx = c->mesh_vtx;
    s.mesh_idx = c->mesh_idx;
    s.ctr = c->ctr;
    s.err = c->err;
    s.clr_hkeys = c->hkeys[prv];
    s.clr_hvals = c->hvals[prv];
    s.clear_tail = 1u;
    return s;
}

uint32_t grid_for(uint64_t work, uint32_t threads, uint32_t max_ctas) {
    const uint64_t g = (work + threads - 1) / threads;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, max_ctas));
}

// Kernels of one substep, in launch order (profiling names).
constexpr int N_KERNELS = 16;
const char *const KERNEL_NAMES[N_KERNELS] = {
    "k_grid_reuse", "k_touch",      "k_neighbors",   "k_hist_scan", "k_bin_scatter", "k_rank",
    "k_block_setup", "k_block_scan", "k_reuse_perm", "k_reuse_cells", "k_scatter",   "k_canon",
    "k_p2g",        "k_grid_update", "k_g2p_update", "k_rigid"};

// Optional per-kernel CUDA-event timing of the substep launches.
struct Prof {
    cudaEvent_t ev[N_KERNELS][2];
    bool used[N_KERNELS];
    cudaStream_t st;
    void begin(int k) {
        used[k] = true;
        cudaEventRecord(ev[k][0], st);
    }
    void end(int k) { cudaEventRecord(ev[k][1], st); }
};

#define PROF_BEGIN(k) \
    if (p) p->begin(k)
#define PROF_END(k) \
    if (p) p->end(k)

// Grid build of one substep (stages shared by the substep and the debug
// entry points).  Within a substep sequence the hash map, key histogram and
// counters were cleared by the previous substep's last kernels (or by the
// upload); a standalone build (debug entry points) clears them first.
// front: activation and ranking of the blocks and their cell counts.
template <int D> void enqueue_build_front(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    const uint32_t sm = (uint32_t)c->sm_count;
    PROF_BEGIN(1);
    launch_k(c, grid_for(c->n, 256, sm * 8), 256, 0, st, k_touch<D>, s);  // one wave of warps, a chunk each
    PROF_END(1);
    PROF_BEGIN(2);
    launch_k(c, grid_for((uint64_t)c->cap * (Geo<D>::NASSOC - 1), 256, sm * 8), 256, 0, st, k_neighbors<D>, s);
    PROF_END(2);
    PROF_BEGIN(3);
    launch_k(c, HIST_COARSE, 256, 0, st, k_hist_scan<256>, s);
    PROF_END(3);
    PROF_BEGIN(4);
    launch_k(c, grid_for(2ull * c->cap, 256, sm * 8), 256, 0, st, k_bin_scatter, s);
    PROF_END(4);
    PROF_BEGIN(5);
    launch_k(c, grid_for(2ull * c->cap * RANK_LANES, 256, sm * 8), 256, 0, st, k_rank, s);
    PROF_END(5);
    PROF_BEGIN(6);
    launch_k(c, grid_for((uint64_t)c->cap * 32, 256, sm * 16), 256, 0, st, k_block_setup<D>, s);
    PROF_END(6);
}

void enqueue_block_scan(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    PROF_BEGIN(7);
    launch_k(c, 1, 1024, 0, st, k_block_scan<1024>, s);
    PROF_END(7);
}

// The kept grid's permutation and its touched cells (both return at once
// when the full build runs).
template <int D> void enqueue_reuse_perm(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    PROF_BEGIN(8);
    launch_k(c, grid_for((uint64_t)c->cap * 32, 256, (uint32_t)c->sm_count * 8), 256, 0, st, k_reuse_perm<D>, s);
    PROF_END(8);
    PROF_BEGIN(9);
    launch_k(c, (uint32_t)c->sm_count * 8, 256, 0, st, k_reuse_cells<D>, s);
    PROF_END(9);
}

// back: the permutation of the full build.
void enqueue_build_back(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    const uint32_t sm = (uint32_t)c->sm_count;
    PROF_BEGIN(10);
    launch_k(c, grid_for(c->n, 256, sm * 8), 256, 0, st, k_scatter<false>, s);  // longer chunks: fewer cells split for k_canon
    PROF_END(10);
    PROF_BEGIN(11);
    launch_k(c, grid_for((uint64_t)c->cap * 32, 256, sm * 16), 256, 0, st, k_canon, s);
    PROF_END(11);
}

// The decision between keeping the previous grid and a full build.
template <int D> void enqueue_reuse_decision(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    PROF_BEGIN(0);
    const uint32_t ctas = std::min<uint32_t>((uint32_t)c->sm_count * 8, REUSE_MAX_CTAS);
    launch_k(c, grid_for((uint64_t)c->cap * 32, 256, ctas), 256, 0, st, k_grid_reuse<D>, s);
    PROF_END(0);
}

// A whole grid build as one launch sequence.  With grid reuse on, the full
// build's kernels and the reuse permutation each return at once unless the
// substep's decision selects them; standalone builds run with reuse off.
template <int D>
void enqueue_grid_build(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p = nullptr, bool standalone = false) {
    if (standalone) launch_k(c, (uint32_t)c->sm_count * 4, 256, 0, st, k_clear<false>, s);
    enqueue_build_front<D>(c, s, st, p);
    enqueue_block_scan(c, s, st, p);
    if (s.reuse) enqueue_reuse_perm<D>(c, s, st, p);
    enqueue_build_back(c, s, st, p);
}

template <int D> void enqueue_p2g(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p = nullptr) {
    PROF_BEGIN(12);
    if (c->p2g_variant == 3) {
        const uint32_t g = std::min<uint32_t>(c->cap, (uint32_t)c->sm_count * 8);
        launch_k(c, g, P2G_ATOMIC_THREADS, 0, st, k_p2g_atomic<D>, s);
    } else {
        if (c->n < P2G_WIDE_PARTICLES) {
            // a small scene: CTAs of six warps, one pass of a shared block each
            const uint32_t g = std::min<uint32_t>(c->cap, (uint32_t)c->sm_count * 3);
            constexpr size_t smem = sizeof(P2gSmem<D, 3, P2G_WIDE_WARPS>);
            if (s.force_pending) launch_k(c, g, 32 * P2G_WIDE_WARPS, smem, st, k_p2g_wide<D, true>, s);
            else launch_k(c, g, 32 * P2G_WIDE_WARPS, smem, st, k_p2g_wide<D, false>, s);
        } else {
            const uint32_t g = std::min<uint32_t>((c->cap + P2G_WARPS - 1) / P2G_WARPS, (uint32_t)c->sm_count * 5);
            if (s.force_pending) launch_k(c, g, 32 * P2G_WARPS, 0, st, k_p2g<D, false, true>, s);
            else launch_k(c, g, 32 * P2G_WARPS, 0, st, k_p2g<D>, s);
        }
    }
    PROF_END(12);
}

template <int D> void enqueue_grid_update(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p = nullptr) {
    PROF_BEGIN(13);
    launch_k(c, grid_for((uint64_t)c->cap * 64, 256, (uint32_t)c->sm_count * 16), 256, 0, st, k_grid_update<D>, s);
    PROF_END(13);
}

// Restores the cleared state a debug build consumed, so that the next real
// substep starts from a cleared hash map and counters.
void enqueue_clear(slosh_ctx *c, const DevScene &s, cudaStream_t st) {
    launch_k(c, (uint32_t)c->sm_count * 4, 256, 0, st, k_clear<false>, s);
}

// P2G, grid update, fused G2P/update and the rigid update.
// Instantiated for a power-of-two cell width and, with it, for scenes of a
// single model among the linear elastic, sand and fluid ones.
template <int D, int NT> void launch_g2p(slosh_ctx *c, const DevScene &s, cudaStream_t st) {
    const uint32_t g2p_grid = std::min<uint32_t>(c->cap, (uint32_t)c->sm_count * (512u / NT));
    if (!s.h_pow2) launch_k(c, g2p_grid, NT, 0, st, k_g2p_update<D, NT, false, false>, s);
    else if (c->model_mask == 1u << SLOSH_MODEL_SAND_LINEAR)
        launch_k(c, g2p_grid, NT, 0, st, k_g2p_update<D, NT, false, true, SLOSH_MODEL_SAND_LINEAR>, s);
    else if (c->model_mask == 1u << SLOSH_MODEL_ELASTIC_LINEAR)
        launch_k(c, g2p_grid, NT, 0, st, k_g2p_update<D, NT, false, true, SLOSH_MODEL_ELASTIC_LINEAR>, s);
    else if (c->model_mask == 1u << SLOSH_MODEL_FLUID_TAIT)
        launch_k(c, g2p_grid, NT, 0, st, k_g2p_update<D, NT, false, true, SLOSH_MODEL_FLUID_TAIT>, s);
    else launch_k(c, g2p_grid, NT, 0, st, k_g2p_update<D, NT, false, true>, s);
}

// Persistent CTAs taking blocks from the queue.  A large scene runs 8 CTAs
// of 64 an SM: small CTAs wait less at the per-block barriers (tile load,
// the slowest thread's last particle).  A small scene has too few blocks to
// fill those CTAs, and a CTA of 64 takes several rounds for one block in
// sequence; there CTAs of 256 (2 an SM) take a block in one round.
// SLOSH_G2P_THREADS (64, 128 or 256) overrides the choice.
template <int D> void enqueue_g2p(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    PROF_BEGIN(14);
    const uint32_t nt = c->g2p_threads ? c->g2p_threads : (c->n < G2P_SMALL_PARTICLES ? 256u : 64u);
    if (nt == 256u) launch_g2p<D, 256>(c, s, st);
    else if (nt == 128u) launch_g2p<D, 128>(c, s, st);
    else launch_g2p<D, 64>(c, s, st);
    PROF_END(14);
}

template <int D> void enqueue_transfer(slosh_ctx *c, const DevScene &s, cudaStream_t st, Prof *p) {
    enqueue_p2g<D>(c, s, st, p);
    enqueue_grid_update<D>(c, s, st, p);
    enqueue_g2p<D>(c, s, st, p);
    PROF_BEGIN(15);
    launch_k(c, 1, 32, 0, st, k_rigid<D>, s);
    PROF_END(15);
}

template <int D>
void enqueue_substep(slosh_ctx *c, cudaStream_t st, uint32_t parity, bool force, Prof *p = nullptr) {
    const DevScene s = make_scene(c, parity, force);
    if (s.reuse) enqueue_reuse_decision<D>(c, s, st, p);
    enqueue_grid_build<D>(c, s, st, p);
    enqueue_transfer<D>(c, s, st, p);
}

void enqueue_substep_any(slosh_ctx *c, cudaStream_t st, uint32_t parity, bool force, Prof *p = nullptr) {
    if (c->dim == 3) enqueue_substep<3>(c, st, parity, force, p);
    else enqueue_substep<2>(c, st, parity, force, p);
}

// Makes the next substep run the full grid build: after an upload, an
// append or removal, or a standalone build (debug entry points), the
// previous substep's grid no longer describes storage.  G2P's pending
// per-cell bookkeeping is dropped with it.
int force_grid_rebuild(slosh_ctx *c, cudaStream_t st) {
    if (!c->cell_delta) return SLOSH_OK;  // batches keep no bookkeeping
    CK(cudaMemsetAsync(c->cell_delta, 0, (size_t)c->cap * CELLS * sizeof(int), st));
    CK(cudaMemsetAsync(c->touch, 0, (size_t)c->cap * sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(c->ctr->rebuild, 1, sizeof(c->ctr->rebuild), st));  // nonzero: rebuild
    return SLOSH_OK;
}

// Grid reuse pays once the grid build's kernels outweigh the reuse's own
// launches: scenes below this many particles are launch-bound, and their
// full build inside the substep graph is faster (measured: the 62,628-
// particle dam break at 0.054 ms a substep with the full build, 0.061 with
// reuse; the 524,288-particle elastic drop 0.152 and 0.147).
constexpr uint32_t REUSE_MIN_PARTICLES = 262144;

void destroy_graphs(slosh_ctx *c);

// Sets whether substeps keep their grid, from the mode and the particle
// count; the graphs are rebuilt when that changes.
void update_reuse(slosh_ctx *c) {
    const uint32_t want = c->reuse_mode == 1 || (c->reuse_mode == 2 && c->n >= REUSE_MIN_PARTICLES) ? 1u : 0u;
    if (want != c->reuse) {
        c->reuse = want;
        destroy_graphs(c);
    }
}

// One substep with the stage hooks called between its kernels, in the
// order of slosh's launch_step (src/pipeline.rs:562-770).
int call_hook(slosh_ctx *c, const DevScene &s, uint32_t pt, cudaStream_t st) {
    if (!c->hooks[pt]) return 0;
    c->in_hook = true;
    c->hook_point = pt;
    c->hook_scene = s;
    const int r = c->hooks[pt](c, pt, (void *)st, c->hook_user[pt]);
    c->in_hook = false;
    return r;
}

template <int D> int enqueue_substep_hooked(slosh_ctx *c, cudaStream_t st, uint32_t parity, bool force) {
    const DevScene s = make_scene(c, parity, force);
    // A hook that fails drops the substep: storage (the input planes) is
    // untouched, and the grid state is reset so that the substep can run
    // again from a full build.
    auto drop = [&](int code) {
        launch_k(c, (uint32_t)c->sm_count * 4, 256, 0, st, k_clear<false>, s);
        force_grid_rebuild(c, st);
        return code;
    };
    if (s.reuse) enqueue_reuse_decision<D>(c, s, st, nullptr);
    enqueue_grid_build<D>(c, s, st);
    int r = call_hook(c, s, SLOSH_HOOK_AFTER_PARTICLE_SORT, st);
    if (r < 0) return drop(r);
    // P2G; the grid update reads node sums from `nodes` when a hook wrote or
    // may change them (the sums land there bit for bit as the update's own
    // gather computes them)
    r = call_hook(c, s, SLOSH_HOOK_RUN_P2G, st);
    if (r < 0) return drop(r);
    const bool p2g_replaced = r == 1;
    DevScene from_nodes = s;
    from_nodes.use_partial = 0u;
    if (!p2g_replaced) {
        enqueue_p2g<D>(c, s, st);
        if (c->hooks[SLOSH_HOOK_AFTER_P2G]) {
            DevScene gather = s;
            gather.gather_only = 1u;
            enqueue_grid_update<D>(c, gather, st);
        }
    }
    if ((r = call_hook(c, s, SLOSH_HOOK_AFTER_P2G, st)) < 0) return drop(r);
    const bool via_nodes = p2g_replaced || c->hooks[SLOSH_HOOK_AFTER_P2G] != nullptr;
    enqueue_grid_update<D>(c, via_nodes ? from_nodes : s, st);
    if ((r = call_hook(c, s, SLOSH_HOOK_AFTER_GRID_UPDATE, st)) < 0) return drop(r);
    r = call_hook(c, s, SLOSH_HOOK_RUN_G2P, st);
    if (r < 0) return drop(r);
    if (r == 1) {
        // a replaced update records no cell changes: the next substep rebuilds
        launch_k(c, (uint32_t)c->sm_count * 4, 256, 0, st, k_after_replaced_g2p, s);
        if (c->reuse && cudaMemsetAsync(&c->ctr->rebuild[s.par ^ 1u], 1, 4, st) != cudaSuccess) return SLOSH_E_CUDA;
    } else {
        enqueue_g2p<D>(c, s, st, nullptr);
    }
    if ((r = call_hook(c, s, SLOSH_HOOK_AFTER_G2P, st)) < 0) return drop(r);
    if ((r = call_hook(c, s, SLOSH_HOOK_AFTER_PARTICLES_UPDATE, st)) < 0) return drop(r);
    launch_k(c, 1, 32, 0, st, k_rigid<D>, s);
    return cudaGetLastError() == cudaSuccess ? SLOSH_OK : SLOSH_E_CUDA;
}

void destroy_graphs(slosh_ctx *c) {
    for (int k = 0; k < 2; ++k)
        if (c->graph[k]) {
            cudaGraphExecDestroy(c->graph[k]);
            c->graph[k] = nullptr;
        }
    c->graphs_valid = false;
}

// Substep graph with the grid build under a conditional node: the reuse
// decision, then IF (full build) ELSE (reuse permutation), then the transfer
// kernels.  Only the selected branch's kernels launch.
template <int D> cudaError_t capture_conditional(slosh_ctx *c, uint32_t par, cudaGraph_t *out) {
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
    cudaStream_t st = c->stream;
    *out = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return e;
    auto bail = [&](cudaError_t err) {
        cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(st, &cst) == cudaSuccess && cst != cudaStreamCaptureStatusNone) {
            cudaGraph_t left = nullptr;  // the graph being captured into: destroyed below (or owned by g)
            cudaStreamEndCapture(st, &left);
        }
        cudaGraphDestroy(g);
        return err;
    };
    cudaGraphConditionalHandle handle = 0;
    if ((e = cudaGraphConditionalHandleCreate(&handle, g, 1u, cudaGraphCondAssignDefault)) != cudaSuccess) return bail(e);
    DevScene s = make_scene(c, par, false);
    s.cond = handle;
    s.use_cond = 1u;
    // the decision
    if ((e = cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, mode)) != cudaSuccess) return bail(e);
    c->pdl_link = false;
    enqueue_reuse_decision<D>(c, s, st, nullptr);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, nullptr, &deps, &nd);
    cudaGraphNode_t decision = (e == cudaSuccess && nd == 1) ? deps[0] : nullptr;
    cudaGraph_t captured = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &captured);
    if (e != cudaSuccess) return bail(e);
    if (e2 != cudaSuccess) return bail(e2);
    if (!decision) return bail(cudaErrorInvalidValue);
    // IF rebuild: the full build; ELSE: the reuse
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 2;
    cudaGraphNode_t cnode = nullptr;
    if ((e = cudaGraphAddNode(&cnode, g, &decision, 1, &cp)) != cudaSuccess) return bail(e);
    cudaGraph_t full = cp.conditional.phGraph_out[0], reuse = cp.conditional.phGraph_out[1];
    if ((e = cudaStreamBeginCaptureToGraph(st, full, nullptr, nullptr, 0, mode)) != cudaSuccess) return bail(e);
    c->pdl_link = false;
    enqueue_build_front<D>(c, s, st, nullptr);
    enqueue_block_scan(c, s, st, nullptr);
    enqueue_build_back(c, s, st, nullptr);
    if ((e = cudaStreamEndCapture(st, &full)) != cudaSuccess) return bail(e);
    if ((e = cudaStreamBeginCaptureToGraph(st, reuse, nullptr, nullptr, 0, mode)) != cudaSuccess) return bail(e);
    c->pdl_link = false;
    enqueue_reuse_perm<D>(c, s, st, nullptr);
    if ((e = cudaStreamEndCapture(st, &reuse)) != cudaSuccess) return bail(e);
    // the transfer kernels after either branch
    if ((e = cudaStreamBeginCaptureToGraph(st, g, &cnode, nullptr, 1, mode)) != cudaSuccess) return bail(e);
    c->pdl_link = false;  // after the conditional node
    enqueue_transfer<D>(c, s, st, nullptr);
    if ((e = cudaStreamEndCapture(st, &captured)) != cudaSuccess) return bail(e);
    *out = g;
    return cudaSuccess;
}

int build_graphs_once(slosh_ctx *c) {
    destroy_graphs(c);
    c->cond_graphs = false;
    if (c->reuse) {
        // the grid build under a conditional node; on any failure the plain
        // sequence below (every kernel, the unused ones returning at once)
        cudaGraph_t g[2] = {nullptr, nullptr};
        bool ok = true;
        for (uint32_t par = 0; par < 2 && ok; ++par) {
            const cudaError_t e = c->dim == 3 ? capture_conditional<3>(c, par, &g[par]) : capture_conditional<2>(c, par, &g[par]);
            ok = e == cudaSuccess && cudaGraphInstantiate(&c->graph[par], g[par], 0) == cudaSuccess;
        }
        for (auto &x : g)
            if (x) cudaGraphDestroy(x);
        if (ok) {
            c->cond_graphs = true;
            c->graphs_valid = true;
            return SLOSH_OK;
        }
        destroy_graphs(c);
        cudaGetLastError();  // the failed capture is not the caller's error
    }
    for (uint32_t par = 0; par < 2; ++par) {
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->pdl_link = false;
        enqueue_substep_any(c, c->stream, par, false);
        cudaGraph_t g = nullptr;
        CK(cudaStreamEndCapture(c->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&c->graph[par], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(c, SLOSH_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    }
    c->graphs_valid = true;
    return SLOSH_OK;
}

// The substep graphs, with programmatic edges between consecutive kernels
// unless SLOSH_PDL=0; a runtime that refuses those captures gets the graphs
// with plain edges.
int build_graphs(slosh_ctx *c) {
    c->pdl_capture = c->pdl;
    int r = build_graphs_once(c);
    // a grid-reusing scene prefers the conditional graph with plain edges to
    // the unconditional one with programmatic edges
    if (c->pdl && (r != SLOSH_OK || (c->reuse && !c->cond_graphs))) {
        cudaGetLastError();
        c->pdl = false;
        c->pdl_capture = false;
        r = build_graphs_once(c);
    }
    c->pdl_capture = false;
    c->pdl_link = false;
    return r;
}

int check_device_error(slosh_ctx *c) {
    uint32_t e = 0;
    CK(cudaMemcpy(&e, c->err, 4, cudaMemcpyDeviceToHost));
    if (e == 0) return SLOSH_OK;
    CK(cudaMemset(c->err, 0, 4));
    if (e & (ERR_HASH_OVERFLOW | ERR_BLOCK_OVERFLOW))
        return fail(c, SLOSH_E_OVERFLOW, "active blocks exceed the grid capacity %u (error bits 0x%x)", c->cap, e);
    if (e & ERR_BLOCK_PARTICLES)
        return fail(c, SLOSH_E_OVERFLOW, "a block holds 2^26 particles or more (error bits 0x%x)", e);
    if (e & ERR_KEY_RANGE)
        return fail(c, SLOSH_E_OVERFLOW, "a particle left the packed block-key range (error bits 0x%x)", e);
    if (e & ERR_GRID_REUSE)
        return fail(c, SLOSH_E_STATE, "a kept grid's cell counts and gathered cells disagree (error bits 0x%x)", e);
    if (e & (ERR_MATERIALS | ERR_MATERIAL_HASH))
        return fail(c, SLOSH_E_MATERIAL, "material table error (bits 0x%x; max %u materials)", e, MAX_MATERIALS);
    return fail(c, SLOSH_E_CUDA, "device error bits 0x%x", e);
}

cudaStream_t pick(slosh_ctx *c, void *stream) { return stream ? (cudaStream_t)stream : c->stream; }

void to_dev_body(const slosh_body &b, DevBody &d, int dim) {
    std::memset(&d, 0, sizeof(d));
    std::memcpy(&d.shape_type, &b.shape_a[3], 4);
    for (int k = 0; k < 4; ++k) {
        d.sa[k] = b.shape_a[k];
        d.sb[k] = b.shape_b[k];
        d.rot[k] = b.rotation[k];
    }
    for (int k = 0; k < 3; ++k) {
        d.tra[k] = b.translation[k];
        d.linvel[k] = b.linvel[k];
        d.angvel[k] = b.angvel[k];
        d.inv_mass[k] = b.inv_mass[k];
        d.local_com[k] = b.local_com[k];
    }
    d.scale = b.translation[3];
    d.bc_type = b.bc_type;
    d.friction = b.bc_friction;
    d.coupling = b.coupling;
    // the record's world-space inverse inertia, taken to the body frame (a
    // 2D scalar is frame-independent)
    if (dim == 3) {
        float W[9], R[3][3];
        for (int r = 0; r < 3; ++r)
            for (int col = 0; col < 3; ++col) W[r * 3 + col] = b.inv_inertia[col * 4 + r];
        quat_matrix(b.rotation, R);
        rotate_tensor(R, W, d.inv_inertia, false);
    } else {
        d.inv_inertia[0] = b.inv_inertia[0];
    }
}

// Collider shapes the projection handles: ball, cuboid and capsule in 2D and
// 3D; cylinder and cone in 3D (shaders/slosh/rbd/shapes/shape.slang:99-125).
bool shape_supported(uint32_t ty, int dim) {
    if (ty == SLOSH_SHAPE_BALL || ty == SLOSH_SHAPE_CUBOID || ty == SLOSH_SHAPE_CAPSULE) return true;
    return dim == 3 && (ty == SLOSH_SHAPE_CYLINDER || ty == SLOSH_SHAPE_CONE);
}

// A trimesh shape record names a mesh of this context's buffers.
bool trimesh_in_range(const slosh_ctx *c, const DevBody &d) {
    const TriMeshRef m = trimesh_ref(d.sa, d.sb);
    return m.ordinal < c->n_meshes &&
           (uint64_t)m.vtx_root + 2ull * m.n_nodes + 2ull * m.n_verts + 3ull * m.n_tris <= c->mesh_vtx_host.size() &&
           (uint64_t)m.idx_root + 3ull * m.n_nodes + 3ull * m.n_tris <= c->mesh_idx_host.size();
}

void from_dev_body(const DevBody &d, slosh_body &b, int dim) {
    std::memset(&b, 0, sizeof(b));
    for (int k = 0; k < 4; ++k) {
        b.shape_a[k] = d.sa[k];
        b.shape_b[k] = d.sb[k];
        b.rotation[k] = d.rot[k];
    }
    std::memcpy(&b.shape_a[3], &d.shape_type, 4);
    for (int k = 0; k < 3; ++k) {
        b.translation[k] = d.tra[k];
        b.linvel[k] = d.linvel[k];
        b.angvel[k] = d.angvel[k];
        b.inv_mass[k] = d.inv_mass[k];
        b.local_com[k] = d.local_com[k];
    }
    b.translation[3] = d.scale;
    b.bc_type = d.bc_type;
    b.bc_friction = d.friction;
    b.coupling = d.coupling;
    if (dim == 3) {  // world-space inverse inertia at the current pose
        float W[9], R[3][3];
        quat_matrix(d.rot, R);
        rotate_tensor(R, d.inv_inertia, W, true);
        for (int r = 0; r < 3; ++r)
            for (int col = 0; col < 3; ++col) b.inv_inertia[col * 4 + r] = W[r * 3 + col];
    } else {
        b.inv_inertia[0] = d.inv_inertia[0];
    }
}

// Frees the device resources of a context (not the object itself).
void release_ctx(slosh_ctx *c) {
    cudaSetDevice(c->device);
    destroy_graphs(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void *p : c->allocs) cudaFree(p);
    c->allocs.clear();
    cudaFree(c->mesh_vtx);
    cudaFree(c->mesh_idx);
    c->mesh_vtx = nullptr;
    c->mesh_idx = nullptr;
    if (c->stream) cudaStreamDestroy(c->stream);
    c->stream = nullptr;
}

}  // namespace

extern "C" {

int slosh_ctx_create(const slosh_config *cfg, slosh_ctx **out) {
    if (!cfg || !out) return SLOSH_E_INVALID;
    *out = nullptr;
    if ((cfg->dim != 2 && cfg->dim != 3) || !(cfg->cell_width > 0.f) || cfg->grid_capacity == 0 ||
        cfg->max_particles == 0 || cfg->grid_capacity > (1u << 24))
        return SLOSH_E_INVALID;
    slosh_ctx *c = new slosh_ctx();
    c->dim = (int)cfg->dim;
    c->h = cfg->cell_width;
    c->cap = next_pow2(cfg->grid_capacity);
    c->hcap = 2 * c->cap;
    c->max_n = cfg->max_particles;
    c->device = cfg->device;
    int st = SLOSH_OK;
    auto fail_create = [&](int code) {
        slosh_ctx_destroy(c);
        return code;
    };
    if (cudaSetDevice(c->device) != cudaSuccess) return fail_create(SLOSH_E_CUDA);
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail_create(SLOSH_E_CUDA);
    const size_t N = c->max_n;
    const int D = c->dim;
    const uint32_t cap = c->cap, hcap = c->hcap;
    for (int b = 0; b < 2; ++b) {
        slosh_ctx::Storage &S = c->pb[b];
        if ((st = alloc_storage(c, S, N, D))) return fail_create(st);
    }
    if ((st = dalloc(c, &c->fdt, N * D)) || (st = dalloc(c, &c->r0, N)) || (st = dalloc(c, &c->phase, N)) ||
        (st = dalloc(c, &c->materials, MAX_MATERIALS)) || (st = dalloc(c, &c->mat_hkeys, MAT_HASH)) ||
        (st = dalloc(c, &c->mat_dense, MAT_HASH)) || (st = dalloc(c, &c->hkeys[0], hcap)) ||
        (st = dalloc(c, &c->hkeys[1], hcap)) || (st = dalloc(c, &c->hvals[0], hcap)) ||
        (st = dalloc(c, &c->hvals[1], hcap)) || (st = dalloc(c, &c->slot_counts, (size_t)hcap * CELLS)) ||
        (st = dalloc(c, &c->blist_key, cap)) || (st = dalloc(c, &c->blist_slot, cap)) ||
        (st = dalloc(c, &c->blist2_key, cap)) || (st = dalloc(c, &c->blist2_slot, cap)) ||
        (st = dalloc(c, &c->hist, HIST_BINS)) || (st = dalloc(c, &c->hist_start, HIST_BINS)) ||
        (st = dalloc(c, &c->hist_coarse, HIST_COARSE)) || (st = dalloc(c, &c->tmp_key, 2 * (size_t)cap)) ||
        (st = dalloc(c, &c->tmp_slot, 2 * (size_t)cap)) || (st = dalloc(c, &c->bkey, cap)) ||
        (st = dalloc(c, &c->bslot, cap)) || (st = dalloc(c, &c->bfirst, cap)) || (st = dalloc(c, &c->bnp, cap)) ||
        (st = dalloc(c, &c->bcur, (size_t)cap * CELLS)) || (st = dalloc(c, &c->bcell, (size_t)cap * CELLS)) ||
        (st = dalloc(c, &c->bord, (size_t)cap * CELLS)) || (st = dalloc(c, &c->qorder, cap)) ||
        (st = dalloc(c, &c->bprev, cap)) ||
        (st = dalloc(c, &c->bnbh, (size_t)cap * nnb(D))) || (st = dalloc(c, &c->bnbh_rev, (size_t)cap * nnb(D))) ||
        (st = dalloc(c, &c->partial, (size_t)cap * (D == 3 ? Geo<3>::TILE : Geo<2>::TILE))) ||
        (st = dalloc(c, &c->pslot, N)) || (st = dalloc(c, &c->perm, N)) ||
        (st = dalloc(c, &c->skey, N)) ||
        (st = dalloc(c, &c->nodes, (size_t)cap * 64)) || (st = dalloc(c, &c->coll[0], (size_t)cap * 64)) ||
        (st = dalloc(c, &c->coll[1], (size_t)cap * 64)) || (st = dalloc(c, &c->coll_id[0], (size_t)cap * 64)) ||
        (st = dalloc(c, &c->coll_id[1], (size_t)cap * 64)) || (st = dalloc(c, &c->bodies, MAX_BODIES)) ||
        (st = dalloc(c, &c->body_imp, (size_t)MAX_BODIES * 6)) ||
        (st = dalloc(c, &c->ctr, 1)) || (st = dalloc(c, &c->err, 1)) || (st = dalloc(c, &c->small, 4)) ||
        (st = dalloc(c, &c->staging, N)) || (st = dalloc(c, &c->bfirst2, cap)) || (st = dalloc(c, &c->bnp2, cap)) ||
        (st = dalloc(c, &c->bcell2, (size_t)cap * CELLS)) || (st = dalloc(c, &c->cell_delta, (size_t)cap * CELLS)) ||
        (st = dalloc(c, &c->touch, cap)) || (st = dalloc(c, &c->cur_touch, cap)) ||
        (st = dalloc(c, &c->reuse_cta, 2 * (size_t)REUSE_MAX_CTAS)) ||
        (st = dalloc(c, &c->touched_cells, (size_t)cap * CELLS)) || (st = dalloc(c, &c->bsrc, cap)))
        return fail_create(st);
    cudaMemset(c->hkeys[0], 0xff, hcap * 4);
    cudaMemset(c->hkeys[1], 0xff, hcap * 4);
    cudaMemset(c->hvals[0], 0xff, hcap * 4);
    cudaMemset(c->hvals[1], 0xff, hcap * 4);
    cudaMemset(c->ctr, 0, sizeof(Counters));
    cudaMemset(c->err, 0, 4);
    cudaMemset(c->slot_counts, 0, (size_t)hcap * CELLS * 4);
    cudaMemset(c->body_imp, 0, (size_t)MAX_BODIES * 6 * sizeof(unsigned long long));
    if (const char *variant = std::getenv("SLOSH_P2G")) {
        if (std::strcmp(variant, "direct") == 0) c->p2g_variant = 3;
    }
    if (const char *nt = std::getenv("SLOSH_G2P_THREADS")) {
        const int v = std::atoi(nt);
        if (v == 64 || v == 128 || v == 256) c->g2p_threads = (uint32_t)v;
    }
    // the small-scene P2G's shared memory is above the 48 KB a launch gets by default
    cudaFuncSetAttribute(k_p2g_wide<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(P2gSmem<3, 3, P2G_WIDE_WARPS>));
    cudaFuncSetAttribute(k_p2g_wide<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(P2gSmem<3, 3, P2G_WIDE_WARPS>));
    cudaFuncSetAttribute(k_p2g_wide<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(P2gSmem<2, 3, P2G_WIDE_WARPS>));
    cudaFuncSetAttribute(k_p2g_wide<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(P2gSmem<2, 3, P2G_WIDE_WARPS>));
    if (const char *pdl = std::getenv("SLOSH_PDL")) c->pdl = std::strcmp(pdl, "0") != 0;
    c->reuse_mode = 2u;
    if (const char *r = std::getenv("SLOSH_GRID_REUSE")) c->reuse_mode = std::strcmp(r, "0") == 0 ? 0u : 1u;
    update_reuse(c);
    cudaMemset(c->bcell, 0, (size_t)cap * CELLS * 4);
    cudaMemset(c->bcell2, 0, (size_t)cap * CELLS * 4);
    cudaMemset(c->bnp, 0, (size_t)cap * 4);
    cudaMemset(c->bnp2, 0, (size_t)cap * 4);
    if (force_grid_rebuild(c, nullptr) != SLOSH_OK) return fail_create(SLOSH_E_CUDA);
    if (cudaDeviceSynchronize() != cudaSuccess) return fail_create(SLOSH_E_CUDA);
    c->params.gravity[1] = -9.81f;
    c->params.dt = 1.0f / 60.0f;
    *out = c;
    return SLOSH_OK;
}

void slosh_ctx_destroy(slosh_ctx *c) {
    if (!c) return;
    release_ctx(c);
    delete c;
}

int slosh_set_params(slosh_ctx *c, const slosh_params *p) {
    if (!c || !p || !(p->dt > 0.f)) return fail(c, SLOSH_E_INVALID, "dt must be > 0");
    c->params = *p;
    destroy_graphs(c);
    return SLOSH_OK;
}

int slosh_upload_particles(slosh_ctx *c, const slosh_particle *particles, uint32_t n, void *stream) {
    if (!c || (!particles && n)) return SLOSH_E_INVALID;
    if (n > c->max_n) return fail(c, SLOSH_E_CAPACITY, "%u particles exceed max_particles %u", n, c->max_n);
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    // The substep graphs bake the particle count and the scene flags in; an
    // upload that keeps them keeps the graphs.
    const uint32_t old_mat = c->n_materials, old_damp = c->has_damping, old_sand = c->has_sand,
                   old_models = c->model_mask;
    if (n != c->n) destroy_graphs(c);
    c->n = n;
    update_reuse(c);
    CK(cudaMemcpyAsync(c->staging, particles, (size_t)n * sizeof(slosh_particle), cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(c->mat_hkeys, 0xff, MAT_HASH * 4, st));
    CK(cudaMemsetAsync(c->small, 0, 16, st));
    CK(cudaMemsetAsync(c->err, 0, 4, st));
    CK(cudaMemsetAsync(c->ctr, 0, sizeof(Counters), st));
    if (int r = force_grid_rebuild(c, st)) return r;
    for (int k = 0; k < 2; ++k) {
        CK(cudaMemsetAsync(c->hkeys[k], 0xff, c->hcap * 4, st));
        CK(cudaMemsetAsync(c->hvals[k], 0xff, c->hcap * 4, st));
    }
    CK(cudaMemsetAsync(c->slot_counts, 0, (size_t)c->hcap * CELLS * 4, st));
    CK(cudaMemsetAsync(c->hist, 0, HIST_BINS * 4, st));
    CK(cudaMemsetAsync(c->hist_coarse, 0, HIST_COARSE * 4, st));
    c->parity = 0;
    if (n > 0) {
        DevScene s = make_scene(c, 0, false);
        IoBuffers io{};
        io.in = c->staging;
        io.mat_hkeys = c->mat_hkeys;
        io.mat_dense = c->mat_dense;
        io.n_mat = c->small;
        io.scene_flags = c->small + 1;
        io.r0 = c->r0;
        io.phase = c->phase;
        const uint32_t g = grid_for(n, 256, (uint32_t)c->sm_count * 16);
        k_mat_insert<<<g, 256, 0, st>>>(s, io, n);
        if (c->dim == 3) k_ingest<3><<<g, 256, 0, st>>>(s, io, 0u, n, 0u);
        else k_ingest<2><<<g, 256, 0, st>>>(s, io, 0u, n, 0u);
        CK(cudaGetLastError());
    }
    uint32_t small[2] = {0, 0};
    CK(cudaMemcpyAsync(small, c->small, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    c->n_materials = small[0];
    c->has_damping = (small[1] & SCENE_DAMPING) ? 1u : 0u;
    c->force_pending = (small[1] & SCENE_FORCE) ? 1u : 0u;
    c->has_sand = (small[1] & SCENE_SAND) ? 1u : 0u;
    c->model_mask = (small[1] >> SCENE_MODEL_SHIFT) & 0xffu;
    if (c->n_materials != old_mat || c->has_damping != old_damp || c->has_sand != old_sand ||
        c->model_mask != old_models)
        destroy_graphs(c);
    return check_device_error(c);
}

int slosh_append_particles(slosh_ctx *c, const slosh_particle *particles, uint32_t n, void *stream) {
    if (!c || (!particles && n)) return SLOSH_E_INVALID;
    if ((uint64_t)c->n + n > c->max_n)
        return fail(c, SLOSH_E_CAPACITY, "%u + %u particles exceed max_particles %u", c->n, n, c->max_n);
    if (n == 0) return SLOSH_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    CK(cudaStreamSynchronize(c->stream));
    destroy_graphs(c);
    bool forces = false;
    for (uint32_t i = 0; i < n && !forces; ++i)
        forces = particles[i].force_dt[0] != 0.f || particles[i].force_dt[1] != 0.f || particles[i].force_dt[2] != 0.f;
    const uint32_t base = c->n;
    DevScene s = make_scene(c, c->parity, false);
    if (forces && !c->force_pending && base > 0) {
        // the stored forces of the earlier particles were consumed by a substep
        for (int k = 0; k < c->dim; ++k) CK(cudaMemsetAsync(c->fdt + (size_t)k * c->max_n, 0, (size_t)base * 4, st));
    }
    CK(cudaMemcpyAsync(c->staging, particles, (size_t)n * sizeof(slosh_particle), cudaMemcpyHostToDevice, st));
    IoBuffers io{};
    io.in = c->staging;
    io.mat_hkeys = c->mat_hkeys;
    io.mat_dense = c->mat_dense;
    io.n_mat = c->small;
    io.scene_flags = c->small + 1;
    io.r0 = c->r0;
    io.phase = c->phase;
    const uint32_t g = grid_for(n, 256, (uint32_t)c->sm_count * 16);
    if (int r = force_grid_rebuild(c, st)) return r;
    k_mat_insert<<<g, 256, 0, st>>>(s, io, n);
    if (c->dim == 3) k_ingest<3><<<g, 256, 0, st>>>(s, io, base, n, 0u, base);
    else k_ingest<2><<<g, 256, 0, st>>>(s, io, base, n, 0u, base);
    CK(cudaGetLastError());
    uint32_t small[2] = {0, 0};
    CK(cudaMemcpyAsync(small, c->small, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    c->n = base + n;
    update_reuse(c);
    c->n_materials = small[0];
    c->has_damping = (small[1] & SCENE_DAMPING) ? 1u : 0u;
    c->has_sand = (small[1] & SCENE_SAND) ? 1u : 0u;
    c->model_mask = (small[1] >> SCENE_MODEL_SHIFT) & 0xffu;
    c->force_pending = (c->force_pending || forces) ? 1u : 0u;
    return check_device_error(c);
}

int slosh_remove_particles(slosh_ctx *c, uint32_t start, uint32_t count, uint32_t *removed, void *stream) {
    if (!c) return SLOSH_E_INVALID;
    const uint32_t end = (uint32_t)std::min<uint64_t>((uint64_t)start + count, c->n);
    const uint32_t nrem = start < end ? end - start : 0u;
    if (removed) *removed = nrem;
    if (nrem == 0) return SLOSH_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    CK(cudaStreamSynchronize(c->stream));
    destroy_graphs(c);
    const DevScene s = make_scene(c, c->parity, c->force_pending != 0);
    IoBuffers io{};
    io.r0 = c->r0;
    io.phase = c->phase;
    // the record staging area (192 bytes a particle) holds the (3 + D)-plane temporary
    float *tmp = reinterpret_cast<float *>(c->staging);
    const uint32_t g = grid_for(c->n, 256, (uint32_t)c->sm_count * 16);
    if (int r = force_grid_rebuild(c, st)) return r;
    if (c->dim == 3) k_remove<3><<<g, 256, 0, st>>>(s, io, start, end, tmp);
    else k_remove<2><<<g, 256, 0, st>>>(s, io, start, end, tmp);
    CK(cudaGetLastError());
    const uint32_t left = c->n - nrem;
    // B now holds the survivors in insertion order: make it the current storage
    std::swap(c->pb[c->parity & 1u], c->pb[(c->parity & 1u) ^ 1u]);
    c->n = left;
    update_reuse(c);
    const DevScene s2 = make_scene(c, c->parity, false);
    if (left) {
        const uint32_t g2 = grid_for(left, 256, (uint32_t)c->sm_count * 16);
        if (c->dim == 3) k_remove_sides<3><<<g2, 256, 0, st>>>(s2, io, left, tmp);
        else k_remove_sides<2><<<g2, 256, 0, st>>>(s2, io, left, tmp);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(st));
    return check_device_error(c);
}

int slosh_download_particles(slosh_ctx *c, slosh_particle *out, uint32_t n, void *stream) {
    if (!c || (!out && n)) return SLOSH_E_INVALID;
    if (n > c->n) return fail(c, SLOSH_E_INVALID, "asked for %u particles, context holds %u", n, c->n);
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    if (n > 0) {
        DevScene s = make_scene(c, c->parity, c->force_pending != 0);
        IoBuffers io{};
        io.out = c->staging;
        io.r0 = c->r0;
        io.phase = c->phase;
        const uint32_t g = grid_for(c->n, 256, (uint32_t)c->sm_count * 16);
        if (c->dim == 3) k_egest<3><<<g, 256, 0, st>>>(s, io, 0u);
        else k_egest<2><<<g, 256, 0, st>>>(s, io, 0u);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, c->staging, (size_t)n * sizeof(slosh_particle), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return check_device_error(c);
}

int slosh_download_positions(slosh_ctx *c, float *out, uint32_t n, void *stream) {
    if (!c || (!out && n)) return SLOSH_E_INVALID;
    if (n > c->n) return fail(c, SLOSH_E_INVALID, "asked for %u particles, context holds %u", n, c->n);
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    if (n > 0) {
        DevScene s = make_scene(c, c->parity, false);
        float4 *tmp = (float4 *)c->staging;  // staging holds >= 12 float4 per particle
        k_positions<<<grid_for(c->n, 256, (uint32_t)c->sm_count * 16), 256, 0, st>>>(s, tmp, 0u);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(out, tmp, (size_t)n * 16, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return check_device_error(c);
}

int slosh_set_bodies(slosh_ctx *c, const slosh_body *bodies, uint32_t n) {
    if (!c || (!bodies && n)) return SLOSH_E_INVALID;
    if (n > MAX_BODIES) return fail(c, SLOSH_E_CAPACITY, "%u bodies exceed the limit of %u", n, MAX_BODIES);
    std::vector<DevBody> db(n);
    for (uint32_t i = 0; i < n; ++i) {
        to_dev_body(bodies[i], db[i], c->dim);
        if (!(db[i].scale > 0.f)) return fail(c, SLOSH_E_INVALID, "body %u: scale must be > 0", i);
        if (db[i].coupling > SLOSH_COUPLING_TWO_WAY)
            return fail(c, SLOSH_E_INVALID, "body %u: unknown coupling %u", i, db[i].coupling);
        const bool mesh = c->dim == 3 && db[i].shape_type == SLOSH_SHAPE_TRIMESH;
        if (mesh && !trimesh_in_range(c, db[i]))
            return fail(c, SLOSH_E_INVALID, "body %u: trimesh shape not made by slosh_add_trimesh on this context", i);
        if (!mesh && !shape_supported(db[i].shape_type, c->dim))
            return fail(c, SLOSH_E_INVALID, "body %u: unsupported shape type %u in %dD", i, db[i].shape_type, c->dim);
    }
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (n) CK(cudaMemcpy(c->bodies, db.data(), n * sizeof(DevBody), cudaMemcpyHostToDevice));
    CK(cudaMemset(c->body_imp, 0, (size_t)MAX_BODIES * 6 * sizeof(unsigned long long)));
    c->n_bodies = n;
    c->coll_dynamic = 0;
    for (uint32_t i = 0; i < n; ++i) c->coll_dynamic |= db[i].coupling == SLOSH_COUPLING_TWO_WAY ? 1u : 0u;
    destroy_graphs(c);
    return SLOSH_OK;
}

int slosh_add_trimesh(slosh_ctx *c, const float *vertices, uint32_t n_vertices, const uint32_t *indices,
                      uint32_t n_triangles, slosh_body *body) {
    if (!c || !body || (!vertices && n_vertices) || (!indices && n_triangles)) return SLOSH_E_INVALID;
    if (c->dim != 3) return fail(c, SLOSH_E_INVALID, "triangle meshes are 3D colliders");
    if (n_triangles == 0 || n_triangles > (1u << 24))
        return fail(c, SLOSH_E_INVALID, "a mesh needs 1 to 2^24 triangles (got %u)", n_triangles);
    std::vector<float4> vtx = c->mesh_vtx_host;
    std::vector<uint32_t> idx = c->mesh_idx_host;
    TriMeshRef ref{};
    if (!build_trimesh(vertices, n_vertices, indices, n_triangles, vtx, idx, c->n_meshes, ref))
        return fail(c, SLOSH_E_INVALID, "triangle vertex index out of range (%u vertices)", n_vertices);
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    float4 *dv = nullptr;
    uint32_t *di = nullptr;
    if (cudaMalloc(&dv, vtx.size() * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&di, idx.size() * sizeof(uint32_t)) != cudaSuccess) {
        cudaFree(dv);
        cudaFree(di);
        return fail(c, SLOSH_E_NOMEM, "mesh buffers");
    }
    CK(cudaMemcpy(dv, vtx.data(), vtx.size() * sizeof(float4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(di, idx.data(), idx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    cudaFree(c->mesh_vtx);
    cudaFree(c->mesh_idx);
    c->mesh_vtx = dv;
    c->mesh_idx = di;
    c->mesh_vtx_host.swap(vtx);
    c->mesh_idx_host.swap(idx);
    c->n_meshes += 1;
    destroy_graphs(c);  // the graphs hold the buffer pointers
    const uint32_t ty = SLOSH_SHAPE_TRIMESH;
    const uint32_t a[4] = {ref.vtx_root, ref.idx_root, ref.n_nodes, ty}, b[4] = {ref.n_tris, ref.n_verts, ref.ordinal, 0u};
    std::memcpy(body->shape_a, a, sizeof(a));
    std::memcpy(body->shape_b, b, sizeof(b));
    return SLOSH_OK;
}

int slosh_get_bodies(slosh_ctx *c, slosh_body *out, uint32_t n) {
    if (!c || (!out && n) || n > c->n_bodies) return SLOSH_E_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    std::vector<DevBody> db(n);
    if (n) CK(cudaMemcpy(db.data(), c->bodies, n * sizeof(DevBody), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) from_dev_body(db[i], out[i], c->dim);
    return SLOSH_OK;
}

int slosh_step(slosh_ctx *c, uint32_t n_substeps, void *stream) {
    if (!c) return SLOSH_E_INVALID;
    if (c->n == 0) return fail(c, SLOSH_E_STATE, "no particles uploaded");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    for (uint32_t k = 0; k < n_substeps; ++k) {
        if (c->n_hooks) {
            const int r = c->dim == 3 ? enqueue_substep_hooked<3>(c, st, c->parity, c->force_pending != 0)
                                      : enqueue_substep_hooked<2>(c, st, c->parity, c->force_pending != 0);
            if (r < 0) return r == SLOSH_E_CUDA ? fail(c, r, "substep with stage hooks: CUDA error") : r;
            c->force_pending = 0;
        } else if (c->force_pending) {
            enqueue_substep_any(c, st, c->parity, true);
            CK(cudaGetLastError());
            c->force_pending = 0;
        } else {
            if (!c->graphs_valid) {
                if (st != c->stream) CK(cudaStreamSynchronize(st));
                int r = build_graphs(c);
                if (r) return r;
                if (st != c->stream) CK(cudaStreamSynchronize(c->stream));
            }
            CK(cudaGraphLaunch(c->graph[c->parity], st));
        }
        c->parity ^= 1u;
    }
    return SLOSH_OK;
}

int slosh_set_hook(slosh_ctx *c, uint32_t point, slosh_hook_fn fn, void *user) {
    if (!c || point >= SLOSH_HOOK_COUNT) return SLOSH_E_INVALID;
    if (c->in_hook) return fail(c, SLOSH_E_STATE, "hooks cannot be changed from inside a hook");
    c->hooks[point] = fn;
    c->hook_user[point] = fn ? user : nullptr;
    c->n_hooks = 0;
    for (uint32_t k = 0; k < SLOSH_HOOK_COUNT; ++k) c->n_hooks += c->hooks[k] ? 1u : 0u;
    return SLOSH_OK;
}

int slosh_enqueue_builtin(slosh_ctx *c, uint32_t point, void *stream) {
    if (!c) return SLOSH_E_INVALID;
    if (!c->in_hook || c->hook_point != point || (point != SLOSH_HOOK_RUN_P2G && point != SLOSH_HOOK_RUN_G2P))
        return fail(c, SLOSH_E_STATE, "the built-in stage of hook %u can only be enqueued from inside that run hook", point);
    cudaStream_t st = pick(c, stream);
    const DevScene &s = c->hook_scene;
    if (point == SLOSH_HOOK_RUN_P2G) {
        DevScene gather = s;  // P2G, then its node sums written to `nodes`
        gather.gather_only = 1u;
        if (c->dim == 3) {
            enqueue_p2g<3>(c, s, st);
            enqueue_grid_update<3>(c, gather, st);
        } else {
            enqueue_p2g<2>(c, s, st);
            enqueue_grid_update<2>(c, gather, st);
        }
    } else {
        if (c->dim == 3) enqueue_g2p<3>(c, s, st, nullptr);
        else enqueue_g2p<2>(c, s, st, nullptr);
    }
    CK(cudaGetLastError());
    return SLOSH_OK;
}

int slosh_device_view_get(slosh_ctx *c, slosh_device_view *out) {
    if (!c || !out) return SLOSH_E_INVALID;
    if (!c->in_hook) return fail(c, SLOSH_E_STATE, "the device view is only valid inside a stage hook");
    const DevScene &s = c->hook_scene;
    std::memset(out, 0, sizeof(*out));
    out->dim = (uint32_t)c->dim;
    out->n_particles = c->n;
    out->capacity = c->max_n;
    out->grid_capacity = c->cap;
    out->cell_width = c->h;
    out->dt = c->params.dt;
    out->n_blocks = &c->ctr->n_blocks;
    out->block_keys = s.bkey;
    out->block_first = s.bfirst;
    out->block_count = s.bnp;
    out->perm = s.perm;
    out->x_mass = s.pm;
    out->vel = s.vv;
    out->affine = s.cq;
    out->def_grad = s.fq;
    out->flags = s.fo;
    out->plastic = s.ps;
    out->out_x_mass = s.out_pm;
    out->out_vel = s.out_vv;
    out->out_affine = s.out_cq;
    out->out_def_grad = s.out_fq;
    out->out_flags = s.out_fo;
    out->out_plastic = s.out_ps;
    out->nodes = s.nodes;
    return SLOSH_OK;
}

int slosh_sync(slosh_ctx *c, void *stream) {
    if (!c) return SLOSH_E_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(pick(c, stream)));
    CK(cudaGetLastError());
    return check_device_error(c);
}

uint32_t slosh_kernels_per_substep(const slosh_ctx *c) {
    if (!c) return 0;
    // the full build's 9 kernels, P2G, the grid update, G2P and the rigid
    // update; with grid reuse the decision, and without conditional graphs
    // also the two reuse kernels, which return at once in a full build
    uint32_t k = 9u + 4u;
    if (c->reuse) k += c->cond_graphs ? 1u : 3u;
    return k;
}

int slosh_profile_substeps(slosh_ctx *c, uint32_t n_substeps, void *stream, float *kernel_ms, uint32_t cap,
                           uint32_t *n_kernels) {
    if (!c || (!kernel_ms && cap)) return SLOSH_E_INVALID;
    if (c->n == 0) return fail(c, SLOSH_E_STATE, "no particles uploaded");
    CK(cudaSetDevice(c->device));
    Prof pr{};
    pr.st = pick(c, stream);
    for (int k = 0; k < N_KERNELS; ++k) {
        CK(cudaEventCreate(&pr.ev[k][0]));
        CK(cudaEventCreate(&pr.ev[k][1]));
    }
    double acc[N_KERNELS] = {};
    int rc = SLOSH_OK;
    for (uint32_t it = 0; it < n_substeps && rc == SLOSH_OK; ++it) {
        for (int k = 0; k < N_KERNELS; ++k) pr.used[k] = false;
        enqueue_substep_any(c, pr.st, c->parity, c->force_pending != 0, &pr);
        c->force_pending = 0;
        c->parity ^= 1u;
        cudaError_t e = cudaEventSynchronize(pr.ev[N_KERNELS - 1][1]);
        if (e != cudaSuccess) {
            rc = fail(c, SLOSH_E_CUDA, "profiling: %s", cudaGetErrorString(e));
            break;
        }
        for (int k = 0; k < N_KERNELS; ++k) {
            if (!pr.used[k]) continue;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, pr.ev[k][0], pr.ev[k][1]);
            acc[k] += ms;
        }
    }
    for (int k = 0; k < N_KERNELS; ++k) {
        cudaEventDestroy(pr.ev[k][0]);
        cudaEventDestroy(pr.ev[k][1]);
    }
    if (rc) return rc;
    for (uint32_t k = 0; k < cap && k < (uint32_t)N_KERNELS; ++k) kernel_ms[k] = (float)acc[k];
    if (n_kernels) *n_kernels = N_KERNELS;
    return check_device_error(c);
}

int slosh_get_stats(slosh_ctx *c, slosh_stats *out) {
    if (!c || !out) return SLOSH_E_INVALID;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaDeviceSynchronize());
    Counters ctr;
    CK(cudaMemcpy(&ctr, c->ctr, sizeof(ctr), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    out->n_particles = c->n;
    out->n_blocks = ctr.last_n_blocks;
    out->n_primary_blocks = ctr.last_n_primary;
    out->n_materials = c->n_materials;
    out->n_svd_fp64 = ctr.n_svd_fp64;
    out->n_grid_rebuilds = ctr.n_rebuilds;
    out->n_grid_reuses = ctr.n_reuses;
    out->conditional_graphs = c->cond_graphs ? 1u : 0u;
    return SLOSH_OK;
}

int slosh_kernel_name(uint32_t index, char *buf, size_t len) {
    if (index >= (uint32_t)N_KERNELS || !buf || len == 0) return SLOSH_E_INVALID;
    std::snprintf(buf, len, "%s", KERNEL_NAMES[index]);
    return SLOSH_OK;
}

int slosh_grid_debug(slosh_ctx *c, slosh_grid_dump *dump, uint32_t cap_blocks, uint32_t cap_sorted) {
    if (!c || !dump) return SLOSH_E_INVALID;
    if (c->n == 0) return fail(c, SLOSH_E_STATE, "no particles uploaded");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    DevScene s = make_scene(c, c->parity, false);
    s.reuse = 0u;  // a full standalone build; the next substep rebuilds too
    if (int r = force_grid_rebuild(c, st)) return r;
    if (c->dim == 3) enqueue_grid_build<3>(c, s, st, nullptr, true);
    else enqueue_grid_build<2>(c, s, st, nullptr, true);
    CK(cudaGetLastError());
    Counters ctr;
    CK(cudaMemcpyAsync(&ctr, c->ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    uint32_t err_bits = 0;
    CK(cudaMemcpy(&err_bits, c->err, 4, cudaMemcpyDeviceToHost));
    if (err_bits) {
        enqueue_clear(c, s, st);
        CK(cudaStreamSynchronize(st));
        return check_device_error(c);
    }
    const uint32_t nb = ctr.n_blocks;
    const int NB = nbk(c->dim), NN = nnb(c->dim);
    dump->n_blocks = nb;
    dump->nb_buckets = (uint32_t)NB;
    dump->n_neighbors = (uint32_t)NN;
    // Full layout with extras, on the device.
    const uint32_t cap_entries = (uint32_t)std::min<uint64_t>((uint64_t)c->n * (c->dim == 3 ? 8 : 4), 0xffffffffull);
    DebugBuffers d{};
    void *blob = nullptr;
    const size_t nbs = std::max<uint32_t>(nb, 1);
    const size_t words = nbs * NB * 2 + nbs * 3 + (size_t)cap_entries * 2 + 1 + c->n;
    CK(cudaMalloc(&blob, words * 4));
    uint32_t *w = (uint32_t *)blob;
    d.counts = w;
    d.cursor = w + nbs * NB;
    d.first = w + nbs * NB * 2;
    d.npe = d.first + nbs;
    d.np = d.npe + nbs;
    d.sorted = d.np + nbs;
    d.sorted2 = d.sorted + cap_entries;
    d.total = d.sorted2 + cap_entries;
    d.cap_entries = cap_entries;
    uint32_t *perm_oid = d.total + 1;
    cudaMemsetAsync(d.counts, 0, nbs * NB * 4, st);
    k_perm_to_oid<<<grid_for(c->n, 256, (uint32_t)c->sm_count * 16), 256, 0, st>>>(s, perm_oid);
    const uint32_t g = grid_for(c->n, 256, (uint32_t)c->sm_count * 16);
    if (c->dim == 3) {
        k_dbg_count<3><<<g, 256, 0, st>>>(s, d);
        k_dbg_scan<3, 1024><<<1, 1024, 0, st>>>(s, d);
        k_dbg_scatter<3><<<g, 256, 0, st>>>(s, d);
        k_dbg_canon<3><<<grid_for(nbs * NB, 128, 4096), 128, 0, st>>>(s, d);
    } else {
        k_dbg_count<2><<<g, 256, 0, st>>>(s, d);
        k_dbg_scan<2, 1024><<<1, 1024, 0, st>>>(s, d);
        k_dbg_scatter<2><<<g, 256, 0, st>>>(s, d);
        k_dbg_canon<2><<<grid_for(nbs * NB, 128, 4096), 128, 0, st>>>(s, d);
    }
    uint32_t total = 0;
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&total, d.total, 4, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    dump->n_sorted = total;
    const uint32_t nbc = std::min(nb, cap_blocks);
    auto copy = [&](uint32_t *dst, const uint32_t *src, size_t count) {
        if (dst && count && ce == cudaSuccess) ce = cudaMemcpy(dst, src, count * 4, cudaMemcpyDeviceToHost);
    };
    copy(dump->keys, c->bkey, nbc);
    copy(dump->first_particle, d.first, nbc);
    copy(dump->num_particles, d.np, nbc);
    copy(dump->num_particles_with_extras, d.npe, nbc);
    copy(dump->bucket_counts, d.counts, (size_t)nbc * NB);
    copy(dump->sorted_ids, d.sorted2, std::min(total, cap_sorted));
    copy(dump->primary_first, s.bfirst, nbc);
    copy(dump->primary_perm, perm_oid, c->n);
    copy(dump->neighbors, c->bnbh, (size_t)nbc * NN);
    cudaFree(blob);
    enqueue_clear(c, s, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return fail(c, SLOSH_E_CUDA, "grid debug: %s", cudaGetErrorString(ce));
    if (total > cap_entries) return fail(c, SLOSH_E_CAPACITY, "debug layout overflow");
    return SLOSH_OK;
}

int slosh_debug_nodes(slosh_ctx *c, int stage, float *nodes, uint32_t cap_blocks, uint32_t *n_blocks) {
    if (!c || stage < 1 || stage > 2) return SLOSH_E_INVALID;
    if (c->n == 0) return fail(c, SLOSH_E_STATE, "no particles uploaded");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    DevScene s = make_scene(c, c->parity, c->force_pending != 0);
    s.reuse = 0u;  // a full standalone build; the next substep rebuilds too
    if (int r = force_grid_rebuild(c, st)) return r;
    DevScene gather = s;  // stage 1 of the deterministic P2G: node sums only
    gather.gather_only = 1u;
    if (c->dim == 3) {
        enqueue_grid_build<3>(c, s, st, nullptr, true);
        enqueue_p2g<3>(c, s, st);
        if (stage >= 2) enqueue_grid_update<3>(c, s, st);
        else if (s.use_partial) enqueue_grid_update<3>(c, gather, st);
    } else {
        enqueue_grid_build<2>(c, s, st, nullptr, true);
        enqueue_p2g<2>(c, s, st);
        if (stage >= 2) enqueue_grid_update<2>(c, s, st);
        else if (s.use_partial) enqueue_grid_update<2>(c, gather, st);
    }
    CK(cudaGetLastError());
    Counters ctr;
    CK(cudaMemcpyAsync(&ctr, c->ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (n_blocks) *n_blocks = ctr.n_blocks;
    const uint32_t nbc = std::min(ctr.n_blocks, cap_blocks);
    if (nodes && nbc) CK(cudaMemcpy(nodes, c->nodes, (size_t)nbc * 64 * 16, cudaMemcpyDeviceToHost));
    enqueue_clear(c, s, st);
    CK(cudaStreamSynchronize(st));
    return check_device_error(c);
}

int slosh_prefix_sum(slosh_ctx *c, const uint32_t *in, uint32_t *out, uint32_t n) {
    if (!c || (n && (!in || !out))) return SLOSH_E_INVALID;
    if (n > 2 * c->cap) return fail(c, SLOSH_E_CAPACITY, "prefix sum of %u values exceeds %u", n, 2 * c->cap);
    if (n == 0) return SLOSH_OK;
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    CK(cudaMemcpyAsync(c->tmp_key, in, (size_t)n * 4, cudaMemcpyHostToDevice, st));
    k_exclusive_scan<1024><<<1, 1024, 0, st>>>(c->tmp_key, c->tmp_slot, n);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, c->tmp_slot, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SLOSH_OK;
}

int slosh_timestep_bound(slosh_ctx *c, float *dt_out, void *stream) {
    if (!c || !dt_out) return SLOSH_E_INVALID;
    if (c->n == 0) return fail(c, SLOSH_E_STATE, "no particles uploaded");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = pick(c, stream);
    const DevScene s = make_scene(c, c->parity, false);
    uint32_t *slot = c->small + 3;
    CK(cudaMemsetAsync(slot, 0xff, 4, st));
    const uint32_t g = grid_for(c->n, 256, (uint32_t)c->sm_count * 16);
    if (c->dim == 3) k_timestep_bound<3><<<g, 256, 0, st>>>(s, 0u, slot);
    else k_timestep_bound<2><<<g, 256, 0, st>>>(s, 0u, slot);
    CK(cudaGetLastError());
    uint32_t u = 0;
    CK(cudaMemcpyAsync(&u, slot, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *dt_out = (float)u / TIMESTEP_FLOAT_TO_INT;  // GpuTimestepBounds::computed_dt
    return SLOSH_OK;
}

int slosh_last_error(const slosh_ctx *c, char *buf, size_t len) {
    if (!c || !buf || len == 0) return SLOSH_E_INVALID;
    std::snprintf(buf, len, "%s", c->last_error.c_str());
    return SLOSH_OK;
}

}  // extern "C"

#include "batch.cuh"
#include "server.cuh"
