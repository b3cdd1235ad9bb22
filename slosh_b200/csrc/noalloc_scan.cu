// Allocation-free exclusive prefix sum.
//
// Some callers cannot allocate device memory at the point where they need a
// scan: a host that owns every device allocation up front (a renderer or
// game-engine plugin with a fixed budget, a real-time loop that must not
// allocate), or code that runs inside another framework's memory pool where
// a raw cudaMalloc would fragment it.  For them this entry point takes device
// input and output pointers and keeps its only scratch -- one partial sum per
// 4096-element tile -- in a file-scope __device__ array instead of memory it
// would have to allocate.
//
// Semantics are those of the context-based slosh_prefix_sum (slosh's
// eval_cpu, src/grid/prefix_sum.rs:97-110): out[i] = sum of in[0 .. i-1],
// out[0] = 0, the total is dropped.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/slosh_b200.h"

namespace {

constexpr uint32_t NA_THREADS = 256;
constexpr uint32_t NA_PER_THREAD = 16;
constexpr uint32_t NA_TILE = NA_THREADS * NA_PER_THREAD;  // elements per tile
constexpr uint32_t NA_MAX_TILES = 16384;                  // scratch words
constexpr uint64_t NA_MAX_N = (uint64_t)NA_TILE * NA_MAX_TILES;  // 67,108,864

// One partial sum per tile.  Every GPU that loads the library holds these
// 64 KiB until the process exits.  Shared by all calls: calls that overlap
// on the GPU race on it.
__device__ __align__(256) uint32_t g_scan_scratch[NA_MAX_TILES];

// Device address of g_scan_scratch in the current context.  The host-side
// symbol is only a stand-in for the device array, so the address is looked
// up on every call: the lookup allocates nothing, and a cached address would
// go stale when the caller resets the device or switches contexts (the
// module is then loaded again, possibly at another address).
int scratch_for_current_context(uint32_t **out) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_scan_scratch) != cudaSuccess || !p) return SLOSH_E_CUDA;
    *out = (uint32_t *)p;
    return SLOSH_OK;
}

__device__ __forceinline__ uint32_t warp_incl(uint32_t v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= (uint32_t)off) v += y;
    }
    return v;
}

// Exclusive scan of one value per thread over the CTA (NA_THREADS threads).
__device__ __forceinline__ uint32_t cta_excl(uint32_t v, uint32_t *total) {
    __shared__ uint32_t ws[NA_THREADS / 32];
    __shared__ uint32_t tot;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl(v);
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t x = lane < NA_THREADS / 32 ? ws[lane] : 0u;
        const uint32_t xi = warp_incl(x);
        if (lane < NA_THREADS / 32) ws[lane] = xi - x;
        if (lane == 31) tot = xi;
    }
    __syncthreads();
    const uint32_t r = ws[warp] + incl - v;
    if (total) *total = tot;
    __syncthreads();
    return r;
}

// Pass 1: sum of each tile into the scratch array.
__global__ void __launch_bounds__(NA_THREADS) k_na_tile_sums(const uint32_t *in, uint32_t n, uint32_t *scratch) {
    const uint64_t base = (uint64_t)blockIdx.x * NA_TILE + (uint64_t)threadIdx.x * NA_PER_THREAD;
    uint32_t s = 0;
#pragma unroll
    for (uint32_t k = 0; k < NA_PER_THREAD; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total = 0;
    cta_excl(s, &total);
    if (threadIdx.x == 0) scratch[blockIdx.x] = total;
}

// Pass 2: exclusive scan of the tile sums, in place, by one CTA.
__global__ void __launch_bounds__(NA_THREADS) k_na_scan_tile_sums(uint32_t *scratch, uint32_t ntiles) {
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < ntiles; b0 += NA_THREADS) {
        const uint32_t i = b0 + threadIdx.x;
        const uint32_t v = i < ntiles ? scratch[i] : 0u;
        uint32_t total = 0;
        const uint32_t ex = cta_excl(v, &total);
        if (i < ntiles) scratch[i] = carry + ex;
        carry += total;
    }
}

// Pass 3: exclusive scan inside each tile, offset by the tile's prefix.
__global__ void __launch_bounds__(NA_THREADS) k_na_tile_scan(const uint32_t *in, uint32_t *out, uint32_t n,
                                                            const uint32_t *scratch) {
    const uint64_t base = (uint64_t)blockIdx.x * NA_TILE + (uint64_t)threadIdx.x * NA_PER_THREAD;
    uint32_t v[NA_PER_THREAD];
    uint32_t s = 0;
#pragma unroll
    for (uint32_t k = 0; k < NA_PER_THREAD; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t run = scratch[blockIdx.x] + cta_excl(s, nullptr);
#pragma unroll
    for (uint32_t k = 0; k < NA_PER_THREAD; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

}  // namespace

extern "C" int slosh_prefix_sum_noalloc(const uint32_t *d_in, uint32_t *d_out, uint32_t n, void *stream) {
    if (n == 0) return SLOSH_OK;
    if (!d_in || !d_out || d_in == d_out) return SLOSH_E_INVALID;
    if ((uint64_t)n > NA_MAX_N) return SLOSH_E_CAPACITY;
    // A CUDA error left pending by the caller's earlier work is not ours to
    // consume: return without launching and leave it for its owner.
    if (cudaPeekAtLastError() != cudaSuccess) return SLOSH_E_CUDA;
    uint32_t *scratch = nullptr;
    const int st = scratch_for_current_context(&scratch);
    if (st != SLOSH_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const uint32_t ntiles = (uint32_t)(((uint64_t)n + NA_TILE - 1) / NA_TILE);
    k_na_tile_sums<<<ntiles, NA_THREADS, 0, s>>>(d_in, n, scratch);
    k_na_scan_tile_sums<<<1, NA_THREADS, 0, s>>>(scratch, ntiles);
    k_na_tile_scan<<<ntiles, NA_THREADS, 0, s>>>(d_in, d_out, n, scratch);
    // nothing was pending before the launches, so an error now is theirs
    return cudaGetLastError() == cudaSuccess ? SLOSH_OK : SLOSH_E_CUDA;
}
