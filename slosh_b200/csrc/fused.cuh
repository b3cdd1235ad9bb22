// One persistent, cooperative launch per batched substep: the phases of the
// 13-kernel batch substep (grid build, P2G, grid update, G2P with the
// particle update, bodies) run in order inside one kernel whose CTAs are all
// resident (cudaLaunchAttributeCooperative), separated by grid barriers.
// Every phase is the body of the corresponding stand-alone kernel, so the
// results are those of the multi-kernel substep bit for bit.
//
// The CTA is FUSED_THREADS = 128 threads (P2G's four warps, G2P's CTA of
// 128 particles); P2G's and G2P's shared memory share one dynamic buffer.
#pragma once

#include "grid_build.cuh"
#include "transfer.cuh"

namespace slosh {

constexpr int FUSED_THREADS = 128;
constexpr int FUSED_MIN_CTAS = 4;  // CTAs an SM: 128 registers a thread at most
constexpr int FUSED_NBUF = 3;      // P2G's staging depth

template <int D> constexpr size_t fused_smem_bytes() {
    return sizeof(P2gSmem<D, FUSED_NBUF>) > sizeof(G2pSmem<D, FUSED_THREADS>) ? sizeof(P2gSmem<D, FUSED_NBUF>)
                                                                               : sizeof(G2pSmem<D, FUSED_THREADS>);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid-wide barrier of the fused substep.  Thread 0 of each CTA arrives on
// a counter; the last one resets it and advances the generation, the others
// wait for the generation to move.  The cooperative launch keeps every CTA
// resident, so the wait ends when the slowest CTA arrives.  It is bounded
// all the same (2 s of device time, and an iteration limit in case the timer
// stalls): a CTA that gives up sets ERR_BARRIER, and a CTA that meets that
// bit at a barrier returns false, so every CTA leaves the kernel at its next
// barrier instead of running later phases on incomplete data; the host then
// reports SLOSH_E_TIMEOUT.  Returns true when the CTA may go on.
constexpr unsigned long long BARRIER_NS = 2000000000ull;
constexpr uint32_t BARRIER_SPINS = 1u << 24;
__device__ __forceinline__ bool grid_barrier(const DevScene &s) {
    __shared__ uint32_t go_on;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t *err = s.err;
        uint32_t ok = 0u;
        if (!(*err & ERR_BARRIER)) {
            volatile uint32_t *gen = &s.ctr->bar_gen;
            const uint32_t g0 = *gen;
            __threadfence();
            ok = 1u;
            if (atomicAdd(&s.ctr->bar_count, 1u) == gridDim.x + s.bar_extra - 1u) {
                atomicExch(&s.ctr->bar_count, 0u);
                __threadfence();
                atomicAdd(&s.ctr->bar_gen, 1u);
            } else {
                const unsigned long long t0 = global_ns(), limit = s.bar_ns ? s.bar_ns : BARRIER_NS;
                for (uint32_t it = 0; *gen == g0; ++it) {
                    if (it >= BARRIER_SPINS || global_ns() - t0 > limit) {
                        if (*gen == g0) {
                            atomicOr(s.err, ERR_BARRIER);
                            ok = 0u;
                        }
                        break;
                    }
                    __nanosleep(128);
                }
            }
            __threadfence();
            if (*err & ERR_BARRIER) ok = 0u;
        }
        go_on = ok;
    }
    __syncthreads();
    return go_on != 0u;
}

// The batched substep (B = true everywhere) as one cooperative kernel.
template <int D, bool POW2>
__global__ void __launch_bounds__(FUSED_THREADS, FUSED_MIN_CTAS) k_batch_fused(DevScene s) {
    extern __shared__ __align__(16) unsigned char fsm[];
    const Cta g = launch_cta();
    touch_body<D, true>(s, g);
    if (!grid_barrier(s)) return;
    neighbors_body<D, true>(s, g);
    if (!grid_barrier(s)) return;
    if (g.id == 0) scene_scan_body<FUSED_THREADS>(s);
    if (!grid_barrier(s)) return;
    scene_scatter_body(s, g);
    if (!grid_barrier(s)) return;
    scene_rank_body(s, g);
    if (!grid_barrier(s)) return;
    block_setup_body<D, true>(s, g);
    if (!grid_barrier(s)) return;
    if (g.id == 0) block_scan_body<FUSED_THREADS>(s);
    if (!grid_barrier(s)) return;
    scatter_body<true>(s, g);
    if (!grid_barrier(s)) return;
    canon_body(s, g);
    if (!grid_barrier(s)) return;
    p2g_body<D, true, false, FUSED_NBUF>(s, *reinterpret_cast<P2gSmem<D, FUSED_NBUF> *>(fsm));
    if (!grid_barrier(s)) return;
    grid_update_body<D, true>(s, g);
    if (!grid_barrier(s)) return;
    g2p_update_body<D, FUSED_THREADS, true, POW2>(s, g, *reinterpret_cast<G2pSmem<D, FUSED_THREADS> *>(fsm));
    if (!grid_barrier(s)) return;
    const uint32_t nt = g.n * FUSED_THREADS;
    for (uint32_t id = g.id * FUSED_THREADS + threadIdx.x; id < max(s.n_bodies, 1u); id += nt) rigid_body<D, true>(s, id);
}

}  // namespace slosh
