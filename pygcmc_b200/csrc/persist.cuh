// Persistent step loop (gcmc_options.persistent): one cooperative launch runs
// a batched context's whole step range -- the reference's host loop over
// moveArray (gcmc/cpp/gcmc.cu:77-98), here with every replica advanced per
// step -- instead of a captured graph of per-step kernel launches.
//
// One CTA of kAcceptThreads threads per SM, all co-resident (cooperative
// launch).  Per MC step:
//   1. every CTA's 32 warps take the step's pose-energy items of all replicas
//      (the per-pose-warp kernel's items, energy_items);
//   2. grid barrier;
//   3. CTA r takes replica r (r, r + grid, ...): its accept kernel body, which
//      applies the accepted moves and prepares the replica's next step
//      (accept_step);
//   4. grid barrier.
// The dynamic shared memory is one AcceptSmem, reused as the 32 warps' WarpBuf
// during the energy phase.  State written in one phase is read in the next
// with plain loads after the barrier's acquire fence (the energy path reads no
// mutable state through the read-only cache).
//
// The barrier's wait is bounded: a CTA that has waited spin_cap polls raises
// ERR_SYNC in replica 0's error word and returns; every other CTA then times
// out at the same or the next barrier, so the launch always ends.
#pragma once
#include "accept.cuh"

namespace gcmc {

constexpr int kPersistWarps = kAcceptThreads / 32;
constexpr long long kPersistSpinCap = 1ll << 24;  // polls of about 100 ns: over a second

struct GridSync {
    unsigned count;  // CTAs arrived at the current barrier
    unsigned gen;    // barriers completed
};

// All CTAs of the grid meet here (whole CTA).  Returns false (every thread of
// the CTA) if this CTA gave up waiting.
__device__ __forceinline__ bool grid_barrier(GridSync* g, long long cap, int* err, int* ok_sh) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* gen = &g->gen;
        const unsigned g0 = *gen;
        __threadfence();  // release this CTA's writes before arriving
        if (atomicAdd(&g->count, 1u) + 1u == gridDim.x) {
            atomicExch(&g->count, 0u);
            __threadfence();
            atomicAdd(&g->gen, 1u);
        } else {
            long long polls = 0;
            while (*gen == g0) {
                if (++polls > cap) {
                    atomicOr(err, ERR_SYNC);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();  // acquire: the other CTAs' writes before their arrival
        *ok_sh = ok;
    }
    __syncthreads();
    return *ok_sh != 0;
}

__global__ void __launch_bounds__(kAcceptThreads, 1) k_persist(const RepDev* __restrict__ reps, int nrep, int nsteps,
                                                               GridSync* gs, long long spin_cap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int pre[257];
    __shared__ int wtot[32];
    __shared__ int ok_sh;
    WarpBuf* bufs = reinterpret_cast<WarpBuf*>(smem_raw);
    int* err = reps[0].err;
    for (int s = 0; s < nsteps; ++s) {
        // the two kinds of items one after the other (one code path at a time per SM)
        energy_items<0, 0>(reps, nrep, 0, blockIdx.x * kPersistWarps, gridDim.x * kPersistWarps,
                        bufs[threadIdx.x >> 5], pre, wtot);
        __syncthreads();  // pre / wtot are rewritten by the second prefix
        energy_items<1, 0>(reps, nrep, 0, blockIdx.x * kPersistWarps, gridDim.x * kPersistWarps,
                        bufs[threadIdx.x >> 5], pre, wtot);
        if (!grid_barrier(gs, spin_cap, err, &ok_sh)) return;
        for (int r = blockIdx.x; r < nrep; r += gridDim.x) {
            accept_step<false>(reps[r], 0, smem_raw);  // (no Ewald in the persistent loop)
            __syncthreads();
        }
        if (!grid_barrier(gs, spin_cap, err, &ok_sh)) return;
    }
}

}  // namespace gcmc
