// lbm_batch.cuh -- many independent lattices advanced by one launch.
//
// Each lattice keeps its own parameters (sizes, tau, walls, flags, forces)
// in a BatchLattice record in device memory.  The launch walks a work list
// of (lattice, first cell) items: an item covers `block * cells_per_thread`
// consecutive cells of one lattice, so each block works on one lattice at a
// time and every branch on the lattice's kind is uniform within the block.
// Items are dealt to blocks round-robin (item w -> block w mod gridDim), a
// fixed schedule: the result does not depend on the launch shape.  A block
// reads its lattice's record from a shared-memory copy.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

template <class T>
struct __align__(16) BatchLattice {
    Params P;
    Streams<T> S[2];  // [k & 1]: source / destination buffers of the k-th step of a run
    int vec;          // 2 when nz is even (vector access in SCHED_PAIR_MIXED)
};

struct BatchItem {
    int lattice;
    int start;  // first cell of the item
};

// Work schedules of the batched step (template parameter SCHED).
enum BatchSched : int {
    SCHED_SINGLE = 0,      // one cell per thread
    SCHED_PAIR_SCALAR = 1, // two cells per thread, scalar memory access, f32x2 collision
    SCHED_PAIR_MIXED = 2,  // as 1, but vector access for lattices with an even nz
    SCHED_BRANCHES = 3,    // no batched kernel: each lattice's own step kernels on
                           // parallel streams, captured into one graph per two steps
};

// First step after a state upload: collide in place, one cell per thread.
template <class M, int FM>
__global__ void __launch_bounds__(256) k_collide_batch(const BatchLattice<typename M::T>* __restrict__ lats,
                                                       const BatchItem* __restrict__ items, int nitems, int span,
                                                       int phase)
{
    using C = typename M::C;
    const Outputs<C> none{nullptr, nullptr, nullptr};
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const BatchItem it = items[w];
        const BatchLattice<typename M::T>& B = lats[it.lattice];
        for (int c = it.start + threadIdx.x; c < it.start + span && c < B.P.n; c += blockDim.x)
            collide_single<M, FM, OUT_NONE>(B.P, B.S[phase & 1], none, c, nullptr);
    }
}

// Fused step of every item; an item covers blockDim (SCHED_SINGLE) or
// 2 * blockDim (pair schedules) cells of one lattice.
template <class M, int FM, int SCHED>
__global__ void __launch_bounds__(256, SCHED == SCHED_SINGLE ? 3 : 2)
    k_step_batch(const BatchLattice<typename M::T>* __restrict__ lats, const BatchItem* __restrict__ items,
                 int nitems, int phase)
{
    using C = typename M::C;
    using Rec = BatchLattice<typename M::T>;
    const Outputs<C> none{nullptr, nullptr, nullptr};
    // The record of the block's current lattice, copied into shared memory
    // when the lattice changes (items of one lattice are consecutive, so a
    // block's successive items mostly share it).
    __shared__ __align__(16) unsigned int rec_words[(sizeof(Rec) + 3) / 4];
    const Rec& B = *reinterpret_cast<const Rec*>(rec_words);
    int held = -1;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const BatchItem it = items[w];
        if (it.lattice != held) {
            __syncthreads();  // every thread is done with the previous record
            const unsigned int* src = reinterpret_cast<const unsigned int*>(lats + it.lattice);
            for (int k = threadIdx.x; k < (int)(sizeof(Rec) / 4); k += blockDim.x) rec_words[k] = __ldg(src + k);
            __syncthreads();
            held = it.lattice;
        }
        const Params& P = B.P;
        const Streams<typename M::T>& S = B.S[phase & 1];
        if constexpr (SCHED == SCHED_SINGLE) {
            const int idx = it.start + threadIdx.x;
            if (idx < P.n) step_single<M, FM, OUT_NONE>(P, S, none, idx, nullptr);
        } else {
            const int idx0 = it.start + 2 * threadIdx.x;
            if (idx0 < P.n) {
                if (SCHED == SCHED_PAIR_MIXED && B.vec == 2)
                    step_pair<M, FM, OUT_NONE>(P, S, none, idx0, nullptr);
                else
                    step_pair_scalar<M, FM>(P, S, idx0);
            }
        }
    }
}

}  // namespace lbm
