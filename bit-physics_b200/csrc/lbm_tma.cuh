// lbm_tma.cuh -- fused step with TMA bulk-copy staging in shared memory.
//
// The register-staged kernels (k_step, k_step2) can keep only as many loads
// in flight as their registers hold.  Here the 19 source rows of a tile are
// fetched by the Tensor Memory Accelerator into a multi-stage shared-memory
// ring (1-D cp.async.bulk, completion counted on an mbarrier), so the bytes
// in flight are bounded by shared memory, not registers.
//
// Tile: rows_per_tile consecutive y-rows of one x-plane (contiguous cells).
// For direction d the stage holds, at tile row r, the source row
// (x - c_x, y0 + r - c_y) (periodic wrap in x and y; a wrap in y splits the
// copy in two); the z shift, with its periodic wrap, is an index within the
// shared-memory row.  Two cells per thread, packed f32x2 collision, direct
// vector stores to global memory.  Cells that need a boundary rule use
// k_step's resolve_state (global reloads).
//
// Every mbarrier wait is bounded by a deadline on the global nanosecond
// timer.  A wait that runs out sets *P.err (the host reports it and the state
// is invalid) and a block-wide abort flag in shared memory: from then on the
// producer issues no copy and no thread of the block waits again, so the
// error path ends quickly.  Before the producer warp exits it waits (bounded
// again) for the last copy group it issued into every stage, so no block
// retires with bulk copies still writing into its shared memory.  No
// multicast.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

constexpr int TMA_CONSUMER_WARPS = 8;
constexpr int TMA_CONSUMERS = 32 * TMA_CONSUMER_WARPS;  // cell threads
constexpr int TMA_THREADS = TMA_CONSUMERS + 32;         // + one producer warp
constexpr int TMA_MAX_STAGES = 4;
constexpr unsigned long long TMA_WAIT_NS = 500000000ull;  // 0.5 s per wait before giving up

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Wait for the phase with the given parity, for at most TMA_WAIT_NS of
// wall time; true when it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    const unsigned long long t0 = global_ns();
    for (;;) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
        if (global_ns() - t0 > TMA_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(smem_dst)), "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Issue the copies of tile t into a stage.  Called by the first warp:
// lane 0 registers the stage's byte count, then lane d < 19 copies direction d.
template <class T>
__device__ __forceinline__ void tma_issue_tile(const Params& P, const Streams<T>& S, const TileCfg& G, int t,
                                               T* stage, uint64_t* bar, int lane)
{
    const int x = t / G.tiles_y;
    const int y0 = (t - x * G.tiles_y) * G.rows;
    const int rows = min(G.rows, P.ny - y0);
    const uint32_t row_bytes = (uint32_t)P.nz * sizeof(T);
    if (lane == 0) mbar_expect_tx(bar, (uint32_t)Q * rows * row_bytes);
    __syncwarp();
    if (lane >= Q) return;
    // order the consumers' earlier reads of this stage before the async writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    const int d = lane;
    int xs = x - cx(d);
    xs = xs < 0 ? xs + P.nx : (xs >= P.nx ? xs - P.nx : xs);
    const int ys = y0 - cy(d);
    T* dst = stage + (size_t)d * G.rows * P.nz;
    const T* src = S.src[d] + (size_t)xs * P.nynz;
    if (ys < 0) {  // first tile row pulls from the last y row
        bulk_g2s(dst, src + (size_t)(P.ny - 1) * P.nz, row_bytes, bar);
        if (rows > 1) bulk_g2s(dst + P.nz, src, (rows - 1) * row_bytes, bar);
    } else if (ys + rows > P.ny) {  // last tile row pulls from y row 0
        if (rows > 1) bulk_g2s(dst, src + (size_t)ys * P.nz, (rows - 1) * row_bytes, bar);
        bulk_g2s(dst + (size_t)(rows - 1) * P.nz, src, row_bytes, bar);
    } else {
        bulk_g2s(dst, src + (size_t)ys * P.nz, rows * row_bytes, bar);
    }
}

// Two shared-memory values of one direction as deviations.
template <class T>
__device__ __forceinline__ float2 sm_pair(const T* row, int za, int zb, int d)
{
    return make_float2(ld_dev_sm(row + za, d), ld_dev_sm(row + zb, d));
}

// Warp-specialised: warps 0-7 compute (two cells per thread), warp 8 is the
// producer.  full[s] completes when stage s holds its tile (one arrival with
// the expected byte count + the copies); empty[s] completes when all 8
// consumer warps have finished reading it.  No block-wide barrier in the loop.
template <class M, int FM, int OUT>
__global__ void __launch_bounds__(TMA_THREADS, 2) k_step_tma(Params P, Streams<typename M::T> S, TileCfg G,
                                                             Outputs<typename M::C> out)
{
    using T = typename M::T;
    extern __shared__ __align__(128) unsigned char tma_smem[];
    __shared__ __align__(8) uint64_t full[TMA_MAX_STAGES];
    __shared__ __align__(8) uint64_t empty[TMA_MAX_STAGES];
    __shared__ int abort_flag;  // set by the first wait of the block that runs out
    // Ring base rounded up to 128 bytes (the launch allocates the slack): every
    // bulk-copy destination is then a multiple of the 16-byte row size.
    T* ring = reinterpret_cast<T*>((reinterpret_cast<uintptr_t>(tma_smem) + 127) & ~(uintptr_t)127);
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < G.stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], TMA_CONSUMER_WARPS);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    volatile int* abort_v = &abort_flag;
    auto give_up = [&]() {
        *abort_v = 1;
        atomicExch(P.err, 1);
    };
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (warp == TMA_CONSUMER_WARPS) {
        // producer: refill each stage once its previous tile has been consumed
        int k = 0;
        for (int t = blockIdx.x; t < G.ntiles; t += gridDim.x, ++k) {
            const int s = k % G.stages;
            if (__any_sync(0xffffffffu, *abort_v != 0)) break;
            bool ok = true;
            if (k >= G.stages) ok = mbar_wait(&empty[s], (uint32_t)(k / G.stages - 1) & 1u);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) give_up();
                break;
            }
            tma_issue_tile<T>(P, S, G, t, ring + (size_t)s * G.stage_elems, &full[s], lane);
        }
        // Drain: the last copy group issued into each stage (tile k - 1 - j
        // sits in stage (k - 1 - j) % stages) must land before the block may
        // retire, whatever happened to the consumers.
        for (int j = 0; j < G.stages && j < k; ++j) {
            const int kk = k - 1 - j;
            const bool ok = mbar_wait(&full[kk % G.stages], (uint32_t)(kk / G.stages) & 1u);
            if (!ok && lane == 0) give_up();
        }
    } else {
        int k = 0;
        for (int t = blockIdx.x; t < G.ntiles; t += gridDim.x, ++k) {
            const int s = k % G.stages;
            const int x = t / G.tiles_y;
            const int y0 = (t - x * G.tiles_y) * G.rows;
            const int tile_pairs = (min(G.rows, P.ny - y0) * P.nz) >> 1;
            const int tile_base = (x * P.ny + y0) * P.nz;
            // The first pair's flags are fetched before the stage wait so the
            // two latencies overlap.
            unsigned short both_next = 0;
            if (P.has_flags && tid < tile_pairs)
                both_next = __ldg(reinterpret_cast<const unsigned short*>(P.flags + tile_base + 2 * tid));
            // After a wait of this block ran out, no thread waits again (the
            // host discards the state); the producer drains its copies.
            // Warp-uniform decisions: a consumer warp leaves the loop as a whole.
            if (__any_sync(0xffffffffu, *abort_v != 0)) break;
            const bool ok = mbar_wait(&full[s], (uint32_t)(k / G.stages) & 1u);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) give_up();
                break;
            }
            const T* st = ring + (size_t)s * G.stage_elems;
            for (int p = tid; p < tile_pairs; p += TMA_CONSUMERS) {
                const int c0 = 2 * p;
                const int r = (int)P.div_nz.div((uint32_t)c0);
                const int z0 = c0 - r * P.nz;
                const int idx0 = tile_base + c0;
                int fl0 = 0, fl1 = 0;
                if (P.has_flags) {
                    const unsigned short both =
                        p == tid ? both_next : __ldg(reinterpret_cast<const unsigned short*>(P.flags + idx0));
                    fl0 = both & 0xff;
                    fl1 = both >> 8;
                }
                const int zm = z0 == 0 ? P.nz - 1 : z0 - 1;
                const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2;
                float2 h[Q];
#pragma unroll
                for (int d = 0; d < Q; ++d) {
                    const T* row = st + ((size_t)d * G.rows + r) * P.nz;
                    if (cz(d) == 0) h[d] = ld_dev2_sm(row + z0, d);
                    else if (cz(d) == 1) h[d] = sm_pair(row, zm, z0, d);
                    else h[d] = sm_pair(row, z0 + 1, zp1, d);
                    h[d] = M::unshift2(P, d, h[d]);
                }
                const int y = y0 + r;
                bool fluid0 = true, fluid1 = true;
                const bool face = on_walled_face(P, x, y, z0) || on_walled_face(P, x, y, z0 + 1);
                if ((fl0 | fl1 | (int)face) != 0) {
                    const Nbr nb0 = make_nbr(P, x, y, z0);
                    fluid0 = resolve_state<M>(P, S, idx0, x, y, z0, fl0, nb0, Lane<0>{h});
                    Nbr nb1 = nb0;
                    nb1.Z[0] = z0;
                    nb1.Z[1] = z0 + 1;
                    nb1.Z[2] = zp1;
                    fluid1 = resolve_state<M>(P, S, idx0 + 1, x, y, z0 + 1, fl1, nb1, Lane<1>{h});
                }
                if constexpr (OUT != OUT_NONE) {
                    float f[Q];
#pragma unroll
                    for (int d = 0; d < Q; ++d) f[d] = h[d].x;
                    emit<M, FM, OUT>(P, out, idx0, !fluid0, f, cons);
#pragma unroll
                    for (int d = 0; d < Q; ++d) f[d] = h[d].y;
                    emit<M, FM, OUT>(P, out, idx0 + 1, !fluid1, f, cons);
                }
                M::template collide2<FM>(P, idx0, h,
                                         [&](int d, float2 v) { store_pair<M>(P, S, idx0, d, v, fluid0, fluid1); });
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
    }
    if constexpr ((OUT & OUT_SUMS) != 0) block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
}

}  // namespace lbm
