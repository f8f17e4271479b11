// lbm_fast.cu -- f32-arithmetic step kernels for f32, binary16-shift and
// bfloat16-shift storage (ModeFast).  Built with multiply-add contraction on.
#include "lbm_batch.cuh"
#include "lbm_kernels.cuh"
#include "lbm_launch.h"

namespace lbm {

__global__ void k_list_rule_quads(Params P, int* __restrict__ lists, int cap, int* __restrict__ counts)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int idx0 = 4 * q;
    if (idx0 >= P.n) return;
    int x, y, z0;
    decode_xyz(P, idx0, x, y, z0);
    const uint32_t fl4 = P.has_flags ? *reinterpret_cast<const uint32_t*>(P.flags + idx0) : 0u;
    const bool face = quad_on_walled_face(P, x, y, z0);
    if (!face && (fl4 == 0u || fl4 == QUAD_SOLID || fl4 == QUAD_INFLOW)) return;  // k_step4 steps it
    int kind = QUAD_KIND_OTHER;
    if (!face) {
        // bytes of four cells, each fluid or solid (near-solid bits allowed)
        const uint32_t t = fl4 & 0x03030303u;
        const bool fluid_or_solid = ((t & 0x02020202u) == 0u);
        if (fluid_or_solid) {
            kind = QUAD_KIND_NEAR;
        } else if (fl4 == QUAD_OUTFLOW) {
            const int gx = x == 0 ? P.nx - 1 : x - 1;
            const uint32_t g4 = *reinterpret_cast<const uint32_t*>(P.flags + idx0 + (gx - x) * P.nynz);
            if (g4 == 0u && !quad_on_walled_face(P, gx, y, z0)) kind = QUAD_KIND_OUTFLOW;
        }
    }
    lists[(size_t)kind * cap + atomicAdd(counts + kind, 1)] = q;
}

__global__ void k_face_order(Params P, int vec, int* __restrict__ order, int* __restrict__ face_count)
{
    const int nzi = P.nz / vec;  // items per row
    const int items = P.n / vec;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= items) return;
    int x, y, z0;
    decode_xyz(P, p * vec, x, y, z0);
    const int zi = z0 / vec;
    const int xo = P.walled[0] ? 1 : 0, yo = P.walled[1] ? 1 : 0, zo = P.walled[2] ? 1 : 0;
    const int bx = P.nx - 2 * xo, by = P.ny - 2 * yo, bz = nzi - 2 * zo;
    const bool inner = bx > 0 && by > 0 && bz > 0 && x >= xo && x < P.nx - xo && y >= yo && y < P.ny - yo &&
                       zi >= zo && zi < nzi - zo;
    const int n_inner = bx > 0 && by > 0 && bz > 0 ? bx * by * bz : 0;
    if (inner)
        order[items - n_inner + ((x - xo) * by + (y - yo)) * bz + (zi - zo)] = p;
    else
        order[atomicAdd(face_count, 1)] = p;
}

cudaError_t launch_face_order(const Params& P, int vec, int* order, int* face_count, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(face_count, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    k_face_order<<<grid_for(P.n / vec, 256), 256, 0, s>>>(P, vec, order, face_count);
    return cudaGetLastError();
}

cudaError_t launch_list_rule_quads(const Params& P, int* lists, int cap, int* counts, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * QUAD_KINDS, s);
    if (e != cudaSuccess) return e;
    k_list_rule_quads<<<grid_for(P.n / 4, 256), 256, 0, s>>>(P, lists, cap, counts);
    return cudaGetLastError();
}

// k_step4 over the window's quads, led by the blocks that step the rule quads
// (a.rules_grid of them, at most one task per thread).
template <class M, int FM>
static cudaError_t launch_step4(const LaunchArgs& a, const Streams<typename M::T>& S)
{
    const int total = a.rule_counts[0] + a.rule_counts[1] + a.rule_counts[2];
    const size_t cap = (size_t)a.P.n / 4;
    const int* L = a.rule_quads;
    RuleQuads rq{L + QUAD_KIND_NEAR * cap, L + QUAD_KIND_OUTFLOW * cap, L + QUAD_KIND_OTHER * cap,
                 a.rule_counts[QUAD_KIND_NEAR], a.rule_counts[QUAD_KIND_OUTFLOW], a.rule_counts[QUAD_KIND_OTHER], 0};
    const int block = a.block < 128 ? a.block : 128;  // the kernel's bound
    if (total > 0) {
        const int one_each = grid_for(2LL * total, block);
        rq.blocks = a.rules_grid > 0 && a.rules_grid < one_each ? a.rules_grid : one_each;
    }
    k_step4<M, FM><<<rq.blocks + grid_for(window_cells(a.P) / 4, block), block, 0, a.stream>>>(a.P, S, rq);
    return cudaGetLastError();
}

template <class M, int FM, int OUT>
static cudaError_t launch_step_out(int kernel, const LaunchArgs& a, int grid)
{
    using T = typename M::T;
    Outputs<float> out{(float*)a.rho, (float*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums};
    const Streams<T> S = make_streams<T>(a.src, a.dst, a.P.n);
    if constexpr (sizeof(T) == 2 && OUT == OUT_NONE) {
        if (kernel == KERNEL_STEP && a.vec == 2 && a.pipe_grid > 0) {
            k_step2_pipe<M, FM><<<a.pipe_grid, a.block, 0, a.stream>>>(a.P, S);
            if (a.grid_used) *a.grid_used = a.pipe_grid;
            return cudaGetLastError();
        }
        if (kernel == KERNEL_STEP && a.vec == 4) return launch_step4<M, FM>(a, S);
    }
    // Steps with readback or sums of a four-cell lattice run the two-cell kernels.
    if constexpr (OUT == OUT_SUMS) {
        if (kernel == KERNEL_STEP && a.vec >= 2 && a.sums_grid > 0) {
            k_step2_sums<M, FM><<<a.sums_grid, a.block, 0, a.stream>>>(a.P, S, out);
            if (a.grid_used) *a.grid_used = a.sums_grid;
            return cudaGetLastError();
        }
    }
    if (kernel == KERNEL_STEP && a.vec >= 2) {
        // at most the kernel's bound (128 threads for 16-bit storage)
        const int block = a.block < Step2Bounds<T>::threads ? a.block : Step2Bounds<T>::threads;
        const int grid2 = grid_for(window_cells(a.P) / 2, block);
        k_step2<M, FM, OUT><<<grid2, block, 0, a.stream>>>(a.P, S, out);
        if (a.grid_used) *a.grid_used = grid2;
        return cudaGetLastError();
    }
    if (kernel == KERNEL_STEP)
        k_step<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    else
        k_collide_local<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    if (a.grid_used) *a.grid_used = grid;
    return cudaGetLastError();
}

template <class T, int FM>
static cudaError_t launch_fast_t(int kernel, const LaunchArgs& a)
{
    using M = ModeFast<T>;
    const int grid = grid_for(kernel == KERNEL_OBSERVE ? a.P.n : window_cells(a.P), a.block);
    if (kernel == KERNEL_OBSERVE) {
        Outputs<float> out{(float*)a.rho, (float*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums,
                          a.first, a.count};
        const int ogrid = a.count < 0 ? grid : grid_for(a.count, a.block);
        k_observe<M, FM><<<ogrid, a.block, 0, a.stream>>>(a.P, make_streams<T>(a.src, nullptr, a.P.n), a.post,
                                                          a.f_out, out);
        return cudaGetLastError();
    }
    if (kernel != KERNEL_STEP && kernel != KERNEL_COLLIDE_LOCAL) return cudaErrorInvalidValue;
    if ((a.vec == 2 && (a.P.nz % 2) != 0) || (a.vec == 4 && (a.P.nz % 4 != 0 || sizeof(T) != 2)))
        return cudaErrorInvalidValue;
    switch (out_bits(a)) {
    case OUT_NONE: return launch_step_out<M, FM, OUT_NONE>(kernel, a, grid);
    case OUT_RHO_U: return launch_step_out<M, FM, OUT_RHO_U>(kernel, a, grid);
    case OUT_SUMS: return launch_step_out<M, FM, OUT_SUMS>(kernel, a, grid);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
static cudaError_t launch_fast_fm(int kernel, int force_mode, const LaunchArgs& a)
{
    switch (force_mode) {
    case FORCE_NONE: return launch_fast_t<T, FORCE_NONE>(kernel, a);
    case FORCE_UNIFORM: return launch_fast_t<T, FORCE_UNIFORM>(kernel, a);
    case FORCE_FIELD: return launch_fast_t<T, FORCE_FIELD>(kernel, a);
    case FORCE_DRAG: return launch_fast_t<T, FORCE_DRAG>(kernel, a);
    default: return cudaErrorInvalidValue;
    }
}

template <class T, int FM>
static cudaError_t batch_fm(int sched, bool collide, const void* records, const void* items, int nitems, int span,
                            int phase, int grid, int block, cudaStream_t s)
{
    using M = ModeFast<T>;
    const auto* L = (const BatchLattice<T>*)records;
    const auto* I = (const BatchItem*)items;
    if (collide) {
        k_collide_batch<M, FM><<<grid, block, 0, s>>>(L, I, nitems, span, phase);
        return cudaGetLastError();
    }
    if constexpr (FM == FORCE_NONE || FM == FORCE_UNIFORM) {
        if (sched == SCHED_PAIR_SCALAR) {
            k_step_batch<M, FM, SCHED_PAIR_SCALAR><<<grid, block, 0, s>>>(L, I, nitems, phase);
            return cudaGetLastError();
        }
        if (sched == SCHED_PAIR_MIXED) {
            k_step_batch<M, FM, SCHED_PAIR_MIXED><<<grid, block, 0, s>>>(L, I, nitems, phase);
            return cudaGetLastError();
        }
    }
    if (sched != SCHED_SINGLE) return cudaErrorInvalidValue;
    k_step_batch<M, FM, SCHED_SINGLE><<<grid, block, 0, s>>>(L, I, nitems, phase);
    return cudaGetLastError();
}

template <class T>
static cudaError_t batch_t(int force_mode, int sched, bool collide, const void* records, const void* items,
                           int nitems, int span, int phase, int grid, int block, cudaStream_t s)
{
    switch (force_mode) {
    case FORCE_NONE: return batch_fm<T, FORCE_NONE>(sched, collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_UNIFORM:
        return batch_fm<T, FORCE_UNIFORM>(sched, collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_FIELD:
        return batch_fm<T, FORCE_FIELD>(sched, collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_DRAG: return batch_fm<T, FORCE_DRAG>(sched, collide, records, items, nitems, span, phase, grid, block, s);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_exact(int force_mode, bool collide, const void* records, const void* items, int nitems,
                               int span, int phase, int grid, int block, cudaStream_t s);

cudaError_t launch_batch_step(int storage, int force_mode, int sched, bool collide, const void* records,
                              const void* items, int nitems, int span, int phase, int grid, int block,
                              cudaStream_t s)
{
    switch (storage) {
    case STORAGE_F64:
        if (sched != SCHED_SINGLE && !collide) return cudaErrorInvalidValue;
        return launch_batch_exact(force_mode, collide, records, items, nitems, span, phase, grid, block, s);
    case STORAGE_F32:
        return batch_t<float>(force_mode, sched, collide, records, items, nitems, span, phase, grid, block, s);
    case STORAGE_F16:
        return batch_t<__half>(force_mode, sched, collide, records, items, nitems, span, phase, grid, block, s);
    case STORAGE_BF16:
        return batch_t<__nv_bfloat16>(force_mode, sched, collide, records, items, nitems, span, phase, grid, block,
                                      s);
    default: return cudaErrorInvalidValue;
    }
}

size_t batch_record_bytes(int storage)
{
    switch (storage) {
    case STORAGE_F64: return sizeof(BatchLattice<double>);
    case STORAGE_F32: return sizeof(BatchLattice<float>);
    case STORAGE_F16: return sizeof(BatchLattice<__half>);
    case STORAGE_BF16: return sizeof(BatchLattice<__nv_bfloat16>);
    default: return 0;
    }
}

// Resident blocks per SM x SMs of the current device for a kernel.
template <class K>
static int resident_grid(K kernel, int block)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess) return 0;
    return sms * per_sm;
}

template <class T, int FM>
static int loop_grid_t(bool sums, int block)
{
    if (sums) return resident_grid(k_step2_sums<ModeFast<T>, FM>, block);
    if constexpr (sizeof(T) == 2) return resident_grid(k_step2_pipe<ModeFast<T>, FM>, block);
    return 0;
}

template <class T>
static int loop_grid_fm(bool sums, int force_mode, int block)
{
    switch (force_mode) {
    case FORCE_NONE: return loop_grid_t<T, FORCE_NONE>(sums, block);
    case FORCE_UNIFORM: return loop_grid_t<T, FORCE_UNIFORM>(sums, block);
    case FORCE_FIELD: return loop_grid_t<T, FORCE_FIELD>(sums, block);
    case FORCE_DRAG: return loop_grid_t<T, FORCE_DRAG>(sums, block);
    default: return 0;
    }
}

static int loop_grid(bool sums, int storage, int force_mode, int block)
{
    switch (storage) {
    case STORAGE_F32: return loop_grid_fm<float>(sums, force_mode, block);
    case STORAGE_F16: return loop_grid_fm<__half>(sums, force_mode, block);
    case STORAGE_BF16: return loop_grid_fm<__nv_bfloat16>(sums, force_mode, block);
    default: return 0;
    }
}

int pipe_grid_fast(int storage, int force_mode, int block) { return loop_grid(false, storage, force_mode, block); }

int sums_grid_fast(int storage, int force_mode, int block) { return loop_grid(true, storage, force_mode, block); }

template <class T, int FM>
static cudaError_t persistent_fm_t(const LaunchArgs& a, int steps, GridBarrier* bar, unsigned missing,
                                   unsigned long long timeout_ns, int* grid_out)
{
    if (a.vec >= 2) return persistent_t<ModeFast<T, true>, FM, 2>(a, steps, bar, missing, timeout_ns, grid_out);
    return persistent_t<ModeFast<T, true>, FM, 1>(a, steps, bar, missing, timeout_ns, grid_out);
}

template <class T>
static cudaError_t persistent_fast_t(int force_mode, const LaunchArgs& a, int steps, GridBarrier* bar,
                                     unsigned missing, unsigned long long timeout_ns, int* grid_out)
{
    switch (force_mode) {
    case FORCE_NONE: return persistent_fm_t<T, FORCE_NONE>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_UNIFORM: return persistent_fm_t<T, FORCE_UNIFORM>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_FIELD: return persistent_fm_t<T, FORCE_FIELD>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_DRAG: return persistent_fm_t<T, FORCE_DRAG>(a, steps, bar, missing, timeout_ns, grid_out);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_persistent_exact(int force_mode, const LaunchArgs& a, int steps, GridBarrier* bar,
                                    unsigned missing, unsigned long long timeout_ns, int* grid_out);

cudaError_t launch_persistent(int storage, int force_mode, const LaunchArgs& a, int steps, GridBarrier* bar,
                              unsigned missing, unsigned long long timeout_ns, int* grid_out)
{
    switch (storage) {
    case STORAGE_F64: return launch_persistent_exact(force_mode, a, steps, bar, missing, timeout_ns, grid_out);
    case STORAGE_F32: return persistent_fast_t<float>(force_mode, a, steps, bar, missing, timeout_ns, grid_out);
    case STORAGE_F16: return persistent_fast_t<__half>(force_mode, a, steps, bar, missing, timeout_ns, grid_out);
    case STORAGE_BF16:
        return persistent_fast_t<__nv_bfloat16>(force_mode, a, steps, bar, missing, timeout_ns, grid_out);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fast(int storage, int kernel, int force_mode, const LaunchArgs& a)
{
    switch (storage) {
    case STORAGE_F32: return launch_fast_fm<float>(kernel, force_mode, a);
    case STORAGE_F16: return launch_fast_fm<__half>(kernel, force_mode, a);
    case STORAGE_BF16: return launch_fast_fm<__nv_bfloat16>(kernel, force_mode, a);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace lbm
