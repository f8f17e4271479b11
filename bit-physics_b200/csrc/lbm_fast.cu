// lbm_fast.cu -- f32-arithmetic step kernels for f32, binary16-shift and
// bfloat16-shift storage (ModeFast).  Built with multiply-add contraction on.
#include "lbm_batch.cuh"
#include "lbm_kernels.cuh"
#include "lbm_launch.h"

namespace lbm {

template <class M, int FM, int OUT>
static void launch_step_out(int kernel, const LaunchArgs& a, int grid)
{
    using T = typename M::T;
    Outputs<float> out{(float*)a.rho, (float*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums};
    const Streams<T> S = make_streams<T>(a.src, a.dst, a.P.n);
    if constexpr (sizeof(T) == 2 && OUT == OUT_NONE) {
        if (kernel == KERNEL_STEP && a.vec == 2 && a.pipe_grid > 0) {
            k_step2_pipe<M, FM><<<a.pipe_grid, a.block, 0, a.stream>>>(a.P, S);
            if (a.grid_used) *a.grid_used = a.pipe_grid;
            return;
        }
    }
    if constexpr (OUT == OUT_SUMS) {
        if (kernel == KERNEL_STEP && a.vec == 2 && a.sums_grid > 0) {
            k_step2_sums<M, FM><<<a.sums_grid, a.block, 0, a.stream>>>(a.P, S, out);
            if (a.grid_used) *a.grid_used = a.sums_grid;
            return;
        }
    }
    if (kernel == KERNEL_STEP && a.vec == 2) {
        // at most the kernel's bound (128 threads for 16-bit storage)
        const int block = a.block < Step2Bounds<T>::threads ? a.block : Step2Bounds<T>::threads;
        const int grid2 = grid_for(a.P.n / 2, block);
        k_step2<M, FM, OUT><<<grid2, block, 0, a.stream>>>(a.P, S, out);
        if (a.grid_used) *a.grid_used = grid2;
        return;
    }
    if (kernel == KERNEL_STEP)
        k_step<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    else
        k_collide_local<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    if (a.grid_used) *a.grid_used = grid;
}

template <class T, int FM>
static cudaError_t launch_fast_t(int kernel, const LaunchArgs& a)
{
    using M = ModeFast<T>;
    const int grid = grid_for(a.P.n, a.block);
    if (kernel == KERNEL_OBSERVE) {
        Outputs<float> out{(float*)a.rho, (float*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums,
                          a.first, a.count};
        const int ogrid = a.count < 0 ? grid : grid_for(a.count, a.block);
        k_observe<M, FM><<<ogrid, a.block, 0, a.stream>>>(a.P, make_streams<T>(a.src, nullptr, a.P.n), a.post,
                                                          a.f_out, out);
        return cudaGetLastError();
    }
    if (kernel != KERNEL_STEP && kernel != KERNEL_COLLIDE_LOCAL) return cudaErrorInvalidValue;
    if (a.vec == 2 && (a.P.nz % 2) != 0) return cudaErrorInvalidValue;
    switch (out_bits(a)) {
    case OUT_NONE: launch_step_out<M, FM, OUT_NONE>(kernel, a, grid); break;
    case OUT_RHO_U: launch_step_out<M, FM, OUT_RHO_U>(kernel, a, grid); break;
    case OUT_SUMS: launch_step_out<M, FM, OUT_SUMS>(kernel, a, grid); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
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
