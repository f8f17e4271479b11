// lbm_adjoint.cu -- adjoint level kernels for every storage and force model,
// and the small helpers of the tape API.  Contraction on: the adjoint needs
// no bit-exactness (the forward states it reads are recomputed by the step
// kernels themselves).
#include "lbm_adjoint.cuh"
#include "lbm_launch.h"

// Threads per block of the per-cell adjoint level kernels.
#ifndef LBM_ADJ_BLOCK
#define LBM_ADJ_BLOCK 128
#endif

namespace lbm {

__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, size_t count)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (double)in[i];
}

__global__ void k_check_unit_interval(const float* __restrict__ a, int n, int* __restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(a[i] >= 0.0f && a[i] <= 1.0f)) *flag = 1;
}

__global__ void k_list_special(Params P, int* __restrict__ list, int* __restrict__ count)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.n) return;
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int fl = P.has_flags ? (int)P.flags[idx] : 0;
    if ((fl & 3) != CELL_SOLID && adj_special(P, idx, x, y, z, fl)) list[atomicAdd(count, 1)] = idx;
}

namespace {

template <class M, int FM>
cudaError_t launch_level_m(int level, const AdjointArgs& a)
{
    using T = typename M::T;
    using C = typename M::C;
    AdjIO<C> io{(const C*)a.Lin, (C*)a.Lout, a.grad_rho, a.grad_u, a.dalpha, a.grad_f0};
    const Streams<T> S = make_streams<T>(a.src, nullptr, a.P.n);
    const int block = LBM_ADJ_BLOCK;
    const int grid = grid_for(a.P.n, block);
    const int sb = 128, sg = grid_for(a.n_special, sb);
    cudaStream_t ss = a.special_stream ? a.special_stream : a.stream;
    switch (level) {
    case ADJ_INIT:
        if (a.n_special > 0)
            k_adjoint_special<M, FM, ADJ_INIT><<<sg, sb, 0, ss>>>(a.P, S, io, a.special, a.n_special);
        k_adjoint_plain<M, FM, ADJ_INIT><<<grid, block, 0, a.stream>>>(a.P, S, io);
        break;
    case ADJ_STEP:
        if (a.n_special > 0)
            k_adjoint_special<M, FM, ADJ_STEP><<<sg, sb, 0, ss>>>(a.P, S, io, a.special, a.n_special);
        k_adjoint_plain<M, FM, ADJ_STEP><<<grid, block, 0, a.stream>>>(a.P, S, io);
        break;
    case ADJ_FINAL: k_adjoint_final<M, FM><<<grid, block, 0, a.stream>>>(a.P, S, io); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <class M>
cudaError_t launch_level_fm(int force_mode, int level, const AdjointArgs& a)
{
    switch (force_mode) {
    case FORCE_NONE: return launch_level_m<M, FORCE_NONE>(level, a);
    case FORCE_UNIFORM: return launch_level_m<M, FORCE_UNIFORM>(level, a);
    case FORCE_FIELD: return launch_level_m<M, FORCE_FIELD>(level, a);
    case FORCE_DRAG: return launch_level_m<M, FORCE_DRAG>(level, a);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_adjoint_level(int storage, int force_mode, int level, const AdjointArgs& a)
{
    switch (storage) {
    case STORAGE_F64: return launch_level_fm<ModeExact>(force_mode, level, a);
    case STORAGE_F32: return launch_level_fm<ModeFast<float>>(force_mode, level, a);
    case STORAGE_F16: return launch_level_fm<ModeFast<__half>>(force_mode, level, a);
    case STORAGE_BF16: return launch_level_fm<ModeFast<__nv_bfloat16>>(force_mode, level, a);
    default: return cudaErrorInvalidValue;
    }
}

size_t adjoint_elem_bytes(int storage) { return storage == STORAGE_F64 ? sizeof(double) : sizeof(float); }

cudaError_t launch_list_special(const Params& P, int* list, int* count, cudaStream_t s)
{
    const int block = 256;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    k_list_special<<<grid_for(P.n, block), block, 0, s>>>(P, list, count);
    return cudaGetLastError();
}

cudaError_t launch_widen(const float* in, double* out, size_t count, cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    const int block = 256;
    k_widen<<<(unsigned)((count + block - 1) / block), block, 0, s>>>(in, out, count);
    return cudaGetLastError();
}

cudaError_t launch_check_unit_interval(const float* a, int n, int* flag, cudaStream_t s)
{
    const int block = 256;
    k_check_unit_interval<<<grid_for(n, block), block, 0, s>>>(a, n, flag);
    return cudaGetLastError();
}

}  // namespace lbm
