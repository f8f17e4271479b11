// lbm_tma.cu -- launch of the TMA-staged step kernel (f32-arithmetic storages).
#include "lbm_launch.h"
#include "lbm_tma.cuh"

namespace lbm {

// Raise a kernel's dynamic shared-memory limit to at least `smem` (the
// attribute is process-wide per kernel; remember the largest value set).
template <class T, int FM, int OUT>
static cudaError_t allow_smem(size_t smem)
{
    static size_t allowed = 0;
    if (smem <= allowed) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_step_tma<ModeFast<T>, FM, OUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) allowed = smem;
    return e;
}

template <class T, int FM, int OUT>
static cudaError_t tma_out(const LaunchArgs& a)
{
    using M = ModeFast<T>;
    auto kern = k_step_tma<M, FM, OUT>;
    const size_t smem = (size_t)a.tile.stages * a.tile.stage_elems * sizeof(T) + 128;
    cudaError_t e = allow_smem<T, FM, OUT>(smem);
    if (e != cudaSuccess) return e;
    Outputs<float> out{(float*)a.rho, (float*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums};
    kern<<<a.tma_grid, TMA_THREADS, smem, a.stream>>>(a.P, make_streams<T>(a.src, a.dst, a.P.n), a.tile, out);
    if (a.grid_used) *a.grid_used = a.tma_grid;
    return cudaGetLastError();
}

template <class T, int FM>
static cudaError_t tma_fm(const LaunchArgs& a)
{
    switch (out_bits(a)) {
    case OUT_NONE: return tma_out<T, FM, OUT_NONE>(a);
    case OUT_RHO_U: return tma_out<T, FM, OUT_RHO_U>(a);
    case OUT_SUMS: return tma_out<T, FM, OUT_SUMS>(a);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
static cudaError_t tma_t(int force_mode, const LaunchArgs& a)
{
    switch (force_mode) {
    case FORCE_NONE: return tma_fm<T, FORCE_NONE>(a);
    case FORCE_UNIFORM: return tma_fm<T, FORCE_UNIFORM>(a);
    case FORCE_FIELD: return tma_fm<T, FORCE_FIELD>(a);
    case FORCE_DRAG: return tma_fm<T, FORCE_DRAG>(a);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_tma_step(int storage, int force_mode, const LaunchArgs& a)
{
    switch (storage) {
    case STORAGE_F32: return tma_t<float>(force_mode, a);
    case STORAGE_F16: return tma_t<__half>(force_mode, a);
    case STORAGE_BF16: return tma_t<__nv_bfloat16>(force_mode, a);
    default: return cudaErrorInvalidValue;
    }
}

template <class T, int FM, int OUT>
static int tma_blocks_per_sm_out(size_t smem)
{
    int blocks = 0;
    if (allow_smem<T, FM, OUT>(smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_step_tma<ModeFast<T>, FM, OUT>, TMA_THREADS,
                                                      smem) != cudaSuccess)
        return 0;
    return blocks;
}

template <class T>
static int tma_blocks_per_sm_t(size_t smem)
{
    return tma_blocks_per_sm_out<T, FORCE_NONE, OUT_NONE>(smem);
}

// Tile geometry for a lattice, or stages = 0 when the TMA path does not apply.
TileCfg plan_tma(int storage, int nx, int ny, int nz, int* grid, int device)
{
    TileCfg G{};
    const size_t S = storage == STORAGE_F32 ? 4 : 2;
    if (storage == STORAGE_F64 || nz % 2 != 0 || (nz * S) % 16 != 0) return G;
    int rows = 1;
    for (int r : {8, 4, 2}) {
        if (r <= ny && (long long)r * nz <= 512) {
            rows = r;
            break;
        }
    }
    if ((long long)rows * nz > 4096) return G;  // one row too long for a stage
    G.rows = rows;
    G.tiles_y = (ny + rows - 1) / rows;
    G.ntiles = nx * G.tiles_y;
    G.stage_elems = Q * rows * nz;
    const size_t stage_bytes = (size_t)G.stage_elems * S;
    int stages = (int)((110 * 1024) / stage_bytes);
    stages = stages > TMA_MAX_STAGES ? TMA_MAX_STAGES : stages;
    if (stages < 2) stages = 2;
    if (stages * stage_bytes > 200 * 1024) return TileCfg{};
    G.stages = stages;
    const size_t smem = stages * stage_bytes + 128;
    int per_sm = 0;
    switch (storage) {
    case STORAGE_F32: per_sm = tma_blocks_per_sm_t<float>(smem); break;
    case STORAGE_F16: per_sm = tma_blocks_per_sm_t<__half>(smem); break;
    default: per_sm = tma_blocks_per_sm_t<__nv_bfloat16>(smem); break;
    }
    int sms = 0;
    if (per_sm < 1 || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1)
        return TileCfg{};
    *grid = G.ntiles < sms * per_sm ? G.ntiles : sms * per_sm;
    return G;
}

}  // namespace lbm
