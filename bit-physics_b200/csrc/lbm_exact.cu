// lbm_exact.cu -- f64 kernels in the reference's operation order.
//
// Built with --fmad=false (no multiply-add contraction), IEEE division, so
// every value matches the reference's NumPy / Warp-CPU f64 arithmetic:
//   stateful engine with f64 storage           (ModeExact)
//   f64 <-> storage conversions, feq init       (all storages: the f64 value
//                                                is rounded once, as the CPU
//                                                oracle's store_round does)
//   the stateless reference functions           (d3q19_warp.py:87-212, :253-415)
#include "lbm_batch.cuh"
#include "lbm_kernels.cuh"
#include "lbm_launch.h"

namespace lbm {

// ---------------------------------------------------------------------------
// Stateful engine, f64 storage
// ---------------------------------------------------------------------------
template <class M, int FM, int OUT>
static void launch_step_out(int kernel, const LaunchArgs& a, int grid)
{
    using T = typename M::T;
    using C = typename M::C;
    Outputs<C> out{(C*)a.rho, (C*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums};
    const Streams<T> S = make_streams<T>(a.src, a.dst, a.P.n);
    if (kernel == KERNEL_STEP)
        k_step<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    else
        k_collide_local<M, FM, OUT><<<grid, a.block, 0, a.stream>>>(a.P, S, out);
    if (a.grid_used) *a.grid_used = grid;
}

template <int FM>
static cudaError_t launch_exact_fm(int kernel, const LaunchArgs& a)
{
    using M = ModeExact;
    const int grid = grid_for(a.P.n, a.block);
    if (kernel == KERNEL_OBSERVE) {
        Outputs<double> out{(double*)a.rho, (double*)a.u, a.partials, a.prev_partials, a.prev_count, a.prev_sums,
                          a.first, a.count};
        const int ogrid = a.count < 0 ? grid : grid_for(a.count, a.block);
        k_observe<M, FM><<<ogrid, a.block, 0, a.stream>>>(a.P, make_streams<double>(a.src, nullptr, a.P.n), a.post,
                                                          a.f_out, out);
        return cudaGetLastError();
    }
    if (kernel != KERNEL_STEP && kernel != KERNEL_COLLIDE_LOCAL) return cudaErrorInvalidValue;
    switch (out_bits(a)) {
    case OUT_NONE: launch_step_out<M, FM, OUT_NONE>(kernel, a, grid); break;
    case OUT_RHO_U: launch_step_out<M, FM, OUT_RHO_U>(kernel, a, grid); break;
    case OUT_SUMS: launch_step_out<M, FM, OUT_SUMS>(kernel, a, grid); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_exact(int kernel, int force_mode, const LaunchArgs& a)
{
    switch (force_mode) {
    case FORCE_NONE: return launch_exact_fm<FORCE_NONE>(kernel, a);
    case FORCE_UNIFORM: return launch_exact_fm<FORCE_UNIFORM>(kernel, a);
    case FORCE_FIELD: return launch_exact_fm<FORCE_FIELD>(kernel, a);
    case FORCE_DRAG: return launch_exact_fm<FORCE_DRAG>(kernel, a);
    default: return cudaErrorInvalidValue;
    }
}

// Batched step, f64 storage (one cell per thread).
template <int FM>
static cudaError_t batch_exact_fm(bool collide, const void* records, const void* items, int nitems, int span,
                                  int phase, int grid, int block, cudaStream_t s)
{
    using M = ModeExact;
    const auto* L = (const BatchLattice<double>*)records;
    const auto* I = (const BatchItem*)items;
    if (collide)
        k_collide_batch<M, FM><<<grid, block, 0, s>>>(L, I, nitems, span, phase);
    else
        k_step_batch<M, FM, SCHED_SINGLE><<<grid, block, 0, s>>>(L, I, nitems, phase);
    return cudaGetLastError();
}

cudaError_t launch_batch_exact(int force_mode, bool collide, const void* records, const void* items, int nitems,
                               int span, int phase, int grid, int block, cudaStream_t s)
{
    switch (force_mode) {
    case FORCE_NONE: return batch_exact_fm<FORCE_NONE>(collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_UNIFORM:
        return batch_exact_fm<FORCE_UNIFORM>(collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_FIELD: return batch_exact_fm<FORCE_FIELD>(collide, records, items, nitems, span, phase, grid, block, s);
    case FORCE_DRAG: return batch_exact_fm<FORCE_DRAG>(collide, records, items, nitems, span, phase, grid, block, s);
    default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Conversions, feq init, flags, reductions (all storages)
// ---------------------------------------------------------------------------
template <class T>
static cudaError_t store_t(const Params& P, const double* f, void* dst, cudaStream_t s)
{
    const int block = 256;
    k_store_f64<T><<<grid_for((long long)Q * P.n, block), block, 0, s>>>(P, f, (T*)dst);
    return cudaGetLastError();
}

cudaError_t launch_store_f64(int storage, const Params& P, const double* f, void* dst, cudaStream_t s)
{
    switch (storage) {
    case STORAGE_F64: return store_t<double>(P, f, dst, s);
    case STORAGE_F32: return store_t<float>(P, f, dst, s);
    case STORAGE_F16: return store_t<__half>(P, f, dst, s);
    case STORAGE_BF16: return store_t<__nv_bfloat16>(P, f, dst, s);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
static cudaError_t load_t(const Params& P, const void* src, double* f, cudaStream_t s)
{
    const int block = 256;
    k_load_f64<T><<<grid_for((long long)Q * P.n, block), block, 0, s>>>(P, (const T*)src, f);
    return cudaGetLastError();
}

cudaError_t launch_load_f64(int storage, const Params& P, const void* src, double* f, cudaStream_t s)
{
    switch (storage) {
    case STORAGE_F64: return load_t<double>(P, src, f, s);
    case STORAGE_F32: return load_t<float>(P, src, f, s);
    case STORAGE_F16: return load_t<__half>(P, src, f, s);
    case STORAGE_BF16: return load_t<__nv_bfloat16>(P, src, f, s);
    default: return cudaErrorInvalidValue;
    }
}

template <class T>
static cudaError_t feq_t(const Params& P, const double* rho, const double* u, void* dst, cudaStream_t s)
{
    const int block = 256;
    k_feq_init<T><<<grid_for(P.n, block), block, 0, s>>>(P, rho, u, (T*)dst);
    return cudaGetLastError();
}

cudaError_t launch_feq_init(int storage, const Params& P, const double* rho, const double* u, void* dst,
                            cudaStream_t s)
{
    switch (storage) {
    case STORAGE_F64: return feq_t<double>(P, rho, u, dst, s);
    case STORAGE_F32: return feq_t<float>(P, rho, u, dst, s);
    case STORAGE_F16: return feq_t<__half>(P, rho, u, dst, s);
    case STORAGE_BF16: return feq_t<__nv_bfloat16>(P, rho, u, dst, s);
    default: return cudaErrorInvalidValue;
    }
}

__global__ void k_mark_near_solid(Params P, uint8_t* __restrict__ flags, uint32_t* __restrict__ bbmask)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.n) return;
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int type = flags[idx] & 3;
    uint32_t mask = 0;
    if (type != CELL_SOLID) {
        const Nbr nb = make_nbr(P, x, y, z);
#pragma unroll
        for (int d = 1; d < Q; ++d)
            if ((flags[nb.src(d)] & 3) == CELL_SOLID) mask |= 1u << d;
    }
    const int fl = type | (mask ? FLAG_NEAR_SOLID : 0);
    bbmask[idx] = mask | ((uint32_t)fl << CW_FLAG_SHIFT);
    // Every thread reads only the low bits of its neighbours, so writing the
    // high bit in place is race-free.
    flags[idx] = (uint8_t)fl;
}

cudaError_t launch_mark_near_solid(const Params& P, uint8_t* flags, uint32_t* bbmask, cudaStream_t s)
{
    const int block = 256;
    k_mark_near_solid<<<grid_for(P.n, block), block, 0, s>>>(P, flags, bbmask);
    return cudaGetLastError();
}

__global__ void k_reduce_partials(const double* __restrict__ partials, int nblocks, double* __restrict__ out5)
{
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] += partials[(size_t)b * 5 + k];
    block_sum5(v, out5);
}

// Plane copies of the x-slab exchange: blockIdx.y picks the k-th direction of
// the mask (dirs[k]); each thread moves words of W bytes between the plane of
// that direction in the stored array and slot k of the packed buffer.
struct PlaneDirs {
    int d[Q];
};

template <class W>
__global__ void k_plane_copy(char* __restrict__ base, size_t dir_stride, size_t plane_off, size_t words,
                             PlaneDirs dirs, char* __restrict__ buf, bool get)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= words) return;
    const int k = blockIdx.y;
    W* plane = reinterpret_cast<W*>(base + (size_t)dirs.d[k] * dir_stride + plane_off);
    W* slot = reinterpret_cast<W*>(buf) + (size_t)k * words;
    if (get) slot[i] = plane[i];
    else plane[i] = slot[i];
}

cudaError_t launch_plane_copy(void* base, size_t dir_stride, size_t plane_off, size_t plane_bytes, uint32_t mask,
                              void* buf, bool get, cudaStream_t s)
{
    PlaneDirs dirs{};
    int count = 0;
    for (int d = 0; d < Q; ++d)
        if ((mask >> d) & 1u) dirs.d[count++] = d;
    if (count == 0) return cudaErrorInvalidValue;
    const int block = 256;
    // 16-byte words when every plane, slot and the buffer are 16-byte aligned
    const bool wide = plane_bytes % 16 == 0 && dir_stride % 16 == 0 && plane_off % 16 == 0 &&
                      reinterpret_cast<uintptr_t>(base) % 16 == 0 && reinterpret_cast<uintptr_t>(buf) % 16 == 0;
    if (wide) {
        const size_t words = plane_bytes / 16;
        const dim3 grid((unsigned)((words + block - 1) / block), (unsigned)count);
        k_plane_copy<uint4><<<grid, block, 0, s>>>((char*)base, dir_stride, plane_off, words, dirs, (char*)buf, get);
    } else {
        const size_t words = plane_bytes / 2;  // every storage element is a multiple of 2 bytes
        const dim3 grid((unsigned)((words + block - 1) / block), (unsigned)count);
        k_plane_copy<unsigned short><<<grid, block, 0, s>>>((char*)base, dir_stride, plane_off, words, dirs,
                                                            (char*)buf, get);
    }
    return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const double* partials, int nblocks, double* out5, cudaStream_t s)
{
    // one block of 1024 threads: a readback of 4.2 M cells in 128-thread
    // blocks leaves 32,768 partial rows, reduced in 23 us (58 with 256)
    k_reduce_partials<<<1, 1024, 0, s>>>(partials, nblocks, out5);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stateless reference functions (d3q19_warp.py)
// ---------------------------------------------------------------------------

// _k_feq_field (d3q19_warp.py:87-108)
__global__ void k_ref_feq_field(Params P, const double* __restrict__ rho, const double* __restrict__ u,
                                double* __restrict__ feq)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const double ux = u[c], uy = u[P.n + c], uz = u[2 * P.n + c];
    const double u_sq = ux * ux + uy * uy + uz * uz;
    const double r = rho[c];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        double cu = (double)cx(d) * ux + (double)cy(d) * uy + (double)cz(d) * uz;
        feq[(size_t)d * P.n + c] = P.w[d] * r * (1.0 + cu * P.inv_cs2 + cu * cu * P.inv_two_cs4 - u_sq * P.inv_two_cs2);
    }
}

// _k_density_field (d3q19_warp.py:111-120)
__global__ void k_ref_density(Params P, const double* __restrict__ f, double* __restrict__ rho)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < Q; ++d) acc = acc + f[(size_t)d * P.n + c];
    rho[c] = acc;
}

// _k_momentum_field (d3q19_warp.py:123-140)
__global__ void k_ref_momentum(Params P, const double* __restrict__ f, double* __restrict__ mom)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    double mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const double fd = f[(size_t)d * P.n + c];
        mx = mx + (double)cx(d) * fd;
        my = my + (double)cy(d) * fd;
        mz = mz + (double)cz(d) * fd;
    }
    mom[c] = mx;
    mom[P.n + c] = my;
    mom[2 * P.n + c] = mz;
}

// macroscopic_velocity (d3q19_warp.py:371-383): (m [+ 0.5 F]) / max(rho, 1e-30)
__global__ void k_ref_macro_u(Params P, const double* __restrict__ f, const double* __restrict__ force,
                              double* __restrict__ u)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    double r = 0.0, m[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const double fd = f[(size_t)d * P.n + c];
        r = r + fd;
        m[0] = m[0] + (double)cx(d) * fd;
        m[1] = m[1] + (double)cy(d) * fd;
        m[2] = m[2] + (double)cz(d) * fd;
    }
    const double rs = rho_safe(r);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double ma = m[a];
        if (force) ma = ma + 0.5 * force[(size_t)a * P.n + c];
        u[(size_t)a * P.n + c] = ma / rs;
    }
}

// _k_stream (d3q19_warp.py:198-212): out[d, x] = in[d, (x - c_d) mod n]
__global__ void k_ref_stream(Params P, const double* __restrict__ fin, double* __restrict__ fout)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    int x, y, z;
    decode_xyz(P, c, x, y, z);
    const Nbr nb = make_nbr(P, x, y, z);
#pragma unroll
    for (int d = 0; d < Q; ++d) fout[(size_t)d * P.n + c] = fin[(size_t)d * P.n + nb.src(d)];
}

// bgk_step (d3q19_warp.py:321-368): _k_collide_guo then _k_stream, fused as
// collide-in-place + push to (x + c_d) mod n.  Each output element is written
// by exactly one thread.
template <int FM>
__global__ void k_ref_bgk_step(Params P, const double* __restrict__ f, double* __restrict__ fout)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    int x, y, z;
    decode_xyz(P, c, x, y, z);
    double fl[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) fl[d] = f[(size_t)d * P.n + c];
    ModeExact::collide<FM>(P, c, fl);
    const Nbr nb = make_nbr(P, x, y, z);
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        fout[(size_t)d * P.n + nb.dst(d)] = fl[d];
    }
}

// apply_bounce_back_y_walls (d3q19_warp.py:386-415): copy, then at y = 0
// replace c_y > 0 directions and at y = ny-1 replace c_y < 0 directions by
// f[opp] + (-2 w rho_wall (c . u_wall) / c_s^2), all read from the input.
__global__ void k_ref_bounce_y(Params P, const double* __restrict__ f, double* __restrict__ fout)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    int x, y, z;
    decode_xyz(P, c, x, y, z);
    double fl[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) fl[d] = f[(size_t)d * P.n + c];
    double out[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) out[d] = fl[d];
    if (y == 0 || y == P.ny - 1) {
        const double rho_wall = ModeExact::rho_wall(P, fl);
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            if (cy(d) > 0 && y == 0) out[d] = fl[opp(d)] + ModeExact::inject(P, FACE_YM, d, rho_wall);
            if (cy(d) < 0 && y == P.ny - 1) out[d] = fl[opp(d)] + ModeExact::inject(P, FACE_YP, d, rho_wall);
        }
    }
#pragma unroll
    for (int d = 0; d < Q; ++d) fout[(size_t)d * P.n + c] = out[d];
}

static constexpr int REF_BLOCK = 256;

cudaError_t ref_feq_field(const Params& P, const double* rho, const double* u, double* feq, cudaStream_t s)
{
    k_ref_feq_field<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, rho, u, feq);
    return cudaGetLastError();
}
cudaError_t ref_density(const Params& P, const double* f, double* rho, cudaStream_t s)
{
    k_ref_density<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, f, rho);
    return cudaGetLastError();
}
cudaError_t ref_momentum(const Params& P, const double* f, double* mom, cudaStream_t s)
{
    k_ref_momentum<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, f, mom);
    return cudaGetLastError();
}
cudaError_t ref_macro_velocity(const Params& P, const double* f, const double* force, double* u, cudaStream_t s)
{
    k_ref_macro_u<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, f, force, u);
    return cudaGetLastError();
}
cudaError_t ref_stream(const Params& P, const double* fin, double* fout, cudaStream_t s)
{
    k_ref_stream<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, fin, fout);
    return cudaGetLastError();
}
cudaError_t ref_bgk_step(const Params& P, const double* f, const double* force, double* fout, cudaStream_t s)
{
    if (force) {
        Params Q2 = P;
        Q2.force = force;
        k_ref_bgk_step<FORCE_FIELD><<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(Q2, f, fout);
    } else {
        k_ref_bgk_step<FORCE_NONE><<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, f, fout);
    }
    return cudaGetLastError();
}
cudaError_t ref_bounce_y(const Params& P, const double* f, double* fout, cudaStream_t s)
{
    k_ref_bounce_y<<<grid_for(P.n, REF_BLOCK), REF_BLOCK, 0, s>>>(P, f, fout);
    return cudaGetLastError();
}

}  // namespace lbm
