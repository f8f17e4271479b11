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
    const int grid = grid_for(kernel == KERNEL_OBSERVE ? a.P.n : window_cells(a.P), a.block);
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

cudaError_t launch_persistent_exact(int force_mode, const LaunchArgs& a, int steps, GridBarrier* bar,
                                    unsigned missing, unsigned long long timeout_ns, int* grid_out)
{
    using M = ModeExactT<true>;
    switch (force_mode) {
    case FORCE_NONE: return persistent_t<M, FORCE_NONE, 1>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_UNIFORM: return persistent_t<M, FORCE_UNIFORM, 1>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_FIELD: return persistent_t<M, FORCE_FIELD, 1>(a, steps, bar, missing, timeout_ns, grid_out);
    case FORCE_DRAG: return persistent_t<M, FORCE_DRAG, 1>(a, steps, bar, missing, timeout_ns, grid_out);
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

// ---------------------------------------------------------------------------
// Tier-1 / Tier-2 diagnostics of a rho / u readback on the device
// (Stack-E sim.py:89-109), built --fmad=false so that every value matches
// the reference's NumPy expressions bit for bit (the circulation sum only up
// to its summation order).
// ---------------------------------------------------------------------------

// NumPy's min / max: a NaN anywhere gives NaN.
__device__ __forceinline__ double np_min(double a, double b) { return (a != a || b != b) ? nan("") : (b < a ? b : a); }
__device__ __forceinline__ double np_max(double a, double b) { return (a != a || b != b) ? nan("") : (b > a ? b : a); }

constexpr int DIAG_BLOCK = 256;
constexpr int DIAG_VALUES = 6;  // non-finite count, rho min, rho max, max |u|^2, max |div|, sum u_x (z = 0)

// Block reduction with op (identity: op's neutral value); the result is
// valid in thread 0.  Fixed order: deterministic for a fixed launch shape.
template <class OP>
__device__ __forceinline__ double block_reduce(double v, OP op, double identity, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
    __syncthreads();  // red[] of an earlier call has been read
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? red[lane] : identity;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    return v;
}

struct OpMin { __device__ double operator()(double a, double b) const { return np_min(a, b); } };
struct OpMax { __device__ double operator()(double a, double b) const { return np_max(a, b); } };
struct OpSum { __device__ double operator()(double a, double b) const { return a + b; } };

// Per-block partials over a grid-stride share of the cells.  u_max uses
// sqrt(max s) = max sqrt(s) (sqrt is monotonic and correctly rounded).
__global__ void __launch_bounds__(DIAG_BLOCK) k_diag_partials(Params P, const double* __restrict__ rho,
                                                              const double* __restrict__ u, double inv_2dx,
                                                              double* __restrict__ partials)
{
    __shared__ double red[32];
    double bad = 0.0, rmin = 1.0 / 0.0, rmax = -1.0 / 0.0, smax = -1.0 / 0.0, dmax = 0.0, usum = 0.0;
    const int n = P.n;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const double r = rho[idx], ux = u[idx], uy = u[n + idx], uz = u[2 * n + idx];
        bad += (isfinite(r) && isfinite(ux) && isfinite(uy) && isfinite(uz)) ? 0.0 : 1.0;
        rmin = np_min(rmin, r);
        rmax = np_max(rmax, r);
        smax = np_max(smax, (ux * ux + uy * uy) + uz * uz);
    }
    // z = 0 slice: central differences with periodic wrap in x and y
    const int slice = P.nx * P.ny;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < slice; k += gridDim.x * blockDim.x) {
        const int x = k / P.ny, y = k - x * P.ny;
        const int xp = x + 1 == P.nx ? 0 : x + 1, xm = x == 0 ? P.nx - 1 : x - 1;
        const int yp = y + 1 == P.ny ? 0 : y + 1, ym = y == 0 ? P.ny - 1 : y - 1;
        const double* ux = u;
        const double* uy = u + n;
        const double div = (ux[(xp * P.ny + y) * P.nz] - ux[(xm * P.ny + y) * P.nz]) * inv_2dx +
                           (uy[(x * P.ny + yp) * P.nz] - uy[(x * P.ny + ym) * P.nz]) * inv_2dx;
        dmax = np_max(dmax, fabs(div));
        usum += ux[(x * P.ny + y) * P.nz];
    }
    double* out = partials + (size_t)blockIdx.x * DIAG_VALUES;
    double v;
    v = block_reduce(bad, OpSum{}, 0.0, red);
    if (threadIdx.x == 0) out[0] = v;
    v = block_reduce(rmin, OpMin{}, 1.0 / 0.0, red);
    if (threadIdx.x == 0) out[1] = v;
    v = block_reduce(rmax, OpMax{}, -1.0 / 0.0, red);
    if (threadIdx.x == 0) out[2] = v;
    v = block_reduce(smax, OpMax{}, -1.0 / 0.0, red);
    if (threadIdx.x == 0) out[3] = v;
    v = block_reduce(dmax, OpMax{}, 0.0, red);
    if (threadIdx.x == 0) out[4] = v;
    v = block_reduce(usum, OpSum{}, 0.0, red);
    if (threadIdx.x == 0) out[5] = v;
}

// The block partials -> {check_health, rho_min, rho_max, u_max_lat,
// check_divergence_free, check_circulation} (one block, fixed order).
__global__ void __launch_bounds__(DIAG_BLOCK) k_diag_final(const double* __restrict__ partials, int nblocks,
                                                           double dx, double* __restrict__ out6)
{
    __shared__ double red[32];
    double acc[DIAG_VALUES] = {0.0, 1.0 / 0.0, -1.0 / 0.0, -1.0 / 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        const double* p = partials + (size_t)b * DIAG_VALUES;
        acc[0] += p[0];
        acc[1] = np_min(acc[1], p[1]);
        acc[2] = np_max(acc[2], p[2]);
        acc[3] = np_max(acc[3], p[3]);
        acc[4] = np_max(acc[4], p[4]);
        acc[5] += p[5];
    }
    const double bad = block_reduce(acc[0], OpSum{}, 0.0, red);
    const double rmin = block_reduce(acc[1], OpMin{}, 1.0 / 0.0, red);
    const double rmax = block_reduce(acc[2], OpMax{}, -1.0 / 0.0, red);
    const double smax = block_reduce(acc[3], OpMax{}, -1.0 / 0.0, red);
    const double dmax = block_reduce(acc[4], OpMax{}, 0.0, red);
    const double usum = block_reduce(acc[5], OpSum{}, 0.0, red);
    if (threadIdx.x == 0) {
        out6[0] = bad > 0.0 ? 1.0 : 0.0;
        out6[1] = rmin;
        out6[2] = rmax;
        out6[3] = sqrt(smax);
        out6[4] = dmax;
        out6[5] = usum * dx * dx;
    }
}

int diag_grid(int n)
{
    const int g = (n + DIAG_BLOCK - 1) / DIAG_BLOCK;
    return g < DIAG_MAX_BLOCKS ? g : DIAG_MAX_BLOCKS;
}

cudaError_t launch_diagnostics(const Params& P, const double* rho, const double* u, double dx_phys, double* scratch,
                               double* out6, cudaStream_t s)
{
    const int grid = diag_grid(P.n);
    k_diag_partials<<<grid, DIAG_BLOCK, 0, s>>>(P, rho, u, 0.5 / dx_phys, scratch);
    k_diag_final<<<1, DIAG_BLOCK, 0, s>>>(scratch, grid, dx_phys, out6);
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
