// lbm_kernels.cuh -- kernel templates of the stateful engine.
//
// State machine of a lattice (one storage buffer pair A/B):
//   PRE   buffer holds f_n itself (after set_populations / set_equilibrium).
//   POST  buffer holds P_{n-1} = collide(f_{n-1}); f_n = bounce(stream(P_{n-1}))
//         is rebuilt on the fly by gather + resolve_state.
// A step from PRE runs k_collide_local (read f_n in place, write P_n);
// a step from POST runs k_step, the fused pull-stream + boundary + collide
// kernel that reads P_{n-1} and writes P_n.  Either way the state advances
// by exactly one reference step (d3q19_warp.py bgk_step :321-368 followed by
// apply_bounce_back_y_walls :386-415).
#pragma once

#include "lbm_device.cuh"

#ifndef LBM_STEP2_MIN_BLOCKS
#define LBM_STEP2_MIN_BLOCKS 3
#endif

namespace lbm {

// Tile plan of the TMA-staged step kernel (lbm_tma.cuh).
struct TileCfg {
    int rows;        // y-rows per tile
    int tiles_y;     // ceil(ny / rows)
    int ntiles;      // nx * tiles_y
    int stages;      // pipeline depth; 0 = the TMA path does not apply
    int stage_elems; // 19 * rows * nz
};

// What a kernel writes besides the populations (template parameter OUT).
enum OutBits : int { OUT_NONE = 0, OUT_RHO_U = 1, OUT_SUMS = 2 };

// Optional outputs: rho/u readback of the pre-collision state and per-block
// FP64 conservation partials (mass or mass deviation, m_x, m_y, m_z, cells).
template <class C>
struct Outputs {
    C* rho;                                // (n)
    C* u;                                  // (3, n)
    double* partials;                      // (gridDim.x, 5)
    const double* prev_partials = nullptr; // optional: partials of the previous launch on the
    int prev_count = 0;                    // stream (prev_count rows), which block 0 reduces
    double* prev_sums = nullptr;           // into prev_sums (5)
    int first = 0;                         // k_observe: the window of cells [first,
    int count = -1;                        // first + count); count < 0: all cells
};

// Block-level FP64 reduction of 5 values, fixed tree (deterministic for a
// fixed launch shape).  blockDim.x must be a multiple of 32 and <= 1024.
__device__ __forceinline__ void block_sum5(double v[5], double* out)
{
    __shared__ double red[32][5];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 5; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < 5; ++k) out[k] = v[k];
    }
}

// Grid total of the previous launch's partials, by block 0 of this launch
// (launched after that one on the same stream, so the partials are complete
// and visible): a fixed-order sum, deterministic, that overlaps the other
// blocks' work instead of costing a launch of its own.  Call with every
// thread of the block.
template <class C>
__device__ __forceinline__ void reduce_prev(const Outputs<C>& out)
{
    if (blockIdx.x != 0 || !out.prev_sums) return;
    double w[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < out.prev_count; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 5; ++k) w[k] += out.prev_partials[(size_t)b * 5 + k];
    block_sum5(w, out.prev_sums);
    __syncthreads();  // the shared reduction array is reused by the caller
}

template <class M, int FM, int OUT>
__device__ __forceinline__ void emit(const Params& P, const Outputs<typename M::C>& out, int idx, bool solid,
                                     const typename M::C* f, double* cons)
{
    using C = typename M::C;
    if constexpr ((OUT & OUT_RHO_U) != 0) {
        C r = C(0), u[3] = {C(0), C(0), C(0)};
        if (!solid) M::template readback<FM>(P, idx, f, r, u);
        out.rho[idx] = r;
        out.u[idx] = u[0];
        out.u[P.n + idx] = u[1];
        out.u[2 * P.n + idx] = u[2];
    }
    if constexpr ((OUT & OUT_SUMS) != 0) {
        if (!solid) {
            double m, a, b, c;
            M::cons_terms(f, m, a, b, c);
            cons[0] += m; cons[1] += a; cons[2] += b; cons[3] += c; cons[4] += 1.0;
        }
    }
}

template <class M>
__device__ __forceinline__ void store_all(const Streams<typename M::T>& S, int idx, const typename M::C* f)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) M::store(S.dst[d] + idx, d, f[d]);
}

template <class M>
__device__ __forceinline__ void store_solid(const Params& P, const Streams<typename M::T>& S, int idx)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) M::store(S.dst[d] + idx, d, M::solid(P, d));
}

// Fused step from POST for one cell: f_n = gather + resolve_state(P_{n-1});
// optional outputs of f_n; P_n = collide(f_n).  Solid cells store their rest
// value.  The own-position gather is issued before the flag byte is examined,
// so the 19 loads and the flag load are in flight together.
template <class M, int FM, int OUT>
__device__ __forceinline__ void step_single(const Params& P, const Streams<typename M::T>& S,
                                            const Outputs<typename M::C>& out, int idx, double* cons)
{
    using C = typename M::C;
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int fl = P.has_flags ? (int)P.flags[idx] : 0;
    const Nbr nb = make_nbr(P, x, y, z);
    C f[Q];
    gather<M>(S, nb, f);
    if (resolve_state<M>(P, S, idx, x, y, z, fl, nb, f)) {
        emit<M, FM, OUT>(P, out, idx, false, f, cons);
        M::template collide<FM>(P, idx, f);
        store_all<M>(S, idx, f);
    } else {
        emit<M, FM, OUT>(P, out, idx, true, f, cons);
        store_solid<M>(P, S, idx);
    }
}

template <class M, int FM, int OUT>
__global__ void __launch_bounds__(256) k_step(Params P, Streams<typename M::T> S, Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n) step_single<M, FM, OUT>(P, S, out, idx, cons);
    if constexpr ((OUT & OUT_SUMS) != 0) block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
}

// Fused step from POST, two z-adjacent cells (z0 even, z0 + 1) per thread, for
// the f32-arithmetic storages; requires nz even (both cells share a row, rows
// start at even indices).  Both cells' values of a direction live in one
// float2 and the collision runs in packed f32x2 arithmetic (one FFMA2 / FADD2
// per operation for the two cells).  The 9 directions with c_z = 0 pull both
// values with one vector load, the 10 z-shifted ones with two scalar loads;
// all 19 stores are vector stores.  Cells that need a boundary rule are
// resolved one at a time with the scalar resolve_state.
template <class M, int FM, int OUT>
__device__ __forceinline__ void step_pair(const Params& P, const Streams<typename M::T>& S,
                                          const Outputs<typename M::C>& out, int idx0, double* cons,
                                          bool live = true)
{
    using T = typename M::T;
    int x, y, z0;
    decode_xyz(P, idx0, x, y, z0);
    int fl0 = 0, fl1 = 0;
    if (P.has_flags) {
        const unsigned short both = __ldg(reinterpret_cast<const unsigned short*>(P.flags + idx0));
        fl0 = both & 0xff;
        fl1 = both >> 8;
    }
    const Nbr nb0 = make_nbr(P, x, y, z0);
    const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2; // (z0 + 1) + 1, wrapped
    float2 h[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const T* p = S.src[d] + nb0.X[1 - cx(d)] + nb0.Y[1 - cy(d)];
        if (cz(d) == 0) {
            ld_dev2(p + z0, d, h[d].x, h[d].y);
        } else if (cz(d) == 1) {
            h[d] = ld_dev_pair(p + nb0.Z[0], p + z0, d);
        } else {
            h[d] = ld_dev_pair(p + z0 + 1, p + zp1, d);
        }
    }
    bool fluid0 = true, fluid1 = true;
    const bool face = on_walled_face(P, x, y, z0) || on_walled_face(P, x, y, z0 + 1);
    if ((fl0 | fl1 | (int)face) != 0) {
        fluid0 = resolve_state<M>(P, S, idx0, x, y, z0, fl0, nb0, Lane<0>{h});
        Nbr nb1 = nb0;
        nb1.Z[0] = z0;
        nb1.Z[1] = z0 + 1;
        nb1.Z[2] = zp1;
        fluid1 = resolve_state<M>(P, S, idx0 + 1, x, y, z0 + 1, fl1, nb1, Lane<1>{h});
    }
    if constexpr ((OUT & OUT_RHO_U) != 0) {
        float f[Q];
#pragma unroll
        for (int d = 0; d < Q; ++d) f[d] = h[d].x;
        emit<M, FM, OUT_RHO_U>(P, out, idx0, !fluid0, f, cons);
#pragma unroll
        for (int d = 0; d < Q; ++d) f[d] = h[d].y;
        emit<M, FM, OUT_RHO_U>(P, out, idx0 + 1, !fluid1, f, cons);
    }
    const auto mo = M::template collide2<FM>(P, idx0, h, [&](int d, float2 v) {
        if (live) st_dev2(S.dst[d] + idx0, d, fluid0 ? v.x : M::solid(P, d), fluid1 ? v.y : M::solid(P, d));
    });
    if constexpr ((OUT & OUT_SUMS) != 0) {
        // the collision's own pre-collision moments (density deviation,
        // momentum), assigned: the caller's sums hold this pair only, so they
        // are not live during the step
        const double k0 = live && fluid0 ? 1.0 : 0.0, k1 = live && fluid1 ? 1.0 : 0.0;
        cons[0] = k0 * (double)mo.rd.x + k1 * (double)mo.rd.y;
        cons[1] = k0 * (double)mo.mx.x + k1 * (double)mo.mx.y;
        cons[2] = k0 * (double)mo.my.x + k1 * (double)mo.my.y;
        cons[3] = k0 * (double)mo.mz.x + k1 * (double)mo.mz.y;
        cons[4] = k0 + k1;
    }
}

// Two consecutive cells idx0, idx0 + 1 of any lattice (they may sit in
// different rows, and idx0 + 1 may be past the end) with scalar memory
// accesses and the packed f32x2 collision.  Used by the batched step for
// lattices whose rows are not even-length.
template <class M, int FM>
__device__ __forceinline__ void step_pair_scalar(const Params& P, const Streams<typename M::T>& S, int idx0)
{
    const int idx1 = idx0 + 1 < P.n ? idx0 + 1 : idx0;  // a lone last cell is computed twice, stored once
    int x0, y0, z0, x1, y1, z1;
    decode_xyz(P, idx0, x0, y0, z0);
    decode_xyz(P, idx1, x1, y1, z1);
    const int fl0 = P.has_flags ? (int)P.flags[idx0] : 0;
    const int fl1 = P.has_flags ? (int)P.flags[idx1] : 0;
    const Nbr nb0 = make_nbr(P, x0, y0, z0);
    const Nbr nb1 = make_nbr(P, x1, y1, z1);
    float2 h[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) h[d] = ld_dev_pair(S.src[d] + nb0.src(d), S.src[d] + nb1.src(d), d);
    bool fluid0 = true, fluid1 = true;
    if ((fl0 | fl1 | (int)on_walled_face(P, x0, y0, z0) | (int)on_walled_face(P, x1, y1, z1)) != 0) {
        fluid0 = resolve_state<M>(P, S, idx0, x0, y0, z0, fl0, nb0, Lane<0>{h});
        fluid1 = resolve_state<M>(P, S, idx1, x1, y1, z1, fl1, nb1, Lane<1>{h});
    }
    const bool two = idx1 != idx0;
    // The packed collision reads (cell, cell + 1) pairs of per-cell force
    // inputs; the scalar path serves the force-free and uniform models only.
    static_assert(FM == FORCE_NONE || FM == FORCE_UNIFORM, "step_pair_scalar: per-cell forces unsupported");
    M::template collide2<FM>(P, idx0, h, [&](int d, float2 v) {
        M::store(S.dst[d] + idx0, d, fluid0 ? v.x : M::solid(P, d));
        if (two) M::store(S.dst[d] + idx1, d, fluid1 ? v.y : M::solid(P, d));
    });
}

template <class M, int FM, int OUT>
__global__ void __launch_bounds__(256, LBM_STEP2_MIN_BLOCKS) k_step2(Params P, Streams<typename M::T> S,
                                                                    Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int idx0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if constexpr ((OUT & OUT_SUMS) != 0) {
        // Threads past the end compute the last pair again, store nothing and
        // add nothing: a step with no branch around it and a block reduction
        // after it keeps the register allocation of the plain kernel (a
        // guarded step followed by the reduction spilled ~3x as many bytes).
        const bool live = idx0 < P.n;
        step_pair<M, FM, OUT>(P, S, out, live ? idx0 : P.n - 2, cons, live);
        block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
    } else {
        if (idx0 < P.n) step_pair<M, FM, OUT>(P, S, out, idx0, cons);
    }
}

// Step from PRE for one cell: read f_n in place, collide, write P_n.
template <class M, int FM, int OUT>
__device__ __forceinline__ void collide_single(const Params& P, const Streams<typename M::T>& S,
                                               const Outputs<typename M::C>& out, int idx, double* cons)
{
    using C = typename M::C;
    const int type = P.has_flags ? (P.flags[idx] & 3) : CELL_FLUID;
    C f[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) f[d] = M::load(S.src[d] + idx, d);
    if (type == CELL_SOLID) {
        emit<M, FM, OUT>(P, out, idx, true, f, cons);
        store_solid<M>(P, S, idx);
    } else {
        emit<M, FM, OUT>(P, out, idx, false, f, cons);
        M::template collide<FM>(P, idx, f);
        store_all<M>(S, idx, f);
    }
}

// Step from PRE: S.src holds the buffer base pointers (direction d at S.src[d]).
template <class M, int FM, int OUT>
__global__ void __launch_bounds__(256) k_collide_local(Params P, Streams<typename M::T> S,
                                                       Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n) collide_single<M, FM, OUT>(P, S, out, idx, cons);
    if constexpr ((OUT & OUT_SUMS) != 0) block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
}

// Current state without advancing it: f_n as f64 (optional; used for POST
// states -- a PRE buffer is read out exactly by k_load_f64), readback and
// conservation partials, over the cell window of out (default: all cells).  post = true rebuilds f_n from P_{n-1}; false reads
// the PRE buffer in place.
template <class M, int FM>
__global__ void __launch_bounds__(256) k_observe(Params P, Streams<typename M::T> S, bool post,
                                                 double* __restrict__ f_out, Outputs<typename M::C> out)
{
    using C = typename M::C;
    const int end = out.count < 0 ? P.n : out.first + out.count;
    const int idx = out.first + blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < end) {
        C f[Q];
        bool solid;
        const int fl = P.has_flags ? (int)P.flags[idx] : 0;
        if (post) {
            int x, y, z;
            decode_xyz(P, idx, x, y, z);
            const Nbr nb = make_nbr(P, x, y, z);
            gather<M>(S, nb, f);
            solid = !resolve_state<M>(P, S, idx, x, y, z, fl, nb, f);
            if (solid) {
#pragma unroll
                for (int d = 0; d < Q; ++d) f[d] = M::solid(P, d);
            }
        } else {
            solid = (fl & 3) == CELL_SOLID;
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::load(S.src[d] + idx, d);
        }
        if (f_out) {
#pragma unroll
            for (int d = 0; d < Q; ++d) f_out[(size_t)d * P.n + idx] = M::to_f64(P, d, f[d]);
        }
        if (out.rho) emit<M, FM, OUT_RHO_U>(P, out, idx, solid, f, cons);
        if (out.partials) emit<M, FM, OUT_SUMS>(P, out, idx, solid, f, cons);
    }
    if (out.partials) block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
}

// Sum per-block partials in a fixed order (one block).
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblocks, double* __restrict__ out5);

// f64 array (device) -> storage, with the storage's rounding.
template <class T>
__global__ void k_store_f64(Params P, const double* __restrict__ f, T* __restrict__ dst)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Q * P.n) return;
    const int d = (int)(i / (size_t)P.n);
    st_f64(dst + i, d, f[i], P);
}

// storage -> f64 array (PRE state read-out).
template <class T>
__global__ void k_load_f64(Params P, const T* __restrict__ src, double* __restrict__ f)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)Q * P.n) return;
    const int d = (int)(i / (size_t)P.n);
    f[i] = ld_f64(src + i, d, P);
}

// f = feq(rho, u) with the reference's reciprocal form (equilibrium.py:310-322),
// in f64, then rounded to the storage.  rho / u may be null (1 / 0).
template <class T>
__global__ void k_feq_init(Params P, const double* __restrict__ rho, const double* __restrict__ u,
                           T* __restrict__ dst)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.n) return;
    const double ux = u ? u[c] : 0.0, uy = u ? u[P.n + c] : 0.0, uz = u ? u[2 * P.n + c] : 0.0;
    const double u_sq = ux * ux + uy * uy + uz * uz;
    const double r = rho ? rho[c] : 1.0;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        double cu = (double)cx(d) * ux + (double)cy(d) * uy + (double)cz(d) * uz;
        double feq = P.w[d] * r * (1.0 + cu * P.inv_cs2 + cu * cu * P.inv_two_cs4 - u_sq * P.inv_two_cs2);
        st_f64(dst + (size_t)d * P.n + c, d, feq, P);
    }
}

// Bounce-back masks: for every non-solid cell, bit d set when its pull
// source x - c_d is solid; the flag byte's FLAG_NEAR_SOLID bit mirrors
// mask != 0.
__global__ void k_mark_near_solid(Params P, uint8_t* __restrict__ flags, uint32_t* __restrict__ bbmask);

// Per-direction base pointers of a population buffer of n cells.
template <class T>
inline Streams<T> make_streams(const void* src, void* dst, int n)
{
    Streams<T> S;
    for (int d = 0; d < Q; ++d) {
        S.src[d] = src ? (const T*)src + (size_t)d * n : nullptr;
        S.dst[d] = dst ? (T*)dst + (size_t)d * n : nullptr;
    }
    return S;
}

}  // namespace lbm
