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
// k_step2_sums at 2 blocks of 256 per SM (128 registers, no spills) against
// 3 (80 registers, 204 B of spill stores): steps with FP64 sums, f32 sphere
// channel, 34.5 against 32.2 GLUPS.
#ifndef LBM_SUMS_MIN_BLOCKS
#define LBM_SUMS_MIN_BLOCKS 2
#endif
// Which two-cell step kernels read the 32-bit cell words (flag byte and
// bounce-back mask in one load) instead of the flag bytes: 0 none, 1 the
// 16-bit storages, 2 all.  Measured on the 256x128x128 sphere channel: f32
// 36.2 GLUPS with cell words against 39.0 with flag bytes (4 B per cell
// read instead of 1); f16 / bf16 equal or faster.
#ifndef LBM_CELL_WORD
#define LBM_CELL_WORD 1
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
__device__ __forceinline__ void store_all(const Params& P, const Streams<typename M::T>& S, int idx,
                                          const typename M::C* f)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) M::store(P, S.dst[d] + idx, d, f[d]);
}

template <class M>
__device__ __forceinline__ void store_solid(const Params& P, const Streams<typename M::T>& S, int idx)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) M::store(P, S.dst[d] + idx, d, M::solid(P, d));
}

// Post-collision direction d of a pair (cells idx0, idx0 + 1 of one row) as
// one vector store; a solid cell stores its rest state.
template <class M>
__device__ __forceinline__ void store_pair(const Params& P, const Streams<typename M::T>& S, int idx0, int d,
                                           float2 v, bool fluid0, bool fluid1)
{
    const float2 s = M::shift2(P, d, make_float2(fluid0 ? v.x : M::solid(P, d), fluid1 ? v.y : M::solid(P, d)));
    st_dev2(S.dst[d] + idx0, d, s.x, s.y);
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
    gather<M>(P, S, nb, f);
    if (resolve_state<M>(P, S, idx, x, y, z, fl, nb, f)) {
        emit<M, FM, OUT>(P, out, idx, false, f, cons);
        M::template collide<FM>(P, idx, f);
        store_all<M>(P, S, idx, f);
    } else {
        emit<M, FM, OUT>(P, out, idx, true, f, cons);
        store_solid<M>(P, S, idx);
    }
}

// One cell per thread (f64 storage; odd-nz f32-arithmetic lattices).  At 3
// blocks of 256 per SM the f64 kernel runs in 80 registers (93 unbounded,
// 2 blocks): 17.1 against 14.5 GLUPS on the 256x128x128 sphere channel with
// 128-thread blocks; f64 results do not depend on it (no contraction).
template <class M, int FM, int OUT>
__global__ void __launch_bounds__(256, 3) k_step(Params P, Streams<typename M::T> S, Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int t = P.cell0 + blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (t < P.n && t < P.cell_end) {
        int idx = t;
        if constexpr (OUT == OUT_NONE)
            if (P.order) idx = __ldg(P.order + t);
        step_single<M, FM, OUT>(P, S, out, idx, cons);
    }
    if constexpr ((OUT & OUT_SUMS) != 0) block_sum5(cons, out.partials + (size_t)blockIdx.x * 5);
}

// Plain pull gather of the pair (x, y, z0), (x, y, z0 + 1) described by nb
// (zp1 = z0 + 2, wrapped): the c_z = 0 directions as one vector load.
template <class M>
__device__ __forceinline__ void gather_pair(const Params& P, const Streams<typename M::T>& S, const Nbr& nb, int z0,
                                            int zp1, float2* h)
{
    using T = typename M::T;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const T* p = S.src[d] + nb.X[1 - cx(d)] + nb.Y[1 - cy(d)];
        if (cz(d) == 0) {
            ld_dev2<M::cg>(p + z0, d, h[d].x, h[d].y);
        } else if (cz(d) == 1) {
            h[d] = ld_dev_pair<M::cg>(p + nb.Z[0], p + z0, d);
        } else {
            h[d] = ld_dev_pair<M::cg>(p + z0 + 1, p + zp1, d);
        }
        h[d] = M::unshift2(P, d, h[d]);
    }
}

// Boundary rules of a pair (cells idx0, idx0 + 1 of one row) after the
// speculative own-position gather h.  The common case -- neither cell on a
// walled face nor an inflow / outflow cell, i.e. fluid or solid cells, some
// next to a solid -- is resolved for both cells at once: their bounce-back
// masks (passed in with CW, else one 8-byte load), then all half-way
// bounce-back loads of both cells in one batch, instead of the per-cell
// resolve_state one cell after the other (two dependent memory latencies per
// cell).  Everything else goes through resolve_state per cell.
template <bool CW>
struct PairMasks {
    uint32_t m0 = 0u, m1 = 0u;  // with CW: the cells' masks (zero for solid cells)
};

template <class M, bool CW>
__device__ __forceinline__ void resolve_pair(const Params& P, const Streams<typename M::T>& S, int idx0, int x,
                                             int y, int z0, int fl0, int fl1, bool face, const Nbr& nb0, int zp1,
                                             float2* h, bool& fluid0, bool& fluid1, PairMasks<CW> cm = {})
{
    const int t0 = fl0 & 3, t1 = fl1 & 3;
    const bool plain0 = t0 == CELL_FLUID || t0 == CELL_SOLID, plain1 = t1 == CELL_FLUID || t1 == CELL_SOLID;
    if (!face && plain0 && plain1) {
        fluid0 = t0 == CELL_FLUID;
        fluid1 = t1 == CELL_FLUID;
        const bool near0 = fluid0 && (fl0 & FLAG_NEAR_SOLID), near1 = fluid1 && (fl1 & FLAG_NEAR_SOLID);
        if (near0 || near1) {
            uint32_t m0 = cm.m0, m1 = cm.m1;
            if constexpr (!CW) {
                const uint2 mm = __ldg(reinterpret_cast<const uint2*>(P.bbmask + idx0));
                m0 = near0 ? mm.x & CW_MASK_BITS : 0u;
                m1 = near1 ? mm.y & CW_MASK_BITS : 0u;
            }
#pragma unroll
            for (int d = 1; d < Q; ++d) {
                const int o = opp(d);
                if ((m0 >> d) & 1u) h[d].x = M::load(P, S.src[o] + idx0, o);
                if ((m1 >> d) & 1u) h[d].y = M::load(P, S.src[o] + idx0 + 1, o);
            }
        }
        return;
    }
    // Two outflow cells whose x - 1 neighbours are plain fluid cells (the
    // common case: the outflow plane of a channel): one pair gather at x - 1,
    // as resolve_state does per cell.  f32 storage only: sphere channel
    // 38.9 -> 39.1 GLUPS (inflow / outflow planes only: 40.1 -> 40.8), while
    // the 16-bit kernels compiled with it ran 2-10 % slower even on lattices
    // without flags.
    if (sizeof(typename M::T) == 4 && !face && t0 == CELL_OUTFLOW && t1 == CELL_OUTFLOW) {
        const int gx = x == 0 ? P.nx - 1 : x - 1;
        const int gidx0 = idx0 + (gx - x) * P.nynz;
        const unsigned short gb = __ldg(reinterpret_cast<const unsigned short*>(P.flags + gidx0));
        int g0 = gb & 0xff, g1 = gb >> 8;
        if ((g0 & 3) == CELL_OUTFLOW) g0 &= ~3;
        if ((g1 & 3) == CELL_OUTFLOW) g1 &= ~3;
        if ((g0 | g1) == 0 && !on_walled_face(P, gx, y, z0) && !on_walled_face(P, gx, y, z0 + 1)) {
            gather_pair<M>(P, S, make_nbr(P, gx, y, z0), z0, zp1, h);
            fluid0 = fluid1 = true;
            return;
        }
    }
    fluid0 = resolve_state<M>(P, S, idx0, x, y, z0, fl0, nb0, Lane<0>{h});
    Nbr nb1 = nb0;
    nb1.Z[0] = z0;
    nb1.Z[1] = z0 + 1;
    nb1.Z[2] = zp1;
    fluid1 = resolve_state<M>(P, S, idx0 + 1, x, y, z0 + 1, fl1, nb1, Lane<1>{h});
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
    constexpr bool CW = LBM_CELL_WORD >= 2 || (LBM_CELL_WORD >= 1 && sizeof(T) == 2);
    int x, y, z0;
    decode_xyz(P, idx0, x, y, z0);
    int fl0 = 0, fl1 = 0;
    PairMasks<CW> cm;
    if (P.has_flags) {
        if constexpr (CW) {
            const uint2 w = __ldg(reinterpret_cast<const uint2*>(P.bbmask + idx0));
            fl0 = (int)(w.x >> CW_FLAG_SHIFT);
            fl1 = (int)(w.y >> CW_FLAG_SHIFT);
            cm.m0 = w.x & CW_MASK_BITS;
            cm.m1 = w.y & CW_MASK_BITS;
        } else {
            const unsigned short both = __ldg(reinterpret_cast<const unsigned short*>(P.flags + idx0));
            fl0 = both & 0xff;
            fl1 = both >> 8;
        }
    }
    const Nbr nb0 = make_nbr(P, x, y, z0);
    const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2; // (z0 + 1) + 1, wrapped
    float2 h[Q];
    gather_pair<M>(P, S, nb0, z0, zp1, h);
    bool fluid0 = true, fluid1 = true;
    const bool face = on_walled_face(P, x, y, z0) || on_walled_face(P, x, y, z0 + 1);
    if ((fl0 | fl1 | (int)face) != 0)
        resolve_pair<M, CW>(P, S, idx0, x, y, z0, fl0, fl1, face, nb0, zp1, h, fluid0, fluid1, cm);
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
        if (live) store_pair<M>(P, S, idx0, d, v, fluid0, fluid1);
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
    for (int d = 0; d < Q; ++d)
        h[d] = M::unshift2(P, d, ld_dev_pair<M::cg>(S.src[d] + nb0.src(d), S.src[d] + nb1.src(d), d));
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
        M::store(P, S.dst[d] + idx0, d, fluid0 ? v.x : M::solid(P, d));
        if (two) M::store(P, S.dst[d] + idx1, d, fluid1 ? v.y : M::solid(P, d));
    });
}

// Launch bounds of k_step2: f32 storage at 3 blocks of 256 per SM (80
// registers); the 16-bit storages at 4 blocks of 128 (128 registers: with the
// storage reference shift the kernel spilled 252 B per thread at 96).  The
// 16-bit storages step with k_step4 where nz is a multiple of 4; k_step2
// serves their readback and sums steps and the other even nz.
template <class T>
struct Step2Bounds {
    static constexpr int threads = 256, blocks = LBM_STEP2_MIN_BLOCKS;
};
template <>
struct Step2Bounds<__half> {
    static constexpr int threads = 128, blocks = 4;
};
template <>
struct Step2Bounds<__nv_bfloat16> {
    static constexpr int threads = 128, blocks = 4;
};

template <class M, int FM, int OUT>
__global__ void __launch_bounds__(Step2Bounds<typename M::T>::threads, Step2Bounds<typename M::T>::blocks)
    k_step2(Params P, Streams<typename M::T> S,
                                                                    Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int idx0 = P.cell0 + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
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
        if (idx0 < P.n && idx0 < P.cell_end)
            step_pair<M, FM, OUT>(P, S, out, P.order ? 2 * __ldg(P.order + (idx0 >> 1)) : idx0, cons);
    }
}

// k_step2 with the FP64 conservation sums over a grid of resident blocks: each
// thread steps pairs p, p + G, p + 2G, ... (G threads in the grid) and adds
// their moments in f64 registers; one block reduction per block and launch
// instead of one per 256 pairs, and no block barrier between pairs.  Every
// thread runs the same number of iterations (threads past the end recompute
// the last pair and store and add nothing), so no branch surrounds a step.
// The per-thread sums follow a fixed order: results are deterministic for a
// given grid.
template <class M, int FM>
__global__ void __launch_bounds__(256, LBM_SUMS_MIN_BLOCKS) k_step2_sums(Params P, Streams<typename M::T> S,
                                                                         Outputs<typename M::C> out)
{
    reduce_prev(out);
    const int np = P.n >> 1;
    const int stride = gridDim.x * blockDim.x;
    const int iters = (np + stride - 1) / stride;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int it = 0; it < iters; ++it, p += stride) {
        const bool live = p < np;
        double cons[5];
        step_pair<M, FM, OUT_SUMS>(P, S, out, live ? 2 * p : P.n - 2, cons, live);
#pragma unroll
        for (int k = 0; k < 5; ++k) acc[k] += cons[k];
    }
    block_sum5(acc, out.partials + (size_t)blockIdx.x * 5);
}

// ---------------------------------------------------------------------------
// Software-pipelined two-cell step for 16-bit storage
// ---------------------------------------------------------------------------

// Raw pulled values of one pair as they come from memory: the c_z = 0
// directions as one aligned 32-bit word (both cells), the z-shifted ones as
// two 16-bit values, and the pair's cell words; kept unconverted so that the
// loads stay in flight while the previous pair is collided.
struct Raw16 {
    uint32_t w[Q];
    unsigned short a[Q], b[Q];
    uint32_t cw0, cw1;  // 0 without flags
};

__device__ __forceinline__ float2 word_dev2(uint32_t w, __half)
{
    __half2 v;
    memcpy(&v, &w, sizeof v);
    return __half22float2(v);
}
__device__ __forceinline__ float2 word_dev2(uint32_t w, __nv_bfloat16)
{
    // bfloat16 is the upper half of a binary32: widening is a shift
    return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
__device__ __forceinline__ float half_dev(unsigned short v, __half) { return __half2float(__ushort_as_half(v)); }
__device__ __forceinline__ float half_dev(unsigned short v, __nv_bfloat16)
{
    return __uint_as_float((uint32_t)v << 16);
}

// Issue the loads of pair idx0 (the plain pull gather of step_pair and the
// pair's cell words); nothing waits for them here.
template <class T>
__device__ __forceinline__ void fetch_pair16(const Params& P, const Streams<T>& S, int idx0, Raw16& r)
{
    int x, y, z0;
    decode_xyz(P, idx0, x, y, z0);
    r.cw0 = r.cw1 = 0u;
    if (P.has_flags) {
        const uint2 cw = __ldg(reinterpret_cast<const uint2*>(P.bbmask + idx0));
        r.cw0 = cw.x;
        r.cw1 = cw.y;
    }
    const Nbr nb0 = make_nbr(P, x, y, z0);
    const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const unsigned short* p =
            reinterpret_cast<const unsigned short*>(S.src[d]) + nb0.X[1 - cx(d)] + nb0.Y[1 - cy(d)];
        if (cz(d) == 0) {
            r.w[d] = __ldg(reinterpret_cast<const unsigned int*>(p + z0));
        } else if (cz(d) == 1) {
            r.a[d] = __ldg(p + nb0.Z[0]);
            r.b[d] = __ldg(p + z0);
        } else {
            r.a[d] = __ldg(p + z0 + 1);
            r.b[d] = __ldg(p + zp1);
        }
    }
}

// The two-cell step of k_step2 (no outputs) over a grid-stride loop of
// pairs, with the next pair's gather issued before this pair's boundary
// rules, collision and stores, so that every warp keeps a pair of loads in
// flight through its arithmetic.  For f16 / bf16 storage
// (LBM_STAGING_PIPELINED), 128 registers, 16 warps per SM: 58.6-59.1 GLUPS
// on the 256x128x128 sphere channel, against 54.4 for an 80-register
// k_step2 and 60.5-60.7 for the 96-register one that is the default.
template <class M, int FM>
__global__ void __launch_bounds__(256, 2) k_step2_pipe(Params P, Streams<typename M::T> S)
{
    using T = typename M::T;
    static_assert(sizeof(T) == 2, "k_step2_pipe: 16-bit storage only");
    const int np = P.n >> 1;
    const int stride = gridDim.x * blockDim.x;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    Raw16 r;
    fetch_pair16(P, S, 2 * p, r);
    for (;;) {
        const int idx0 = 2 * p;
        float2 h[Q];
#pragma unroll
        for (int d = 0; d < Q; ++d)
            h[d] = M::unshift2(P, d, cz(d) == 0 ? word_dev2(r.w[d], T{})
                                               : make_float2(half_dev(r.a[d], T{}), half_dev(r.b[d], T{})));
        const int fl0 = (int)(r.cw0 >> CW_FLAG_SHIFT), fl1 = (int)(r.cw1 >> CW_FLAG_SHIFT);
        PairMasks<true> cm;
        cm.m0 = r.cw0 & CW_MASK_BITS;
        cm.m1 = r.cw1 & CW_MASK_BITS;
        const int q = p + stride;
        if (q < np) fetch_pair16(P, S, 2 * q, r);
        int x, y, z0;
        decode_xyz(P, idx0, x, y, z0);
        bool fluid0 = true, fluid1 = true;
        const bool face = on_walled_face(P, x, y, z0) || on_walled_face(P, x, y, z0 + 1);
        if ((fl0 | fl1 | (int)face) != 0) {
            const Nbr nb0 = make_nbr(P, x, y, z0);
            const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2;
            resolve_pair<M, true>(P, S, idx0, x, y, z0, fl0, fl1, face, nb0, zp1, h, fluid0, fluid1, cm);
        }
        M::template collide2<FM>(P, idx0, h, [&](int d, float2 v) { store_pair<M>(P, S, idx0, d, v, fluid0, fluid1); });
        if (q >= np) break;
        p = q;
    }
}

// ---------------------------------------------------------------------------
// Four-cell step for 16-bit storage
// ---------------------------------------------------------------------------

// Two values of the 16-bit storage format packed in a 32-bit word (low half:
// the lower z), rounded as st_dev2 rounds.
__device__ __forceinline__ uint32_t pack_dev2(float a, float b, __half)
{
    const __half2 v = __floats2half2_rn(a, b);
    uint32_t w;
    memcpy(&w, &v, sizeof w);
    return w;
}
__device__ __forceinline__ uint32_t pack_dev2(float a, float b, __nv_bfloat16)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    uint32_t w;
    memcpy(&w, &v, sizeof w);
    return w;
}

// A quad -- four z-adjacent cells z0..z0 + 3 of one row, z0 a multiple of 4
// -- is plain when its four cells are fluid, none pulls from a solid cell
// and none lies on a walled face: its post-stream state is the raw gather.
// k_step4 also steps the quads of four solid cells (the rest state) and of
// four inflow cells (feq(inflow) in every cell) off the walled faces; the
// other quads are rule quads, listed by kind for k_step4's leading blocks:
//   QUAD_KIND_NEAR     fluid and solid cells only, off the walled faces: one
//                      round of loads (gather, cell words and the pair's own
//                      slots, the half-way bounce-back sources) per pair;
//   QUAD_KIND_OUTFLOW  four outflow cells off the walled faces whose x - 1
//                      neighbours are plain fluid cells: the plain gather at
//                      x - 1 (zero gradient);
//   QUAD_KIND_OTHER    everything else, through the general two-cell step.
constexpr uint32_t QUAD_SOLID = 0x01010101u;   // flag bytes of four solid cells
constexpr uint32_t QUAD_INFLOW = 0x02020202u;
constexpr uint32_t QUAD_OUTFLOW = 0x03030303u;
enum QuadKind : int { QUAD_KIND_NEAR = 0, QUAD_KIND_OUTFLOW = 1, QUAD_KIND_OTHER = 2, QUAD_KINDS = 3 };
__device__ __forceinline__ bool quad_on_walled_face(const Params& P, int x, int y, int z0)
{
    return on_walled_face(P, x, y, z0) || on_walled_face(P, x, y, z0 + 3);
}

// The rule quads of a k_step4 launch: quad lists by kind and the number of
// leading blocks that step them.
struct RuleQuads {
    const int* near_q;
    const int* out_q;
    const int* other_q;
    int n_near, n_out, n_other;
    int blocks;
};

// One rule-quad pair task of k_step4: tasks [0, 2 n_near) take the
// NEAR list, then the OUTFLOW list, then the OTHER list.
template <class M, int FM>
__device__ __forceinline__ void rule_pair(const Params& P, const Streams<typename M::T>& S, const int* near_q,
                                          const int* out_q, const int* other_q, int n_near, int n_out, int n_other,
                                          int k)
{
    using T = typename M::T;
    if (k < 2 * n_near) {
        const int idx0 = 4 * near_q[k >> 1] + 2 * (k & 1);
        if (idx0 < P.cell0 || idx0 >= P.cell_end) return;
        int x, y, z0;
        decode_xyz(P, idx0, x, y, z0);
        const Nbr nb0 = make_nbr(P, x, y, z0);
        const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2;
        float2 h[Q];
        gather_pair<M>(P, S, nb0, z0, zp1, h);
        const uint2 cw = __ldg(reinterpret_cast<const uint2*>(P.bbmask + idx0));
        // the pair's own slots: half-way bounce-back sources, loaded with the gather
        uint32_t own[Q];
#pragma unroll
        for (int d = 1; d < Q; ++d) own[d] = __ldg(reinterpret_cast<const unsigned int*>(S.src[d] + idx0));
        const bool fluid0 = ((cw.x >> CW_FLAG_SHIFT) & 3) == CELL_FLUID;
        const bool fluid1 = ((cw.y >> CW_FLAG_SHIFT) & 3) == CELL_FLUID;
        const uint32_t m0 = fluid0 ? cw.x & CW_MASK_BITS : 0u, m1 = fluid1 ? cw.y & CW_MASK_BITS : 0u;
#pragma unroll
        for (int d = 1; d < Q; ++d) {
            const float2 b = M::unshift2(P, opp(d), word_dev2(own[opp(d)], T{}));
            if ((m0 >> d) & 1u) h[d].x = b.x;
            if ((m1 >> d) & 1u) h[d].y = b.y;
        }
        M::template collide2<FM>(P, idx0, h, [&](int d, float2 v) { store_pair<M>(P, S, idx0, d, v, fluid0, fluid1); });
        return;
    }
    k -= 2 * n_near;
    if (k < 2 * n_out) {
        const int idx0 = 4 * out_q[k >> 1] + 2 * (k & 1);
        if (idx0 < P.cell0 || idx0 >= P.cell_end) return;
        int x, y, z0;
        decode_xyz(P, idx0, x, y, z0);
        const int gx = x == 0 ? P.nx - 1 : x - 1;
        const int zp1 = z0 + 2 == P.nz ? 0 : z0 + 2;
        float2 h[Q];
        gather_pair<M>(P, S, make_nbr(P, gx, y, z0), z0, zp1, h);
        M::template collide2<FM>(P, idx0, h, [&](int d, float2 v) { store_pair<M>(P, S, idx0, d, v, true, true); });
        return;
    }
    k -= 2 * n_out;
    if (k >= 2 * n_other) return;
    const int idx0 = 4 * other_q[k >> 1] + 2 * (k & 1);
    if (idx0 < P.cell0 || idx0 >= P.cell_end) return;
    const Outputs<float> none{nullptr, nullptr, nullptr};
    step_pair<M, FM, OUT_NONE>(P, S, none, idx0, nullptr);
}

// Fused step from POST of the plain quads, four cells per thread, 16-bit
// storage, nz a multiple of 4: the default step kernel of the 16-bit storages
// when no readback or sums are asked for.  Every direction is one aligned
// 8-byte load of the four cells' sources, plus one 2-byte load of the fifth
// value a z-shifted direction needs; the packed collision runs on cells
// (z0, z0 + 1), then (z0 + 2, z0 + 3), and each direction leaves as one
// 8-byte store.  Against the two-cell kernel a thread keeps twice the bytes in
// flight per load phase and issues fewer instructions per cell: 78.6 against
// 66.0 GLUPS (f16) on the 256x128x128 lattice without flags.  The plain quads
// collide their stored values with the storage shift folded into constants
// (ModeFast::collide2s): within the storage's rounding of the two-cell
// kernel, not bit for bit.  The quads that need a rule (3.7 % of the sphere channel's)
// return from the plain path: there they would hold up their whole warp (the
// rule quads sit in 23 % of the channel's rows), and their code would raise
// the register demand of the plain path.  The first `rblocks` blocks of the
// launch step them instead, in a grid-stride loop over their pair tasks
// (rule_pair): the block scheduler starts those blocks first, and they run on
// a few SMs beside the plain blocks for the whole launch.  On the sphere
// channel (23,930 rule quads, f16) 32 such blocks take the launch from 66.5
// (the rule quads as a second kernel on a second stream) to 60.1 us, against
// 58.0 us for the plain quads alone.  The flag bytes of the quad are one
// 4-byte load issued with the gather.
template <class M, int FM>
__global__ void __launch_bounds__(128, 4) k_step4(Params P, Streams<typename M::T> S, RuleQuads rq)
{
    using T = typename M::T;
    static_assert(sizeof(T) == 2, "k_step4: 16-bit storage only");
    if ((int)blockIdx.x < rq.blocks) {
        const int total = 2 * (rq.n_near + rq.n_out + rq.n_other);
#pragma unroll 1
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += rq.blocks * blockDim.x)
            rule_pair<M, FM>(P, S, rq.near_q, rq.out_q, rq.other_q, rq.n_near, rq.n_out, rq.n_other, k);
        return;
    }
    const int idx0 = P.cell0 + 4 * ((blockIdx.x - rq.blocks) * blockDim.x + threadIdx.x);
    if (idx0 >= P.n || idx0 >= P.cell_end) return;
    int x, y, z0;
    decode_xyz(P, idx0, x, y, z0);
    const Nbr nb0 = make_nbr(P, x, y, z0);
    const int zr = z0 + 4 == P.nz ? 0 : z0 + 4;
    uint2 raw[Q];
    uint32_t edge[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const unsigned short* p =
            reinterpret_cast<const unsigned short*>(S.src[d]) + nb0.X[1 - cx(d)] + nb0.Y[1 - cy(d)];
        raw[d] = __ldg(reinterpret_cast<const uint2*>(p + z0));
        edge[d] = cz(d) == 1 ? (uint32_t)__ldg(p + nb0.Z[0]) : (cz(d) == -1 ? (uint32_t)__ldg(p + zr) : 0u);
    }
    const uint32_t fl4 = P.has_flags ? __ldg(reinterpret_cast<const uint32_t*>(P.flags + idx0)) : 0u;
    if (fl4 != 0u || quad_on_walled_face(P, x, y, z0)) {
        if (fl4 != QUAD_SOLID && fl4 != QUAD_INFLOW) return;  // a rule quad: the leading blocks
        if (quad_on_walled_face(P, x, y, z0)) return;
        if (fl4 == QUAD_SOLID) {  // four solid cells: the rest state
#pragma unroll
            for (int d = 0; d < Q; ++d) {
                const float2 sv = M::shift2(P, d, make_float2(0.0f, 0.0f));
                const uint32_t w = pack_dev2(sv.x, sv.y, T{});
                *reinterpret_cast<uint2*>(S.dst[d] + idx0) = make_uint2(w, w);
            }
            return;
        }
    }
    const bool inflow4 = fl4 == QUAD_INFLOW;  // four inflow cells: feq(inflow) in every cell
    uint32_t lo[Q];  // stored words of cells z0, z0 + 1
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        float2 h[Q];
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            uint32_t w;
            if (cz(d) == 0) w = half == 0 ? raw[d].x : raw[d].y;
            else if (cz(d) == 1) w = half == 0 ? (raw[d].x << 16) | edge[d] : __funnelshift_r(raw[d].x, raw[d].y, 16);
            else w = half == 0 ? __funnelshift_r(raw[d].x, raw[d].y, 16) : __funnelshift_r(raw[d].y, edge[d], 16);
            h[d] = inflow4 ? make_float2(P.inflow_s[d], P.inflow_s[d]) : word_dev2(w, T{});
        }
        M::template collide2s<FM>(P, idx0 + 2 * half, h, [&](int d, float2 v) {
            const uint32_t w = pack_dev2(v.x, v.y, T{});
            if (half == 0) lo[d] = w;
            else *reinterpret_cast<uint2*>(S.dst[d] + idx0) = make_uint2(lo[d], w);
        });
    }
}

// The visit order of Params::order for items of `vec` cells (1 or 2): the
// items on the walled faces first (appended through *face_count), then the
// others at their rank in the interior box.
__global__ void k_face_order(Params P, int vec, int* __restrict__ order, int* __restrict__ face_count);

// Lists of the rule quads by kind: quad indices of kind k at lists + k * cap,
// their number in counts[k] (order unspecified; each quad's work is
// independent of the others').
__global__ void k_list_rule_quads(Params P, int* __restrict__ lists, int cap, int* __restrict__ counts);

// ---------------------------------------------------------------------------
// Many steps in one cooperative launch (lattices that fit in L2)
// ---------------------------------------------------------------------------

// Device state of a grid barrier: arrivals of the current round and the
// round number; a timed-out wait raises *err (the lattice's error word).
struct GridBarrier {
    unsigned count;
    unsigned gen;
};

__device__ __forceinline__ unsigned long long global_ns_now()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Barrier over the blocks of a cooperative launch (all co-resident).  Thread
// 0 of a block counts its arrival; the last of `expected` arrivals resets the
// count and opens the next round, the others wait for the round to change --
// for at most timeout_ns, or until another block has raised *err.  Returns
// false (every thread of the block) when the wait gave up; *err is then set.
__device__ __forceinline__ bool grid_sync(GridBarrier* b, int* err, unsigned expected,
                                          unsigned long long timeout_ns)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned* gen = &b->gen;
        volatile int* verr = err;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(&b->count, 1u) == expected - 1u) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            const unsigned long long t0 = global_ns_now();
            while (*gen == g) {
                if (*verr != 0) {
                    ok = 0;
                    break;
                }
                if (global_ns_now() - t0 > timeout_ns) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// `steps` fused steps from POST in one cooperative launch: step s reads
// S[s & 1].src and writes S[s & 1].dst, every block working through the
// cells (pairs with VEC = 2) in a grid-stride loop, with a grid barrier
// between steps.  The per-cell work is that of k_step / k_step2, so the
// results are the same bits; what goes away is a launch and its tail per
// step, which dominates lattices small enough to stay in L2.  A barrier wait
// that runs out (expected arrivals that never come) raises *P.err, and every
// block leaves at its next barrier.
template <class M, int FM, int VEC>
__global__ void __launch_bounds__(256) k_step_persistent(Params P, Streams<typename M::T> S0,
                                                         Streams<typename M::T> S1, int steps, GridBarrier* bar,
                                                         unsigned expected, unsigned long long timeout_ns)
{
    const Outputs<typename M::C> none{nullptr, nullptr, nullptr};
    const int items = VEC == 2 ? P.n / 2 : P.n;
    for (int s = 0; s < steps; ++s) {
        const Streams<typename M::T>& S = (s & 1) ? S1 : S0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < items; i += gridDim.x * blockDim.x) {
            if constexpr (VEC == 2) step_pair<M, FM, OUT_NONE>(P, S, none, 2 * i, nullptr);
            else step_single<M, FM, OUT_NONE>(P, S, none, i, nullptr);
        }
        if (s + 1 < steps && !grid_sync(bar, P.err, expected, timeout_ns)) return;
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
    for (int d = 0; d < Q; ++d) f[d] = M::load(P, S.src[d] + idx, d);
    if (type == CELL_SOLID) {
        emit<M, FM, OUT>(P, out, idx, true, f, cons);
        store_solid<M>(P, S, idx);
    } else {
        emit<M, FM, OUT>(P, out, idx, false, f, cons);
        M::template collide<FM>(P, idx, f);
        store_all<M>(P, S, idx, f);
    }
}

// Step from PRE: S.src holds the buffer base pointers (direction d at S.src[d]).
template <class M, int FM, int OUT>
__global__ void __launch_bounds__(256) k_collide_local(Params P, Streams<typename M::T> S,
                                                       Outputs<typename M::C> out)
{
    if constexpr ((OUT & OUT_SUMS) != 0) reduce_prev(out);
    const int idx = P.cell0 + blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n && idx < P.cell_end) collide_single<M, FM, OUT>(P, S, out, idx, cons);
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
            gather<M>(P, S, nb, f);
            solid = !resolve_state<M>(P, S, idx, x, y, z, fl, nb, f);
            if (solid) {
#pragma unroll
                for (int d = 0; d < Q; ++d) f[d] = M::solid(P, d);
            }
        } else {
            solid = (fl & 3) == CELL_SOLID;
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::load(P, S.src[d] + idx, d);
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
