// lbm_kernels.cuh -- kernel templates of the stateful engine.
//
// State machine of a lattice (one storage buffer pair A/B):
//   PRE   buffer holds f_n itself (after set_populations / set_equilibrium).
//   POST  buffer holds P_{n-1} = collide(f_{n-1}); f_n = bounce(stream(P_{n-1}))
//         is rebuilt on the fly by pull_state().
// A step from PRE runs k_collide_local (read f_n in place, write P_n);
// a step from POST runs k_step, the fused pull-stream + boundary + collide
// kernel that reads P_{n-1} and writes P_n.  Either way the state advances
// by exactly one reference step (d3q19_warp.py bgk_step :321-368 followed by
// apply_bounce_back_y_walls :386-415).
#pragma once

#include "lbm_device.cuh"

namespace lbm {

// Optional outputs of a kernel: rho/u readback of the pre-collision state and
// per-block FP64 conservation partials.  Null pointers disable them.
template <class C>
struct Outputs {
    C* rho;          // (n)
    C* u;            // (3, n)
    double* partials; // (gridDim.x, 5): mass, mx, my, mz, fluid-cell count
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
            for (int k = 0; k < 5; ++k) out[blockIdx.x * 5 + k] = v[k];
    }
}

template <class M, int FM>
__device__ __forceinline__ void emit(const Params& P, const Outputs<typename M::C>& out, int idx, bool solid,
                                     const typename M::C* f, double cons[5])
{
    using C = typename M::C;
    if (out.rho) {
        if (solid) {
            out.rho[idx] = C(0);
            out.u[idx] = C(0);
            out.u[P.n + idx] = C(0);
            out.u[2 * P.n + idx] = C(0);
        } else {
            C r, u[3];
            M::template readback<FM>(P, idx, f, r, u);
            out.rho[idx] = r;
            out.u[idx] = u[0];
            out.u[P.n + idx] = u[1];
            out.u[2 * P.n + idx] = u[2];
        }
    }
    if (out.partials && !solid) {
        double m, a, b, c;
        M::cons_terms(f, m, a, b, c);
        cons[0] += m; cons[1] += a; cons[2] += b; cons[3] += c; cons[4] += 1.0;
    }
}

// Fused step from POST: f_n = pull_state(P_{n-1}); optional readback of f_n;
// P_n = collide(f_n) -> dst.  Solid cells store their rest value.
template <class M, int FM>
__global__ void __launch_bounds__(512) k_step(Params P, const typename M::T* __restrict__ src,
                                              typename M::T* __restrict__ dst, Outputs<typename M::C> out)
{
    using C = typename M::C;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n) {
        const Site s = decode_site(P, idx);
        C f[Q];
        if (s.type == CELL_SOLID) {
            emit<M, FM>(P, out, idx, true, f, cons);
#pragma unroll
            for (int d = 0; d < Q; ++d) M::store(dst + (size_t)d * P.n + idx, d, M::solid(P, d));
        } else {
            pull_state<M>(P, src, s, f);
            emit<M, FM>(P, out, idx, false, f, cons);
            M::template collide<FM>(P, idx, f);
#pragma unroll
            for (int d = 0; d < Q; ++d) M::store(dst + (size_t)d * P.n + idx, d, f[d]);
        }
    }
    if (out.partials) block_sum5(cons, out.partials);
}

// Step from PRE: read f_n in place, collide, write P_n.
template <class M, int FM>
__global__ void __launch_bounds__(512) k_collide_local(Params P, const typename M::T* __restrict__ src,
                                                       typename M::T* __restrict__ dst,
                                                       Outputs<typename M::C> out)
{
    using C = typename M::C;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n) {
        const int type = P.has_flags ? (P.flags[idx] & 3) : CELL_FLUID;
        C f[Q];
        if (type == CELL_SOLID) {
            emit<M, FM>(P, out, idx, true, f, cons);
#pragma unroll
            for (int d = 0; d < Q; ++d) M::store(dst + (size_t)d * P.n + idx, d, M::solid(P, d));
        } else {
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::load(src + (size_t)d * P.n + idx, d);
            emit<M, FM>(P, out, idx, false, f, cons);
            M::template collide<FM>(P, idx, f);
#pragma unroll
            for (int d = 0; d < Q; ++d) M::store(dst + (size_t)d * P.n + idx, d, f[d]);
        }
    }
    if (out.partials) block_sum5(cons, out.partials);
}

// Current state without advancing it: f_n (f64, optional; used for POST
// states -- a PRE buffer is read out exactly by k_load_f64), readback and
// conservation partials.  post = true rebuilds f_n from P_{n-1}; false reads
// the PRE buffer in place.
template <class M, int FM>
__global__ void __launch_bounds__(512) k_observe(Params P, const typename M::T* __restrict__ src, bool post,
                                                 double* __restrict__ f_out, Outputs<typename M::C> out)
{
    using C = typename M::C;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double cons[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (idx < P.n) {
        C f[Q];
        bool solid;
        if (post) {
            const Site s = decode_site(P, idx);
            solid = s.type == CELL_SOLID;
            if (solid) {
#pragma unroll
                for (int d = 0; d < Q; ++d) f[d] = M::solid(P, d);
            } else {
                pull_state<M>(P, src, s, f);
            }
        } else {
            solid = P.has_flags && (P.flags[idx] & 3) == CELL_SOLID;
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::load(src + (size_t)d * P.n + idx, d);
        }
        if (f_out) {
#pragma unroll
            for (int d = 0; d < Q; ++d) f_out[(size_t)d * P.n + idx] = M::to_f64(P, d, f[d]);
        }
        emit<M, FM>(P, out, idx, solid, f, cons);
    }
    if (out.partials) block_sum5(cons, out.partials);
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

// Mark fluid / inflow / outflow cells that pull from a solid cell.
__global__ void k_mark_near_solid(Params P, uint8_t* __restrict__ flags);

}  // namespace lbm
