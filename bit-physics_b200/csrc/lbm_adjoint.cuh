// lbm_adjoint.cuh -- discrete adjoint of the engine's step, for the gradient
// of a loss on the final readback (rho_N, u_N) with respect to the per-cell
// porosity alpha (drag model) and the initial populations f_0.
//
// Forward, as the step kernels run it: s_0 = f_0 (a PRE buffer), P_0 = C(f_0),
// and for k >= 1  f_k = B(G(P_{k-1})),  P_k = C(f_k).  G is the pull gather
// g[i](x) = P[i](x - c_i), B the boundary rules at a cell, C the BGK + Guo
// collision with the force F = F_b - beta(alpha) m for the drag model,
// beta = k alpha / (1 + k alpha / 2).  The readback after N steps is rho, u of
// f_N.
//
// Backward, one level k = N .. 0 at a time over the stored post-collision
// states (recomputed from checkpoints by the forward kernels):
//   level N (INIT):  lambda_f_N = d(loss)/d f_N from the seeds dL/drho, dL/du
//   level k (STEP):  lambda_P_k(x)[i] = Lambda_{k+1}(x + c_i)[i]    (G^T)
//                    lambda_f_k(x)    = J_C(f_k(x))^T lambda_P_k(x)
//   both:            Lambda_k(x)      = B_x^T lambda_f_k(x)          (local)
//   level 0 (FINAL): lambda_f_0 = J_C(f_0)^T lambda_P_0, the gradient w.r.t.
//                    the initial populations
// and at every level dL/dalpha(x) += the alpha-derivative of the cell's
// readback (INIT) or collision (STEP, FINAL).
//
// Collision transpose (rho = sum f, m = sum c f, a = 1 - beta / 2,
// u = (a m + F_b / 2) / rho, Phi_i = 1 + 3 c_i.u + 4.5 (c_i.u)^2 - 1.5 u^2,
// w = omega, pref = 1 - w / 2):
//   lambda_f_j = (1 - w) lambda_P_j + s0 + V . c_j
//   A  = w sum_i lP_i w_i Phi_i
//   Bv = sum_i lP_i [ w w_i rho (3 c_i + 9 (c_i.u) c_i - 3 u) + pref w_i (-3 F + 9 (c_i.F) c_i) ]
//   Dv = sum_i lP_i pref w_i (3 (c_i - u) + 9 (c_i.u) c_i)
//   s0 = A - Bv.u / rho,  V = (a / rho) Bv - beta Dv
//   dL/dalpha += beta' (-Bv.m / (2 rho) - Dv.m),  beta' = k / (1 + k alpha / 2)^2
// (the force-free and uniform-force models are the cases beta = 0).
//
// Boundary transpose at a cell x whose gather g(x) builds a state:
//   plain direction j:   Lambda[j] += lambda_f[j]
//   walled face crossed: f[j] = g[opp j] + K_j sum_e g[e] with
//                        K_j = -2 w_j (c_j . u_wall) / c_s^2, so
//                        Lambda[opp j] += lambda_f[j], Lambda[e] += K_j lambda_f[j]
//   solid source:        f[j] = P[opp j](x) (half-way bounce-back).  The raw
//                        gather g[j](x) comes from the solid cell, which never
//                        reads Lambda, so slot j of x holds this bounce term
//                        and the next level's pull at x reads it back from
//                        there (own slot opp d for direction d).  Solid cells
//                        write nothing; their slots stay zero.
//   inflow cell:         its state is a constant: Lambda = 0.
//   outflow cell o:      its state is B_x(g(x)) of x = o - e_x (when x is
//                        fluid or outflow), so Lambda(x) also takes
//                        B_x^T lambda_f(o) (Lambda(o) itself is 0 unless
//                        o + e_x is outflow too).
// Each cell writes only its own 19 slots: no atomics, no races.  Two kernels
// share a level: k_adjoint_plain for the cells no boundary rule touches (the
// bulk, lean) and k_adjoint_special for a list of the others.
#pragma once

#include "lbm_kernels.cuh"

namespace lbm {

enum AdjointLevel : int { ADJ_INIT = 0, ADJ_STEP = 1, ADJ_FINAL = 2 };

// Buffers of one adjoint level (C = the mode's arithmetic type).
template <class C>
struct AdjIO {
    const C* Lin;            // Lambda_{k+1} (STEP, FINAL)
    C* Lout;                 // Lambda_k (INIT, STEP)
    const double* grad_rho;  // INIT seeds: dL/drho (n), dL/du (3, n); either may be null
    const double* grad_u;
    double* dalpha;          // (n) accumulated; null: not wanted
    double* grad_f0;         // FINAL: (19, n) dL/df_0; null: not wanted
};

template <class C>
struct CellMoments {
    C rho, mx, my, mz;
};

// rho and m of a state in the mode's representation (f, or h = f - w).
template <class M>
__device__ __forceinline__ CellMoments<typename M::C> adj_moments(const typename M::C* f)
{
    using C = typename M::C;
    C r = C(0), a = C(0), b = C(0), c = C(0);
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        r += f[d];
        a += C(cx(d)) * f[d];
        b += C(cy(d)) * f[d];
        c += C(cz(d)) * f[d];
    }
    if constexpr (M::mass_is_deviation) r += C(1);
    return {r, a, b, c};
}

template <class M>
__device__ __forceinline__ typename M::C adj_w(const Params& P, int d)
{
    if constexpr (std::is_same<typename M::C, double>::value) return P.w[d];
    else return wf(d);
}

// Drag coefficient beta(alpha) of a cell and its derivative.
template <class C, int FM>
__device__ __forceinline__ void adj_beta(const Params& P, int cell, C& beta, C& dbeta)
{
    if constexpr (FM == FORCE_DRAG) {
        const C k = C(P.drag_k);
        const C ka = k * C(P.porosity[cell]);
        const C den = C(1) + C(0.5) * ka;
        beta = ka / den;
        dbeta = k / (den * den);
    } else {
        beta = C(0);
        dbeta = C(0);
    }
}

// The part of the force that does not depend on the state.
template <class C, int FM>
__device__ __forceinline__ void adj_body_force(const Params& P, int cell, C& Fx, C& Fy, C& Fz)
{
    if constexpr (FM == FORCE_UNIFORM || FM == FORCE_DRAG) {
        Fx = C(P.body_force[0]); Fy = C(P.body_force[1]); Fz = C(P.body_force[2]);
    } else if constexpr (FM == FORCE_FIELD) {
        if constexpr (std::is_same<C, double>::value) {
            const double* F = (const double*)P.force;
            Fx = F[cell]; Fy = F[P.n + cell]; Fz = F[2 * P.n + cell];
        } else {
            const float* F = (const float*)P.force;
            Fx = F[cell]; Fy = F[P.n + cell]; Fz = F[2 * P.n + cell];
        }
    } else {
        Fx = Fy = Fz = C(0);
    }
}

// lam: lambda_P in, lambda_f out, through the collision at a cell whose
// pre-collision state has the moments mo (the transpose needs no more of
// it).  Returns the cell's dL/dalpha term.
template <class M, int FM>
__device__ __forceinline__ double adj_collide(const Params& P, int cell, const CellMoments<typename M::C>& mo,
                                              typename M::C* lam)
{
    using C = typename M::C;
    C beta, dbeta, Fbx, Fby, Fbz;
    adj_beta<C, FM>(P, cell, beta, dbeta);
    adj_body_force<C, FM>(P, cell, Fbx, Fby, Fbz);
    const C rho = mo.rho;
    const C inv = C(1) / rho;
    const C a = C(1) - C(0.5) * beta;
    const C ux = (a * mo.mx + C(0.5) * Fbx) * inv;
    const C uy = (a * mo.my + C(0.5) * Fby) * inv;
    const C uz = (a * mo.mz + C(0.5) * Fbz) * inv;
    const C Fx = Fbx - beta * mo.mx, Fy = Fby - beta * mo.my, Fz = Fbz - beta * mo.mz;
    const C om = C(1) / C(P.tau);
    const C pref = C(1) - C(0.5) * om;
    const C usq = ux * ux + uy * uy + uz * uz;
    C A = C(0), W1 = C(0);
    C bx = C(0), by = C(0), bz = C(0), dx = C(0), dy = C(0), dz = C(0);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const C lw = lam[i] * adj_w<M>(P, i);
        const C cu = C(cx(i)) * ux + C(cy(i)) * uy + C(cz(i)) * uz;
        const C cF = C(cx(i)) * Fx + C(cy(i)) * Fy + C(cz(i)) * Fz;
        A += lw * (C(1) + C(3) * cu + C(4.5) * cu * cu - C(1.5) * usq);
        W1 += lw;
        // coefficients of c_i in Bv and Dv
        const C cd = lw * pref * (C(3) + C(9) * cu);
        const C cb = lw * om * rho * (C(3) + C(9) * cu) + lw * pref * C(9) * cF;
        bx += cb * C(cx(i)); by += cb * C(cy(i)); bz += cb * C(cz(i));
        dx += cd * C(cx(i)); dy += cd * C(cy(i)); dz += cd * C(cz(i));
    }
    A *= om;
    // the parts of Bv and Dv along u and F
    const C ku = C(3) * om * rho * W1, kF = C(3) * pref * W1;
    bx -= ku * ux + kF * Fx; by -= ku * uy + kF * Fy; bz -= ku * uz + kF * Fz;
    dx -= kF * ux; dy -= kF * uy; dz -= kF * uz;
    const C s0 = A - (bx * ux + by * uy + bz * uz) * inv;
    const C ai = a * inv;
    const C vx = ai * bx - beta * dx, vy = ai * by - beta * dy, vz = ai * bz - beta * dz;
    const C keep = C(1) - om;
#pragma unroll
    for (int j = 0; j < Q; ++j) lam[j] = keep * lam[j] + s0 + C(cx(j)) * vx + C(cy(j)) * vy + C(cz(j)) * vz;
    if constexpr (FM == FORCE_DRAG) {
        const C bm = bx * mo.mx + by * mo.my + bz * mo.mz;
        const C dm = dx * mo.mx + dy * mo.my + dz * mo.mz;
        return (double)(dbeta * (-(C(0.5) * inv) * bm - dm));
    } else {
        return 0.0;
    }
}

// lambda_f of the readback at a cell: rho = sum f, u = (a m + F_b / 2) / rho,
// seeds gr = dL/drho, gu = dL/du:  lambda_f_j = gr + (a c_j.gu - gu.u) / rho.
// Returns the cell's dL/dalpha term beta' gu.(-m / (2 rho)).
template <class M, int FM>
__device__ __forceinline__ double adj_seed(const Params& P, int cell, const CellMoments<typename M::C>& mo,
                                           const double* grad_rho, const double* grad_u, typename M::C* lam)
{
    using C = typename M::C;
    C beta, dbeta, Fbx, Fby, Fbz;
    adj_beta<C, FM>(P, cell, beta, dbeta);
    adj_body_force<C, FM>(P, cell, Fbx, Fby, Fbz);
    const C gr = grad_rho ? C(grad_rho[cell]) : C(0);
    C gx = C(0), gy = C(0), gz = C(0);
    if (grad_u) {
        gx = C(grad_u[cell]);
        gy = C(grad_u[(size_t)P.n + cell]);
        gz = C(grad_u[2 * (size_t)P.n + cell]);
    }
    const C inv = C(1) / mo.rho;
    const C a = C(1) - C(0.5) * beta;
    const C ux = (a * mo.mx + C(0.5) * Fbx) * inv;
    const C uy = (a * mo.my + C(0.5) * Fby) * inv;
    const C uz = (a * mo.mz + C(0.5) * Fbz) * inv;
    const C gu_u = gx * ux + gy * uy + gz * uz;
    const C ai = a * inv;
#pragma unroll
    for (int j = 0; j < Q; ++j)
        lam[j] = gr + ai * (C(cx(j)) * gx + C(cy(j)) * gy + C(cz(j)) * gz) - gu_u * inv;
    if constexpr (FM == FORCE_DRAG) return (double)(-dbeta * C(0.5) * inv * (gx * mo.mx + gy * mo.my + gz * mo.mz));
    else return 0.0;
}

// G^T at cell idx: lambda_P[d] = Lambda(x + c_d)[d], except where x bounced
// direction opp(d) off a solid cell (bit opp(d) of its mask, no walled face
// taking priority): then the term sits in x's own slot opp(d).
template <class C>
__device__ __forceinline__ void adj_pull(const Params& P, const C* __restrict__ L, const Nbr& nb, int idx, int x,
                                         int y, int z, uint32_t bb, C* lam)
{
    const bool face = bb != 0u && on_walled_face(P, x, y, z);
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const int j = opp(d);
        bool own = ((bb >> j) & 1u) != 0u;
        if (own && face) own = crossed_face(P, j, x, y, z) < 0;
        lam[d] = own ? L[(size_t)j * P.n + idx] : L[(size_t)d * P.n + nb.dst(d)];
    }
}

// lambda_f of cell c (pre-collision moments mo) at this level; returns its
// dL/dalpha term.
template <class M, int FM, int LEVEL>
__device__ __forceinline__ double cell_lambda(const Params& P, const AdjIO<typename M::C>& io, int c, int x, int y,
                                              int z, const CellMoments<typename M::C>& mo, typename M::C* lam)
{
    if constexpr (LEVEL == ADJ_INIT) {
        return adj_seed<M, FM>(P, c, mo, io.grad_rho, io.grad_u, lam);
    } else {
        const Nbr nb = make_nbr(P, x, y, z);
        const int fl = P.has_flags ? (int)P.flags[c] : 0;
        const uint32_t bb = (fl & FLAG_NEAR_SOLID) ? P.bbmask[c] & CW_MASK_BITS : 0u;
        adj_pull<typename M::C>(P, io.Lin, nb, c, x, y, z, bb, lam);
        return adj_collide<M, FM>(P, c, mo, lam);
    }
}

// B_x^T lf into the cell's own slots of Lout.
template <class M>
__device__ __forceinline__ void adj_boundary_store(const Params& P, int x, int y, int z, int idx, bool face_cell,
                                                   uint32_t bb, const typename M::C* lf,
                                                   typename M::C* __restrict__ Lout)
{
    using C = typename M::C;
    C out[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) out[d] = lf[d];
    if (face_cell) {
        C sumK = C(0);
#pragma unroll
        for (int j = 1; j < Q; ++j) {
            const int face = crossed_face(P, j, x, y, z);
            if (face >= 0) {
                out[j] -= lf[j];
                out[opp(j)] += lf[j];
                const double* uw = P.wall_u[face];
                const C cuw = C(cx(j)) * C(uw[0]) + C(cy(j)) * C(uw[1]) + C(cz(j)) * C(uw[2]);
                sumK += C(-6) * adj_w<M>(P, j) * cuw * lf[j];
            }
        }
#pragma unroll
        for (int d = 0; d < Q; ++d) out[d] += sumK;
    }
    if (bb) {
#pragma unroll
        for (int j = 1; j < Q; ++j)
            if (((bb >> j) & 1u) && (!face_cell || crossed_face(P, j, x, y, z) < 0)) out[j] = lf[j];
    }
#pragma unroll
    for (int d = 0; d < Q; ++d) Lout[(size_t)d * P.n + idx] = out[d];
}

template <class C>
__device__ __forceinline__ void adj_store_zero(C* __restrict__ L, int n, int idx)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) L[(size_t)d * n + idx] = C(0);
}

// Cells of the plain kind: fluid, no solid neighbour, not on a walled face,
// no outflow cell at x + 1.  Their state is the raw gather and their Lambda
// is lambda_f itself.  Every other non-solid cell is special.
__device__ __forceinline__ bool adj_special(const Params& P, int idx, int x, int y, int z, int fl)
{
    if (fl != 0 || on_walled_face(P, x, y, z)) return true;
    if (!P.has_flags) return false;
    const int xo = x == P.nx - 1 ? 0 : x + 1;
    return (P.flags[idx + (xo - x) * P.nynz] & 3) == CELL_OUTFLOW;
}

// List of the special non-solid cells (order unspecified; each cell's work
// is independent of the others').
__global__ void k_list_special(Params P, int* __restrict__ list, int* __restrict__ count);

// One adjoint level (INIT or STEP) over the plain cells.  S.src: the stored
// state P_{k-1}.
template <class M, int FM, int LEVEL>
__global__ void __launch_bounds__(256) k_adjoint_plain(Params P, Streams<typename M::T> S, AdjIO<typename M::C> io)
{
    using C = typename M::C;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.n) return;
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int fl = P.has_flags ? (int)P.flags[idx] : 0;
    if ((fl & 3) == CELL_SOLID || adj_special(P, idx, x, y, z, fl)) return;
    const Nbr nb = make_nbr(P, x, y, z);
    CellMoments<C> mo{C(0), C(0), C(0), C(0)};
#pragma unroll
    for (int d = 0; d < Q; ++d) {
        const C v = M::load(P, S.src[d] + nb.src(d), d);
        mo.rho += v;
        if (cx(d)) mo.mx += C(cx(d)) * v;
        if (cy(d)) mo.my += C(cy(d)) * v;
        if (cz(d)) mo.mz += C(cz(d)) * v;
    }
    if constexpr (M::mass_is_deviation) mo.rho += C(1);
    C lam[Q];
    double da;
    if constexpr (LEVEL == ADJ_INIT) {
        da = adj_seed<M, FM>(P, idx, mo, io.grad_rho, io.grad_u, lam);
    } else {
#pragma unroll
        for (int d = 0; d < Q; ++d) lam[d] = io.Lin[(size_t)d * P.n + nb.dst(d)];
        da = adj_collide<M, FM>(P, idx, mo, lam);
    }
#pragma unroll
    for (int d = 0; d < Q; ++d) io.Lout[(size_t)d * P.n + idx] = lam[d];
    if (FM == FORCE_DRAG && io.dalpha) io.dalpha[idx] += da;
}

// One adjoint level (INIT or STEP) over the listed special cells: boundary
// rules, inflow / outflow, bounce-back slots, and the term of an outflow
// cell at x + 1 whose state is B_x(g(x)).
template <class M, int FM, int LEVEL>
__global__ void __launch_bounds__(128) k_adjoint_special(Params P, Streams<typename M::T> S,
                                                          AdjIO<typename M::C> io, const int* __restrict__ cells,
                                                          int count)
{
    using C = typename M::C;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int idx = cells[k];
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int fl = P.has_flags ? (int)P.flags[idx] : 0;
    const int type = fl & 3;
    const Nbr nb = make_nbr(P, x, y, z);
    C f[Q], lam[Q];
    gather<M>(P, S, nb, f);
    resolve_state<M>(P, S, idx, x, y, z, fl, nb, f);
    const double da = cell_lambda<M, FM, LEVEL>(P, io, idx, x, y, z, adj_moments<M>(f), lam);
    if (FM == FORCE_DRAG && io.dalpha) io.dalpha[idx] += da;
    if (type == CELL_INFLOW) {
        adj_store_zero<C>(io.Lout, P.n, idx);  // constant state
        return;
    }
    const int xo = x == P.nx - 1 ? 0 : x + 1;
    const bool down = P.has_flags && (P.flags[idx + (xo - x) * P.nynz] & 3) == CELL_OUTFLOW;
    if (type == CELL_OUTFLOW && !down) {
        adj_store_zero<C>(io.Lout, P.n, idx);  // its state is the x - 1 cell's
        return;
    }
    const bool face = on_walled_face(P, x, y, z);
    const uint32_t bb = (fl & FLAG_NEAR_SOLID) ? P.bbmask[idx] & CW_MASK_BITS : 0u;
    if (type == CELL_OUTFLOW) {
        // own state came from x - 1; the x + 1 outflow cell copies B_x(g(x))
        gather<M>(P, S, nb, f);
        if (face || bb) boundary_fix<M>(P, S, nb, x, y, z, idx, face, bb, f);
#pragma unroll
        for (int d = 0; d < Q; ++d) lam[d] = C(0);
    }
    if (down) {
        C lo[Q];
        cell_lambda<M, FM, LEVEL>(P, io, idx + (xo - x) * P.nynz, xo, y, z, adj_moments<M>(f), lo);
#pragma unroll
        for (int d = 0; d < Q; ++d) lam[d] += lo[d];
    }
    adj_boundary_store<M>(P, x, y, z, idx, face, bb, lam, io.Lout);
}

// Level 0: lambda_f_0 = J_C(f_0)^T lambda_P_0 at every non-solid cell (the
// first step collides every non-solid cell in place), S.src the PRE buffer.
template <class M, int FM>
__global__ void __launch_bounds__(256) k_adjoint_final(Params P, Streams<typename M::T> S, AdjIO<typename M::C> io)
{
    using C = typename M::C;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.n) return;
    int x, y, z;
    decode_xyz(P, idx, x, y, z);
    const int fl = P.has_flags ? (int)P.flags[idx] : 0;
    if ((fl & 3) == CELL_SOLID) {
        if (io.grad_f0) adj_store_zero<double>(io.grad_f0, P.n, idx);
        return;
    }
    C f[Q], lam[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) f[d] = M::load(P, S.src[d] + idx, d);
    const double da = cell_lambda<M, FM, ADJ_FINAL>(P, io, idx, x, y, z, adj_moments<M>(f), lam);
    if (FM == FORCE_DRAG && io.dalpha) io.dalpha[idx] += da;
    if (io.grad_f0) {
#pragma unroll
        for (int d = 0; d < Q; ++d) io.grad_f0[(size_t)d * P.n + idx] = (double)lam[d];
    }
}

// f32 -> f64 widening copy (readback of the f32-arithmetic storages).
__global__ void k_widen(const float* __restrict__ in, double* __restrict__ out, size_t count);
// flag = 1 when any value lies outside [0, 1] (or is NaN).
__global__ void k_check_unit_interval(const float* __restrict__ a, int n, int* __restrict__ flag);

}  // namespace lbm
