// lbm_device.cuh -- device-side building blocks of the D3Q19 engine.
//
// Lattice: the reference's lex D3Q19 order
//   (packages/lattice-boltzmann-d3q19-stack-e/lattice_boltzmann_d3q19_stack_e/
//    reference/constants.py:27-57, opposite map d3q19_warp.py:61-64).
// Layout in HBM: structure of arrays, direction-major, (19, nx, ny, nz) with z
// contiguous; a cell index is (x*ny + y)*nz + z < 2^31.
//
// Two arithmetic modes share the gather / boundary code:
//   ModeExact      f64 storage; every operation in the reference's order
//                  (d3q19_warp.py:143-195, bgk.py:145-216).  Built with
//                  --fmad=false so the result is bit-identical to the
//                  reference on the same inputs.
//   ModeFast<T>    f32 arithmetic on deviations h_i = f_i - w_i, storage T in
//                  {float (holds f), __half (holds h), __nv_bfloat16 (holds h)}.
#pragma once

#include <cstdint>
#include <type_traits>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace lbm {

constexpr int Q = 19;

enum CellType : int { CELL_FLUID = 0, CELL_SOLID = 1, CELL_INFLOW = 2, CELL_OUTFLOW = 3 };
// Internal flag bit: the cell has a solid cell among its 18 pull sources
// (its bounce-back mask is nonzero).
constexpr int FLAG_NEAR_SOLID = 0x80;
// Per-cell 32-bit cell word (Params::bbmask): bits 1..18 the bounce-back
// mask (bit d: the pull source of direction d is solid), bits 24..31 the
// cell's flag byte (type and FLAG_NEAR_SOLID), so that one load gives a
// step kernel both.
constexpr int CW_FLAG_SHIFT = 24;
constexpr uint32_t CW_MASK_BITS = 0x7fffeu;
enum ForceMode : int { FORCE_NONE = 0, FORCE_UNIFORM = 1, FORCE_FIELD = 2, FORCE_DRAG = 3 };
enum Face : int { FACE_XM = 0, FACE_XP = 1, FACE_YM = 2, FACE_YP = 3, FACE_ZM = 4, FACE_ZP = 5 };

__host__ __device__ constexpr int cx(int d)
{
    return (d == 1 || d == 7 || d == 9 || d == 11 || d == 13) ? 1
         : (d == 2 || d == 8 || d == 10 || d == 12 || d == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int d)
{
    return (d == 3 || d == 7 || d == 10 || d == 15 || d == 17) ? 1
         : (d == 4 || d == 8 || d == 9 || d == 16 || d == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int d)
{
    return (d == 5 || d == 11 || d == 14 || d == 15 || d == 18) ? 1
         : (d == 6 || d == 12 || d == 13 || d == 16 || d == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int d) { return d == 0 ? 0 : ((d & 1) ? d + 1 : d - 1); }
// f32 lattice weights (the f64 ones travel in Params so that they are the
// host-computed values 1.0/3.0, 1.0/18.0, 1.0/36.0).
__host__ __device__ constexpr float wf(int d) { return d == 0 ? (1.0f / 3.0f) : (d < 7 ? (1.0f / 18.0f) : (1.0f / 36.0f)); }

// Division by an invariant divisor with a multiply-high (Granlund & Montgomery
// 1994, "Division by invariant integers using multiplication", round-up
// method): q = (umulhi(n, m) + n) >> l, exact for 0 <= n < 2^31.
struct FastDiv {
    uint32_t d = 1, m = 1, l = 0;
    __host__ void init(uint32_t div)
    {
        d = div;
        l = 0;
        while ((1ull << l) < div) ++l;
        m = (uint32_t)((((1ull << 32) * ((1ull << l) - div)) / div) + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const
    {
#ifdef __CUDA_ARCH__
        uint32_t t = __umulhi(n, m);
#else
        uint32_t t = (uint32_t)(((uint64_t)n * m) >> 32);
#endif
        return (t + n) >> l;
    }
};

// Everything a step kernel needs to know about one lattice; passed by value.
struct Params {
    int nx, ny, nz, n, nynz;
    FastDiv div_nz, div_ny;
    int periodic;      // bit 0 x, 1 y, 2 z
    unsigned walled[3]; // 1 where the axis is not periodic
    int has_flags;
    int wall_sum_pairwise; // nx * nz == 1 (see ModeExact::rho_wall)
    int* err;              // device error word (pipeline wait timeouts), may be null
    const uint8_t* flags;
    const uint32_t* bbmask; // (n) cell words: bounce-back mask | flag byte << CW_FLAG_SHIFT
    const void* force; // (3, n): double for ModeExact, float for ModeFast
    const float* porosity;
    // f64 values (ModeExact), all host-computed with the reference's expressions
    double tau, cs2, inv_cs2, inv_cs4, inv_two_cs4, inv_two_cs2;
    double w[Q];
    double wall_u[6][3];
    double body_force[3];
    double drag_k;
    double inflow_f[Q];
    // f32 values (ModeFast)
    float omega, pref;  // 1/tau, 1 - 0.5/tau
    float wall_uf[6][3];
    float body_force_f[3];
    float drag_kf;
    float inflow_h[Q];  // feq(inflow) - w
    // 16-bit storages: the stored value of direction d is the deviation of f
    // from feq_d(1, storage_ref_u), i.e. (f - w_d) - shift_h[d] in f32; zero
    // for the other storages.
    float shift_h[Q];
    // The same shift folded into the collision of stored values s = h - shift
    // (ModeFast::collide2s; zero for the other storages): its sum and first
    // moments, the relaxation's constant terms -omega shift per direction as
    // the (symmetric, antisymmetric) halves of each opposite pair, and the
    // inflow state as stored values.
    float sh_sum, sh_m[3];
    float sh_c0, sh_csym[Q / 2], sh_casym[Q / 2];
    float inflow_s[Q];
    // Cell window of the step kernels (k_step, k_step2, k_step4 with its rule
    // quads, k_collide_local): they advance the cells [cell0, min(n, cell_end)).
    int cell0 = 0, cell_end = 0x7fffffff;
    // Visit order of the plain steps of k_step (cells) and k_step2 (pairs):
    // item t is order[t], the items on the walled faces first (the slower
    // ones start first), then the others, so that a warp runs one of the
    // two paths (results do not depend on the order).  Null: item t is t.
    // (The persistent kernel deals items to its blocks statically: there
    // the face items gathered into a few blocks would set each step's time,
    // so it keeps them spread.)
    const int* order = nullptr;
};

// Number of cells in the step kernels' window.
__host__ __device__ inline int window_cells(const Params& P) { return (P.cell_end < P.n ? P.cell_end : P.n) - P.cell0; }

// np.maximum(rho, 1e-30): NaN propagates.
__device__ __forceinline__ double rho_safe(double r) { return r != r ? r : (r > 1e-30 ? r : 1e-30); }
__device__ __forceinline__ float rho_safe(float r) { return r != r ? r : (r > 1e-30f ? r : 1e-30f); }

// ---------------------------------------------------------------------------
// Storage loads / stores
// ---------------------------------------------------------------------------
// Loads of population values.  CG = false: the read-only (non-coherent) path,
// for kernels whose source buffer does not change while they run; CG = true:
// cached in L2 only (coherent), for the persistent kernel, whose blocks read
// what other blocks wrote in its previous step.
template <bool CG, class V>
__device__ __forceinline__ V ld_pop(const V* p)
{
    if constexpr (CG) return __ldcg(p);
    else return __ldg(p);
}
template <bool CG = false>
__device__ __forceinline__ float ld_dev(const float* p, int d) { return ld_pop<CG>(p) - wf(d); }
template <bool CG = false>
__device__ __forceinline__ float ld_dev(const __half* p, int) { return __half2float(ld_pop<CG>(p)); }
template <bool CG = false>
__device__ __forceinline__ float ld_dev(const __nv_bfloat16* p, int) { return __bfloat162float(ld_pop<CG>(p)); }
__device__ __forceinline__ void st_dev(float* p, int d, float h) { *p = h + wf(d); }
__device__ __forceinline__ void st_dev(__half* p, int, float h) { *p = __float2half_rn(h); }
__device__ __forceinline__ void st_dev(__nv_bfloat16* p, int, float h) { *p = __float2bfloat16_rn(h); }
// Two consecutive elements (z, z+1) at an 8-byte (f32) / 4-byte (16-bit)
// aligned address, as deviations from the weight.
template <bool CG = false>
__device__ __forceinline__ void ld_dev2(const float* p, int d, float& a, float& b)
{
    const float2 v = ld_pop<CG>(reinterpret_cast<const float2*>(p));
    a = v.x - wf(d);
    b = v.y - wf(d);
}
template <bool CG = false>
__device__ __forceinline__ void ld_dev2(const __half* p, int, float& a, float& b)
{
    const float2 v = __half22float2(ld_pop<CG>(reinterpret_cast<const __half2*>(p)));
    a = v.x;
    b = v.y;
}
template <bool CG = false>
__device__ __forceinline__ void ld_dev2(const __nv_bfloat16* p, int, float& a, float& b)
{
    const float2 v = __bfloat1622float2(ld_pop<CG>(reinterpret_cast<const __nv_bfloat162*>(p)));
    a = v.x;
    b = v.y;
}
__device__ __forceinline__ void st_dev2(float* p, int d, float a, float b)
{
    *reinterpret_cast<float2*>(p) = make_float2(a + wf(d), b + wf(d));
}
__device__ __forceinline__ void st_dev2(__half* p, int, float a, float b)
{
    *reinterpret_cast<__half2*>(p) = __floats2half2_rn(a, b);
}
__device__ __forceinline__ void st_dev2(__nv_bfloat16* p, int, float a, float b)
{
    *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(a, b);
}
// Shared-memory reads of staged populations, as deviations.
__device__ __forceinline__ float ld_dev_sm(const float* p, int d) { return *p - wf(d); }
__device__ __forceinline__ float ld_dev_sm(const __half* p, int) { return __half2float(*p); }
__device__ __forceinline__ float ld_dev_sm(const __nv_bfloat16* p, int) { return __bfloat162float(*p); }
__device__ __forceinline__ float2 ld_dev2_sm(const float* p, int d)
{
    const float2 v = *reinterpret_cast<const float2*>(p);
    return make_float2(v.x - wf(d), v.y - wf(d));
}
__device__ __forceinline__ float2 ld_dev2_sm(const __half* p, int)
{
    return __half22float2(*reinterpret_cast<const __half2*>(p));
}
__device__ __forceinline__ float2 ld_dev2_sm(const __nv_bfloat16* p, int)
{
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}

// Packed two-lane f32 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2): lane x is
// cell z, lane y cell z + 1.  Every operation is correctly rounded per lane.
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, bc2(-1.0f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Two scalar population values (cells z, z + 1 of one direction, stored at
// unrelated addresses) as deviations.
template <bool CG = false, class T>
__device__ __forceinline__ float2 ld_dev_pair(const T* pa, const T* pb, int d)
{
    return make_float2(ld_dev<CG>(pa, d), ld_dev<CG>(pb, d));
}

// f64 value -> storage, rounding as the oracle's store_round does.
__device__ __forceinline__ void st_f64(double* p, int, double v, const Params&) { *p = v; }
__device__ __forceinline__ void st_f64(float* p, int, double v, const Params&) { *p = (float)v; }
__device__ __forceinline__ void st_f64(__half* p, int d, double v, const Params& P)
{
    *p = __float2half_rn((float)(v - P.w[d]) - P.shift_h[d]);
}
__device__ __forceinline__ void st_f64(__nv_bfloat16* p, int d, double v, const Params& P)
{
    *p = __float2bfloat16_rn((float)(v - P.w[d]) - P.shift_h[d]);
}
// storage -> f64 value
__device__ __forceinline__ double ld_f64(const double* p, int, const Params&) { return *p; }
__device__ __forceinline__ double ld_f64(const float* p, int, const Params&) { return (double)*p; }
__device__ __forceinline__ double ld_f64(const __half* p, int d, const Params& P)
{
    return P.w[d] + (double)(__half2float(*p) + P.shift_h[d]);
}
__device__ __forceinline__ double ld_f64(const __nv_bfloat16* p, int d, const Params& P)
{
    return P.w[d] + (double)(__bfloat162float(*p) + P.shift_h[d]);
}

// ---------------------------------------------------------------------------
// Force at a cell (given the post-stream momentum for the drag model)
// ---------------------------------------------------------------------------
template <int FM>
__device__ __forceinline__ void force_exact(const Params& P, int cell, double mx, double my, double mz,
                                            double& Fx, double& Fy, double& Fz)
{
    if (FM == FORCE_UNIFORM) {
        Fx = P.body_force[0]; Fy = P.body_force[1]; Fz = P.body_force[2];
    } else if (FM == FORCE_FIELD) {
        const double* F = (const double*)P.force;
        Fx = F[cell]; Fy = F[P.n + cell]; Fz = F[2 * P.n + cell];
    } else if (FM == FORCE_DRAG) {
        double ka = P.drag_k * (double)P.porosity[cell];
        double beta = ka / (1.0 + 0.5 * ka);
        Fx = P.body_force[0] - beta * mx;
        Fy = P.body_force[1] - beta * my;
        Fz = P.body_force[2] - beta * mz;
    } else {
        Fx = Fy = Fz = 0.0;
    }
}

template <int FM>
__device__ __forceinline__ void force_fast(const Params& P, int cell, float mx, float my, float mz,
                                           float& Fx, float& Fy, float& Fz)
{
    if (FM == FORCE_UNIFORM) {
        Fx = P.body_force_f[0]; Fy = P.body_force_f[1]; Fz = P.body_force_f[2];
    } else if (FM == FORCE_FIELD) {
        const float* F = (const float*)P.force;
        Fx = __ldg(F + cell); Fy = __ldg(F + P.n + cell); Fz = __ldg(F + 2 * P.n + cell);
    } else if (FM == FORCE_DRAG) {
        float ka = P.drag_kf * __ldg(P.porosity + cell);
        float beta = __fdividef(ka, 1.0f + 0.5f * ka);
        Fx = P.body_force_f[0] - beta * mx;
        Fy = P.body_force_f[1] - beta * my;
        Fz = P.body_force_f[2] - beta * mz;
    } else {
        Fx = Fy = Fz = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// ModeExact: f64, reference operation order
// ---------------------------------------------------------------------------
template <bool CG = false>
struct ModeExactT {
    using T = double;
    using C = double;
    static constexpr bool cg = CG;

    static __device__ __forceinline__ C load(const Params&, const T* p, int) { return ld_pop<CG>(p); }
    static __device__ __forceinline__ void store(const Params&, T* p, int, C v) { *p = v; }
    static __device__ __forceinline__ C solid(const Params& P, int d) { return P.w[d]; }
    static __device__ __forceinline__ C inflow(const Params& P, int d) { return P.inflow_f[d]; }
    static __device__ __forceinline__ double to_f64(const Params&, int, C v) { return v; }

    // sum_d f[d] of the raw (pre-bounce) gather, bgk.py:203 / :212.  NumPy
    // reduces a wall row in lex order, except when the row is a single cell
    // (nx * nz == 1): then it runs its 8-accumulator pairwise summation.
    template <class F>
    static __device__ __forceinline__ C rho_wall(const Params& P, const F& f)
    {
        if (!P.wall_sum_pairwise) {
            double r = 0.0;
#pragma unroll
            for (int d = 0; d < Q; ++d) r = r + f[d];
            return r;
        }
        double a[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = f[j] + f[8 + j];
        double r = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
#pragma unroll
        for (int d = 16; d < Q; ++d) r = r + f[d];
        return r;
    }
    // -2 w_i rho_w (c_i . u_w) / c_s^2 in the order of bgk.py:200-205.
    static __device__ __forceinline__ C inject(const Params& P, int face, int d, C rho_w)
    {
        const double* uw = P.wall_u[face];
        double ci_dot_uw = (double)cx(d) * uw[0] + (double)cy(d) * uw[1] + (double)cz(d) * uw[2];
        return -2.0 * P.w[d] * rho_w * ci_dot_uw / P.cs2;
    }

    // _k_collide_guo (d3q19_warp.py:156-195); FORCE_NONE follows the NumPy
    // force-free path of bgk.py:72-85 (no Guo term, u = m / rho_safe).
    template <int FM>
    static __device__ __forceinline__ void collide(const Params& P, int cell, C* f)
    {
        double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            double fd = f[d];
            r = r + fd;
            mx = mx + (double)cx(d) * fd;
            my = my + (double)cy(d) * fd;
            mz = mz + (double)cz(d) * fd;
        }
        double rs = rho_safe(r);
        double Fx, Fy, Fz;
        force_exact<FM>(P, cell, mx, my, mz, Fx, Fy, Fz);
        double ux, uy, uz;
        if (FM == FORCE_NONE) {
            ux = mx / rs; uy = my / rs; uz = mz / rs;
        } else {
            ux = mx / rs + 0.5 * Fx / rs;
            uy = my / rs + 0.5 * Fy / rs;
            uz = mz / rs + 0.5 * Fz / rs;
        }
        double u_sq = ux * ux + uy * uy + uz * uz;
        double pref = 1.0 - 0.5 / P.tau;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            double cd0 = (double)cx(d), cd1 = (double)cy(d), cd2 = (double)cz(d);
            double cu = cd0 * ux + cd1 * uy + cd2 * uz;
            double feq = P.w[d] * r * (1.0 + cu * P.inv_cs2 + cu * cu * P.inv_two_cs4 - u_sq * P.inv_two_cs2);
            double fd = f[d];
            double relaxed = fd - (fd - feq) / P.tau;
            if (FM == FORCE_NONE) {
                f[d] = relaxed;
            } else {
                double tx = (cd0 - ux) * P.inv_cs2 + cu * cd0 * P.inv_cs4;
                double ty = (cd1 - uy) * P.inv_cs2 + cu * cd1 * P.inv_cs4;
                double tz = (cd2 - uz) * P.inv_cs2 + cu * cd2 * P.inv_cs4;
                double force_i = pref * P.w[d] * (tx * Fx + ty * Fy + tz * Fz);
                f[d] = relaxed + force_i;
            }
        }
    }

    // density_field + macroscopic_velocity of one cell (d3q19_warp.py:111-140, :371-383).
    template <int FM>
    static __device__ __forceinline__ void readback(const Params& P, int cell, const C* f, C& rho, C* u)
    {
        double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            double fd = f[d];
            r = r + fd;
            mx = mx + (double)cx(d) * fd;
            my = my + (double)cy(d) * fd;
            mz = mz + (double)cz(d) * fd;
        }
        double rs = rho_safe(r);
        rho = r;
        if (FM == FORCE_NONE) {
            u[0] = mx / rs; u[1] = my / rs; u[2] = mz / rs;
        } else {
            double Fx, Fy, Fz;
            force_exact<FM>(P, cell, mx, my, mz, Fx, Fy, Fz);
            u[0] = (mx + 0.5 * Fx) / rs;
            u[1] = (my + 0.5 * Fy) / rs;
            u[2] = (mz + 0.5 * Fz) / rs;
        }
    }

    // Mass contribution for the FP64 conservation sums.
    static __device__ __forceinline__ void cons_terms(const C* f, double& mass, double& mx, double& my, double& mz)
    {
        double r = 0.0, a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            r = r + f[d];
            a = a + (double)cx(d) * f[d];
            b = b + (double)cy(d) * f[d];
            c = c + (double)cz(d) * f[d];
        }
        mass = r; mx = a; my = b; mz = c;
    }
    static constexpr bool mass_is_deviation = false;
};
using ModeExact = ModeExactT<false>;

// ---------------------------------------------------------------------------
// ModeFast<T>: f32 arithmetic on deviations h = f - w
// ---------------------------------------------------------------------------
template <class TT, bool CG = false>
struct ModeFast {
    using T = TT;
    using C = float;
    static constexpr bool cg = CG;

    // Storage <-> deviation h = f - w: f32 storage holds f itself; the 16-bit
    // storages hold h - shift_h[d] (the deviation from feq(1, storage_ref_u)).
    static __device__ __forceinline__ C load(const Params& P, const T* p, int d)
    {
        if constexpr (sizeof(TT) == 2) return ld_dev<CG>(p, d) + P.shift_h[d];
        else return ld_dev<CG>(p, d);
    }
    static __device__ __forceinline__ void store(const Params& P, T* p, int d, C h)
    {
        if constexpr (sizeof(TT) == 2) st_dev(p, d, h - P.shift_h[d]);
        else st_dev(p, d, h);
    }
    // The same shift for a packed pair (cells z, z + 1) as loaded / to be
    // stored (scalar adds: the shift is a kernel-parameter operand).
    static __device__ __forceinline__ float2 unshift2(const Params& P, int d, float2 v)
    {
        if constexpr (sizeof(TT) == 2) return make_float2(v.x + P.shift_h[d], v.y + P.shift_h[d]);
        else return v;
    }
    static __device__ __forceinline__ float2 shift2(const Params& P, int d, float2 h)
    {
        if constexpr (sizeof(TT) == 2) return make_float2(h.x - P.shift_h[d], h.y - P.shift_h[d]);
        else return h;
    }
    static __device__ __forceinline__ C solid(const Params&, int) { return 0.0f; }
    static __device__ __forceinline__ C inflow(const Params& P, int d) { return P.inflow_h[d]; }
    // The f64 population a stored deviation stands for: f32 storage holds
    // f = h + w in f32; the 16-bit formats hold h, added to the f64 weight.
    static __device__ __forceinline__ double to_f64(const Params& P, int d, C h)
    {
        if constexpr (std::is_same<TT, float>::value) return (double)(h + wf(d));
        else return P.w[d] + (double)h;
    }

    template <class F>
    static __device__ __forceinline__ C rho_wall(const Params&, const F& h)
    {
        float r = 0.0f;
#pragma unroll
        for (int d = 0; d < Q; ++d) r += h[d];
        return 1.0f + r;
    }
    // In deviation form the reflected value keeps its weight (w_opp = w_i).
    static __device__ __forceinline__ C inject(const Params& P, int face, int d, C rho_w)
    {
        const float* uw = P.wall_uf[face];
        float ci_dot_uw = (float)cx(d) * uw[0] + (float)cy(d) * uw[1] + (float)cz(d) * uw[2];
        return (-2.0f * 3.0f) * wf(d) * rho_w * ci_dot_uw;
    }

    // BGK + Guo in deviation form, opposite directions paired:
    //   feq_i - w_i = w_i (rho_dev + rho (3 cu + 4.5 cu^2 - 1.5 u^2))
    //   S_i = (1 - omega/2) w_i (3 (c_i - u).F + 9 (c_i.u)(c_i.F))
    template <int FM>
    static __device__ __forceinline__ void collide(const Params& P, int cell, C* h)
    {
        float rd = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            rd += h[d];
            if (cx(d) == 1) mx += h[d]; else if (cx(d) == -1) mx -= h[d];
            if (cy(d) == 1) my += h[d]; else if (cy(d) == -1) my -= h[d];
            if (cz(d) == 1) mz += h[d]; else if (cz(d) == -1) mz -= h[d];
        }
        float rho = 1.0f + rd;
        float inv = __fdividef(1.0f, rho_safe(rho));
        float Fx, Fy, Fz;
        force_fast<FM>(P, cell, mx, my, mz, Fx, Fy, Fz);
        float ux, uy, uz;
        if (FM == FORCE_NONE) {
            ux = mx * inv; uy = my * inv; uz = mz * inv;
        } else {
            ux = (mx + 0.5f * Fx) * inv; uy = (my + 0.5f * Fy) * inv; uz = (mz + 0.5f * Fz) * inv;
        }
        const float om = P.omega;
        const float usq15 = 1.5f * (ux * ux + uy * uy + uz * uz);
        const float base = rd - rho * usq15; // rho_dev + rho(-1.5 u^2)
        float uF3 = 0.0f, pref = 0.0f;
        if (FM != FORCE_NONE) { uF3 = 3.0f * (ux * Fx + uy * Fy + uz * Fz); pref = P.pref; }
        // rest direction
        h[0] += om * (wf(0) * base - h[0]) - (FM != FORCE_NONE ? pref * wf(0) * uF3 : 0.0f);
#pragma unroll
        for (int d = 1; d < Q; d += 2) {
            const int o = d + 1;
            const float cu = (float)cx(d) * ux + (float)cy(d) * uy + (float)cz(d) * uz;
            const float w = wf(d);
            const float sym = w * (base + rho * 4.5f * cu * cu);
            const float asym = w * rho * 3.0f * cu;
            float hd = h[d] + om * (sym + asym - h[d]);
            float ho = h[o] + om * (sym - asym - h[o]);
            if (FM != FORCE_NONE) {
                const float cF = (float)cx(d) * Fx + (float)cy(d) * Fy + (float)cz(d) * Fz;
                const float s_sym = pref * w * (9.0f * cu * cF - uF3);
                const float s_asym = pref * w * 3.0f * cF;
                hd += s_sym + s_asym;
                ho += s_sym - s_asym;
            }
            h[d] = hd;
            h[o] = ho;
        }
    }

    // The same collision for two cells at once (lanes of float2), in packed
    // f32x2 arithmetic; force fields / porosity are read as (cell, cell + 1)
    // pairs, so cell0 must be even.  Opposite directions are paired through
    // p_d = h_d - h_opp(d) for the momentum sums.  sink(d, value) receives
    // each direction's post-collision pair as soon as it is final; the
    // pre-collision moments are returned (the FP64 monitor sums use them).
    // Pre-collision moments of the two cells: density deviation and momentum.
    struct Moments2 {
        float2 rd, mx, my, mz;
    };

    template <int FM, class Sink>
    static __device__ __forceinline__ Moments2 collide2(const Params& P, int cell0, float2* h, Sink&& sink)
    {
        float2 rd = h[0];
#pragma unroll
        for (int d = 1; d < Q; ++d) rd = add2(rd, h[d]);
        const float2 p1 = sub2(h[1], h[2]), p3 = sub2(h[3], h[4]), p5 = sub2(h[5], h[6]);
        const float2 p7 = sub2(h[7], h[8]), p9 = sub2(h[9], h[10]), p11 = sub2(h[11], h[12]);
        const float2 p13 = sub2(h[13], h[14]), p15 = sub2(h[15], h[16]), p17 = sub2(h[17], h[18]);
        const float2 mx = add2(add2(add2(p1, p7), add2(p9, p11)), p13);
        const float2 my = add2(add2(sub2(add2(p3, p7), p9), p15), p17);
        const float2 mz = sub2(add2(sub2(add2(p5, p11), p13), p15), p17);
        const float2 rho = add2(rd, bc2(1.0f));
        const float2 inv = make_float2(__fdividef(1.0f, rho_safe(rho.x)), __fdividef(1.0f, rho_safe(rho.y)));
        float2 Fx = bc2(0.0f), Fy = bc2(0.0f), Fz = bc2(0.0f);
        if constexpr (FM == FORCE_UNIFORM) {
            Fx = bc2(P.body_force_f[0]); Fy = bc2(P.body_force_f[1]); Fz = bc2(P.body_force_f[2]);
        } else if constexpr (FM == FORCE_FIELD) {
            const float* F = (const float*)P.force;
            Fx = __ldg(reinterpret_cast<const float2*>(F + cell0));
            Fy = __ldg(reinterpret_cast<const float2*>(F + P.n + cell0));
            Fz = __ldg(reinterpret_cast<const float2*>(F + 2 * P.n + cell0));
        } else if constexpr (FM == FORCE_DRAG) {
            const float2 a = __ldg(reinterpret_cast<const float2*>(P.porosity + cell0));
            const float2 ka = mul2(bc2(P.drag_kf), a);
            const float2 den = fma2(bc2(0.5f), ka, bc2(1.0f));
            const float2 nbeta = make_float2(-__fdividef(ka.x, den.x), -__fdividef(ka.y, den.y));
            Fx = fma2(nbeta, mx, bc2(P.body_force_f[0]));
            Fy = fma2(nbeta, my, bc2(P.body_force_f[1]));
            Fz = fma2(nbeta, mz, bc2(P.body_force_f[2]));
        }
        float2 ux, uy, uz;
        if constexpr (FM == FORCE_NONE) {
            ux = mul2(mx, inv); uy = mul2(my, inv); uz = mul2(mz, inv);
        } else {
            ux = mul2(fma2(bc2(0.5f), Fx, mx), inv);
            uy = mul2(fma2(bc2(0.5f), Fy, my), inv);
            uz = mul2(fma2(bc2(0.5f), Fz, mz), inv);
        }
        const float2 usq = fma2(uz, uz, fma2(uy, uy, mul2(ux, ux)));
        const float2 base = fma2(rho, mul2(usq, bc2(-1.5f)), rd);  // rho_dev - 1.5 rho u^2
        const float om = P.omega;
        const float2 keep = bc2(1.0f - om);
        const float2 rho45 = mul2(rho, bc2(4.5f));
        const float2 asym18 = mul2(rho, bc2(3.0f * om * wf(1)));
        const float2 asym36 = mul2(rho, bc2(3.0f * om * wf(7)));
        float2 nuF3 = bc2(0.0f);
        if constexpr (FM != FORCE_NONE) nuF3 = mul2(bc2(-3.0f), fma2(uz, Fz, fma2(uy, Fy, mul2(ux, Fx))));
        // rest direction
        h[0] = fma2(keep, h[0], mul2(bc2(om * wf(0)), base));
        if constexpr (FM != FORCE_NONE) h[0] = fma2(bc2(P.pref * wf(0)), nuF3, h[0]);
        sink(0, h[0]);
#pragma unroll
        for (int d = 1; d < Q; d += 2) {
            float2 cu, cF;
            switch (d) {
            case 1: cu = ux; cF = Fx; break;
            case 3: cu = uy; cF = Fy; break;
            case 5: cu = uz; cF = Fz; break;
            case 7: cu = add2(ux, uy); cF = add2(Fx, Fy); break;
            case 9: cu = sub2(ux, uy); cF = sub2(Fx, Fy); break;
            case 11: cu = add2(ux, uz); cF = add2(Fx, Fz); break;
            case 13: cu = sub2(ux, uz); cF = sub2(Fx, Fz); break;
            case 15: cu = add2(uy, uz); cF = add2(Fy, Fz); break;
            default: cu = sub2(uy, uz); cF = sub2(Fy, Fz); break;
            }
            const float w = wf(d);
            const float2 s1 = fma2(mul2(rho45, cu), cu, base);       // rho_dev + rho(4.5 cu^2 - 1.5 u^2)
            float2 sym = mul2(bc2(om * w), s1);
            float2 asym = mul2(d < 7 ? asym18 : asym36, cu);          // om 3 w rho cu
            if constexpr (FM != FORCE_NONE) {
                const float pw = P.pref * w;
                sym = fma2(bc2(pw), fma2(mul2(bc2(9.0f), cu), cF, nuF3), sym);  // + pref w (9 cu cF - 3 u.F)
                asym = fma2(bc2(3.0f * pw), cF, asym);                            // + pref w 3 c.F
            }
            h[d] = fma2(keep, h[d], add2(sym, asym));
            h[d + 1] = fma2(keep, h[d + 1], sub2(sym, asym));
            sink(d, h[d]);
            sink(d + 1, h[d + 1]);
        }
        return {rd, mx, my, mz};
    }

    // collide2 on the stored values of a 16-bit storage (s = h - shift_h,
    // as loaded; sink receives the post-collision stored values): the shift
    // enters through constants instead of an add per value on the way in and
    // out, since h_new - shift = (1 - omega) s + sym +- asym - omega shift.
    // The same collision as collide2 in exact arithmetic; the f32 roundings
    // differ (both far below the 16-bit rounding of the stored result).
    template <int FM, class Sink>
    static __device__ __forceinline__ void collide2s(const Params& P, int cell0, float2* s, Sink&& sink)
    {
        float2 rs = s[0];
#pragma unroll
        for (int d = 1; d < Q; ++d) rs = add2(rs, s[d]);
        const float2 rd = add2(rs, bc2(P.sh_sum));
        const float2 p1 = sub2(s[1], s[2]), p3 = sub2(s[3], s[4]), p5 = sub2(s[5], s[6]);
        const float2 p7 = sub2(s[7], s[8]), p9 = sub2(s[9], s[10]), p11 = sub2(s[11], s[12]);
        const float2 p13 = sub2(s[13], s[14]), p15 = sub2(s[15], s[16]), p17 = sub2(s[17], s[18]);
        const float2 mx = add2(add2(add2(add2(p1, p7), add2(p9, p11)), p13), bc2(P.sh_m[0]));
        const float2 my = add2(add2(add2(sub2(add2(p3, p7), p9), p15), p17), bc2(P.sh_m[1]));
        const float2 mz = add2(sub2(add2(sub2(add2(p5, p11), p13), p15), p17), bc2(P.sh_m[2]));
        const float2 rho = add2(rd, bc2(1.0f));
        const float2 inv = make_float2(__fdividef(1.0f, rho_safe(rho.x)), __fdividef(1.0f, rho_safe(rho.y)));
        float2 Fx = bc2(0.0f), Fy = bc2(0.0f), Fz = bc2(0.0f);
        if constexpr (FM == FORCE_UNIFORM) {
            Fx = bc2(P.body_force_f[0]); Fy = bc2(P.body_force_f[1]); Fz = bc2(P.body_force_f[2]);
        } else if constexpr (FM == FORCE_FIELD) {
            const float* F = (const float*)P.force;
            Fx = __ldg(reinterpret_cast<const float2*>(F + cell0));
            Fy = __ldg(reinterpret_cast<const float2*>(F + P.n + cell0));
            Fz = __ldg(reinterpret_cast<const float2*>(F + 2 * P.n + cell0));
        } else if constexpr (FM == FORCE_DRAG) {
            const float2 a = __ldg(reinterpret_cast<const float2*>(P.porosity + cell0));
            const float2 ka = mul2(bc2(P.drag_kf), a);
            const float2 den = fma2(bc2(0.5f), ka, bc2(1.0f));
            const float2 nbeta = make_float2(-__fdividef(ka.x, den.x), -__fdividef(ka.y, den.y));
            Fx = fma2(nbeta, mx, bc2(P.body_force_f[0]));
            Fy = fma2(nbeta, my, bc2(P.body_force_f[1]));
            Fz = fma2(nbeta, mz, bc2(P.body_force_f[2]));
        }
        float2 ux, uy, uz;
        if constexpr (FM == FORCE_NONE) {
            ux = mul2(mx, inv); uy = mul2(my, inv); uz = mul2(mz, inv);
        } else {
            ux = mul2(fma2(bc2(0.5f), Fx, mx), inv);
            uy = mul2(fma2(bc2(0.5f), Fy, my), inv);
            uz = mul2(fma2(bc2(0.5f), Fz, mz), inv);
        }
        const float2 usq = fma2(uz, uz, fma2(uy, uy, mul2(ux, ux)));
        const float2 base = fma2(rho, mul2(usq, bc2(-1.5f)), rd);  // rho_dev - 1.5 rho u^2
        const float om = P.omega;
        const float2 keep = bc2(1.0f - om);
        const float2 rho45 = mul2(rho, bc2(4.5f));
        const float2 asym18 = mul2(rho, bc2(3.0f * om * wf(1)));
        const float2 asym36 = mul2(rho, bc2(3.0f * om * wf(7)));
        float2 nuF3 = bc2(0.0f);
        if constexpr (FM != FORCE_NONE) nuF3 = mul2(bc2(-3.0f), fma2(uz, Fz, fma2(uy, Fy, mul2(ux, Fx))));
        s[0] = fma2(keep, s[0], fma2(bc2(om * wf(0)), base, bc2(P.sh_c0)));
        if constexpr (FM != FORCE_NONE) s[0] = fma2(bc2(P.pref * wf(0)), nuF3, s[0]);
        sink(0, s[0]);
#pragma unroll
        for (int d = 1; d < Q; d += 2) {
            float2 cu, cF;
            switch (d) {
            case 1: cu = ux; cF = Fx; break;
            case 3: cu = uy; cF = Fy; break;
            case 5: cu = uz; cF = Fz; break;
            case 7: cu = add2(ux, uy); cF = add2(Fx, Fy); break;
            case 9: cu = sub2(ux, uy); cF = sub2(Fx, Fy); break;
            case 11: cu = add2(ux, uz); cF = add2(Fx, Fz); break;
            case 13: cu = sub2(ux, uz); cF = sub2(Fx, Fz); break;
            case 15: cu = add2(uy, uz); cF = add2(Fy, Fz); break;
            default: cu = sub2(uy, uz); cF = sub2(Fy, Fz); break;
            }
            const float w = wf(d);
            const float2 s1 = fma2(mul2(rho45, cu), cu, base);
            float2 sym = fma2(bc2(om * w), s1, bc2(P.sh_csym[d >> 1]));
            float2 asym = fma2(d < 7 ? asym18 : asym36, cu, bc2(P.sh_casym[d >> 1]));
            if constexpr (FM != FORCE_NONE) {
                const float pw = P.pref * w;
                sym = fma2(bc2(pw), fma2(mul2(bc2(9.0f), cu), cF, nuF3), sym);
                asym = fma2(bc2(3.0f * pw), cF, asym);
            }
            s[d] = fma2(keep, s[d], add2(sym, asym));
            s[d + 1] = fma2(keep, s[d + 1], sub2(sym, asym));
            sink(d, s[d]);
            sink(d + 1, s[d + 1]);
        }
    }

    template <int FM>
    static __device__ __forceinline__ void readback(const Params& P, int cell, const C* h, C& rho, C* u)
    {
        float rd = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            rd += h[d];
            if (cx(d) == 1) mx += h[d]; else if (cx(d) == -1) mx -= h[d];
            if (cy(d) == 1) my += h[d]; else if (cy(d) == -1) my -= h[d];
            if (cz(d) == 1) mz += h[d]; else if (cz(d) == -1) mz -= h[d];
        }
        float r = 1.0f + rd;
        float rs = rho_safe(r);
        rho = r;
        if (FM == FORCE_NONE) {
            u[0] = mx / rs; u[1] = my / rs; u[2] = mz / rs;
        } else {
            float Fx, Fy, Fz;
            force_fast<FM>(P, cell, mx, my, mz, Fx, Fy, Fz);
            u[0] = (mx + 0.5f * Fx) / rs;
            u[1] = (my + 0.5f * Fy) / rs;
            u[2] = (mz + 0.5f * Fz) / rs;
        }
    }

    static __device__ __forceinline__ void cons_terms(const C* h, double& mass_dev, double& mx, double& my, double& mz)
    {
        float rd = 0.0f, a = 0.0f, b = 0.0f, c = 0.0f;
#pragma unroll
        for (int d = 0; d < Q; ++d) {
            rd += h[d];
            if (cx(d) == 1) a += h[d]; else if (cx(d) == -1) a -= h[d];
            if (cy(d) == 1) b += h[d]; else if (cy(d) == -1) b -= h[d];
            if (cz(d) == 1) c += h[d]; else if (cz(d) == -1) c -= h[d];
        }
        mass_dev = (double)rd; mx = (double)a; my = (double)b; mz = (double)c;
    }
    static constexpr bool mass_is_deviation = true;
};

// ---------------------------------------------------------------------------
// Gather (pull streaming) and boundary rules
// ---------------------------------------------------------------------------

// Per-direction base pointers of the source and destination population
// buffers (kernel parameter; one multiply-add per access).
template <class T>
struct Streams {
    const T* src[Q];
    T* dst[Q];
};

// Index of the pull source x - c_d with periodic wrap (d3q19_warp.py:209-211),
// from the wrapped neighbour coordinates precomputed per cell.
struct Nbr {
    int X[3], Y[3], Z[3]; // [0]: coordinate - 1, [1]: coordinate, [2]: coordinate + 1 (scaled)
    __device__ __forceinline__ int src(int d) const { return X[1 - cx(d)] + Y[1 - cy(d)] + Z[1 - cz(d)]; }
    __device__ __forceinline__ int dst(int d) const { return X[1 + cx(d)] + Y[1 + cy(d)] + Z[1 + cz(d)]; }
};

__device__ __forceinline__ Nbr make_nbr(const Params& P, int gx, int y, int z)
{
    Nbr b;
    int xm = gx == 0 ? P.nx - 1 : gx - 1, xp = gx == P.nx - 1 ? 0 : gx + 1;
    int ym = y == 0 ? P.ny - 1 : y - 1, yp = y == P.ny - 1 ? 0 : y + 1;
    int zm = z == 0 ? P.nz - 1 : z - 1, zp = z == P.nz - 1 ? 0 : z + 1;
    b.X[0] = xm * P.nynz; b.X[1] = gx * P.nynz; b.X[2] = xp * P.nynz;
    b.Y[0] = ym * P.nz; b.Y[1] = y * P.nz; b.Y[2] = yp * P.nz;
    b.Z[0] = zm; b.Z[1] = z; b.Z[2] = zp;
    return b;
}

__device__ __forceinline__ void decode_xyz(const Params& P, int idx, int& x, int& y, int& z)
{
    const uint32_t xy = P.div_nz.div((uint32_t)idx);
    z = idx - (int)xy * P.nz;
    const uint32_t xx = P.div_ny.div(xy);
    y = (int)xy - (int)xx * P.ny;
    x = (int)xx;
}

// Branch-free: the cell lies on a face of a walled (non-periodic) axis.
__device__ __forceinline__ bool on_walled_face(const Params& P, int gx, int y, int z)
{
    const unsigned ex = (unsigned)(gx == 0) | (unsigned)(gx == P.nx - 1);
    const unsigned ey = (unsigned)(y == 0) | (unsigned)(y == P.ny - 1);
    const unsigned ez = (unsigned)(z == 0) | (unsigned)(z == P.nz - 1);
    return ((ex & P.walled[0]) | (ey & P.walled[1]) | (ez & P.walled[2])) != 0u;
}

// Walled face crossed by the pull source of direction d, or -1.  Priority when
// several are crossed (edges / corners): y+, y-, x-, x+, z-, z+.
__device__ __forceinline__ int crossed_face(const Params& P, int d, int gx, int y, int z)
{
    const bool wx = !(P.periodic & 1), wy = !(P.periodic & 2), wz = !(P.periodic & 4);
    if (wy && cy(d) == -1 && y == P.ny - 1) return FACE_YP;
    if (wy && cy(d) == 1 && y == 0) return FACE_YM;
    if (wx && cx(d) == 1 && gx == 0) return FACE_XM;
    if (wx && cx(d) == -1 && gx == P.nx - 1) return FACE_XP;
    if (wz && cz(d) == 1 && z == 0) return FACE_ZM;
    if (wz && cz(d) == -1 && z == P.nz - 1) return FACE_ZP;
    return -1;
}

// One lane (cell) of an array of float2 pairs, indexable like a float array;
// lets the scalar boundary code work in place on two-cell state.
template <int L>
struct Lane {
    float2* h;
    __device__ __forceinline__ float& operator[](int d) const { return L ? h[d].y : h[d].x; }
};

// Raw pull of all 19 directions at the position described by nb.
template <class M, class F>
__device__ __forceinline__ void gather(const Params& P, const Streams<typename M::T>& S, const Nbr& nb, F&& f)
{
#pragma unroll
    for (int d = 0; d < Q; ++d) f[d] = M::load(P, S.src[d] + nb.src(d), d);
}

// Replace the pulled values that a boundary rule overrides; every rule sees
// the raw gather as the reference does (bgk.py:190-216 reads its input f and
// writes a copy).
//   walled face crossed:  f[d] = raw[opp(d)] + injection(face, rho_w)
//   solid source (mask):  f[d] = P[opp(d)] at the cell (half-way bounce-back)
// A face rule reads only the raw value of the opposite direction, so each
// opposite pair (d, opp(d)) is resolved from its two raw values held in
// registers (both taken before either is replaced: at an edge or corner both
// members of a pair can cross a face).  The bounce-back values are loads of
// the cell's own slots; their directions cross no face.
template <class M, class F>
__device__ __forceinline__ void boundary_fix(const Params& P, const Streams<typename M::T>& S, const Nbr& nb,
                                             int gx, int y, int z, int gidx, bool face_cell, uint32_t bbmask,
                                             F&& f)
{
    using C = typename M::C;
    if (face_cell) {
        const C rho_w = M::rho_wall(P, f);
#pragma unroll
        for (int d = 1; d < Q; d += 2) {
            const int o = d + 1;
            const int fd = crossed_face(P, d, gx, y, z), fo = crossed_face(P, o, gx, y, z);
            const C rd = f[d], ro = f[o];
            if (fd >= 0) f[d] = ro + M::inject(P, fd, d, rho_w);
            if (fo >= 0) f[o] = rd + M::inject(P, fo, o, rho_w);
            if (fd >= 0) bbmask &= ~(1u << d);
            if (fo >= 0) bbmask &= ~(1u << o);
        }
    }
    if (bbmask) {
#pragma unroll
        for (int d = 1; d < Q; ++d) {
            const int o = opp(d);
            if ((bbmask >> d) & 1u) f[d] = M::load(P, S.src[o] + gidx, o);
        }
    }
}

// Turn the speculative own-position gather f[] into the post-stream
// (pre-collision) state of cell idx.  Returns false for a solid cell.
//   inflow cell:   feq(inflow_rho, inflow_u)
//   outflow cell:  the state of cell (x-1, y, z) (an outflow neighbour is
//                  treated as fluid)
//   fluid cell:    boundary_fix where it sits on a walled face or pulls from
//                  a solid cell
template <class M, class F>
__device__ __forceinline__ bool resolve_state(const Params& P, const Streams<typename M::T>& S, int idx, int x,
                                              int y, int z, int fl, const Nbr& nb, F&& f)
{
    const bool face = on_walled_face(P, x, y, z);
    if ((fl | (int)face) == 0) return true;
    const int type = fl & 3;
    if (type == CELL_SOLID) return false;
    if (type == CELL_INFLOW) {
#pragma unroll
        for (int d = 0; d < Q; ++d) f[d] = M::inflow(P, d);
        return true;
    }
    if (type == CELL_OUTFLOW) {
        const int gx = x == 0 ? P.nx - 1 : x - 1;
        const int gidx = idx + (gx - x) * P.nynz;
        int g = (int)P.flags[gidx];
        if ((g & 3) == CELL_OUTFLOW) g &= ~3;
        if ((g & 3) == CELL_INFLOW) {
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::inflow(P, d);
            return true;
        }
        if ((g & 3) == CELL_SOLID) {
#pragma unroll
            for (int d = 0; d < Q; ++d) f[d] = M::solid(P, d);
            return true;
        }
        const Nbr nb2 = make_nbr(P, gx, y, z);
        gather<M>(P, S, nb2, f);
        const bool face2 = on_walled_face(P, gx, y, z);
        const uint32_t m = (g & FLAG_NEAR_SOLID) ? P.bbmask[gidx] & CW_MASK_BITS : 0u;
        if (face2 || m) boundary_fix<M>(P, S, nb2, gx, y, z, gidx, face2, m, f);
        return true;
    }
    const uint32_t m = (fl & FLAG_NEAR_SOLID) ? P.bbmask[idx] & CW_MASK_BITS : 0u;
    boundary_fix<M>(P, S, nb, x, y, z, idx, face, m, f);
    return true;
}

}  // namespace lbm
