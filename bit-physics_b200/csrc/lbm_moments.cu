// lbm_moments.cu -- 16-bit moment-encoded persistent state.
//
// The reference's frontier variant keeps the lattice state between steps as
// 19 moments per cell quantised to 16 bits over fixed ranges
// (packages/lattice-boltzmann-d3q19-frontier-moment-encoded/src/lbm_me.cpp:
// 71-138 basis and inverse, 212-250 range calibration; shaders/
// lbm_encode.comp, lbm_decode.comp):
//   m = M f,  M[k][i] = monomial k of c_i (1, x, y, z, x^2, y^2, z^2, xy, xz,
//             yz, x^2 y, x^2 z, y^2 x, y^2 z, z^2 x, z^2 y, x^2 y^2, x^2 z^2,
//             y^2 z^2; rank 19 on the D3Q19 set)
//   code_k = round((m_k - lo_k) / (hi_k - lo_k) * 65535), clamped to [0, 65535]
//   decode: m_k = lo_k + code_k (hi_k - lo_k) / 65535,  f = M^-1 m
// with [lo_k, hi_k] the envelope of moment k over an f64 run of the same
// trajectory, padded by a margin.  Here the encoded state is the
// post-collision populations P_n that this engine carries between steps,
// stored direction-major as 19 uint16 planes.  A moment-encoded step is
// decode (codes -> f32 populations) + the fused f32 step + encode: the pull
// of one population needs all 19 moments of the neighbour it comes from, so
// the codec cannot sit inside the fused gather without 19x the reads.
#include <cmath>
#include <cstring>
#include <vector>

#include "lbm_d3q19.h"
#include "lbm_handle.h"
#include "lbm_launch.h"

namespace lbm {
namespace {

// Monomial k of velocity (x, y, z), in the order listed above.
__host__ __device__ constexpr int mono(int k, int x, int y, int z)
{
    switch (k) {
    case 0: return 1;
    case 1: return x;
    case 2: return y;
    case 3: return z;
    case 4: return x * x;
    case 5: return y * y;
    case 6: return z * z;
    case 7: return x * y;
    case 8: return x * z;
    case 9: return y * z;
    case 10: return x * x * y;
    case 11: return x * x * z;
    case 12: return y * y * x;
    case 13: return y * y * z;
    case 14: return z * z * x;
    case 15: return z * z * y;
    case 16: return x * x * y * y;
    case 17: return x * x * z * z;
    default: return y * y * z * z;
    }
}
__host__ __device__ constexpr int basis(int k, int i) { return mono(k, cx(i), cy(i), cz(i)); }

struct MomentCodec {
    float minv[Q][Q];  // f_i = sum_k minv[i][k] m_k
    float lo[Q];
    float step[Q];     // (hi - lo) / 65535
    float inv_step[Q]; // 65535 / (hi - lo)
};

// M^-1 by Gauss-Jordan elimination with partial pivoting, in f64.
bool invert_basis(double inv[Q][Q])
{
    double a[Q][Q];
    for (int k = 0; k < Q; ++k)
        for (int i = 0; i < Q; ++i) {
            a[k][i] = basis(k, i);
            inv[k][i] = k == i ? 1.0 : 0.0;
        }
    for (int col = 0; col < Q; ++col) {
        int piv = col;
        for (int r = col + 1; r < Q; ++r)
            if (std::fabs(a[r][col]) > std::fabs(a[piv][col])) piv = r;
        if (std::fabs(a[piv][col]) < 1e-12) return false;
        for (int j = 0; j < Q; ++j) {
            std::swap(a[piv][j], a[col][j]);
            std::swap(inv[piv][j], inv[col][j]);
        }
        const double dinv = 1.0 / a[col][col];
        for (int j = 0; j < Q; ++j) {
            a[col][j] *= dinv;
            inv[col][j] *= dinv;
        }
        for (int r = 0; r < Q; ++r) {
            if (r == col || a[r][col] == 0.0) continue;
            const double m = a[r][col];
            for (int j = 0; j < Q; ++j) {
                a[r][j] -= m * a[col][j];
                inv[r][j] -= m * inv[col][j];
            }
        }
    }
    return true;
}

// The f32 populations of a cell (f32 storage holds f itself).
__device__ __forceinline__ void me_load(const float* __restrict__ f, size_t n, int c, float* v)
{
#pragma unroll
    for (int i = 0; i < Q; ++i) v[i] = f[(size_t)i * n + c];
}

__global__ void k_me_encode(int n, MomentCodec C, const float* __restrict__ f, uint16_t* __restrict__ codes)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float v[Q];
    me_load(f, n, c, v);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        float m = 0.0f;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            if (basis(k, i) == 1) m += v[i];
            else if (basis(k, i) == -1) m -= v[i];
        }
        const float t = rintf((m - C.lo[k]) * C.inv_step[k]);
        codes[(size_t)k * n + c] = (uint16_t)fminf(fmaxf(t, 0.0f), 65535.0f);
    }
}

__global__ void k_me_decode(int n, MomentCodec C, const uint16_t* __restrict__ codes, float* __restrict__ f)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    float m[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) m[k] = fmaf((float)codes[(size_t)k * n + c], C.step[k], C.lo[k]);
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < Q; ++k) s = fmaf(C.minv[i][k], m[k], s);
        f[(size_t)i * n + c] = s;
    }
}

// Per-block min / max of the 19 moments of a post-collision array over the
// non-solid cells (T: double or float populations), out: grid x 38.
template <class T>
__global__ void __launch_bounds__(256) k_me_envelope(int n, const uint8_t* __restrict__ flags, const T* __restrict__ f,
                                                     double* __restrict__ out)
{
    __shared__ double red[8][2 * Q];
    double lo[Q], hi[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        lo[k] = 1e300;
        hi[k] = -1e300;
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        if (flags && (flags[c] & 3) == CELL_SOLID) continue;
        double v[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) v[i] = (double)f[(size_t)i * n + c];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            double m = 0.0;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                if (basis(k, i) == 1) m += v[i];
                else if (basis(k, i) == -1) m -= v[i];
            }
            lo[k] = fmin(lo[k], m);
            hi[k] = fmax(hi[k], m);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmin(lo[k], __shfl_down_sync(0xffffffffu, lo[k], o));
            hi[k] = fmax(hi[k], __shfl_down_sync(0xffffffffu, hi[k], o));
        }
        if (lane == 0) {
            red[warp][k] = lo[k];
            red[warp][Q + k] = hi[k];
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * Q) {
        const int j = threadIdx.x;
        double v = red[0][j];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = j < Q ? fmin(v, red[w][j]) : fmax(v, red[w][j]);
        out[(size_t)blockIdx.x * 2 * Q + j] = v;
    }
}

constexpr int ENV_GRID = 592;

int codec_from_ranges(const double* lo, const double* hi, MomentCodec& C)
{
    static double inv[Q][Q];
    static bool have = false;
    if (!have) {
        if (!invert_basis(inv)) return api::fail(LBM_ERR_CUDA, "moment basis is singular");
        have = true;
    }
    for (int i = 0; i < Q; ++i)
        for (int k = 0; k < Q; ++k) C.minv[i][k] = (float)inv[i][k];
    for (int k = 0; k < Q; ++k) {
        if (!(hi[k] > lo[k]) || !std::isfinite(lo[k]) || !std::isfinite(hi[k]))
            return api::fail(LBM_ERR_INVALID, "moment range %d must satisfy lo < hi (finite)", k);
        C.lo[k] = (float)lo[k];
        C.step[k] = (float)((hi[k] - lo[k]) / 65535.0);
        C.inv_step[k] = (float)(65535.0 / (hi[k] - lo[k]));
    }
    return LBM_OK;
}

}  // namespace
}  // namespace lbm

using namespace lbm;
using namespace lbm::api;

extern "C" {

int lbm_moment16_basis(double* m_out, double* minv_out)
{
    double inv[Q][Q];
    if (!invert_basis(inv)) return fail(LBM_ERR_CUDA, "moment basis is singular");
    for (int k = 0; k < Q; ++k)
        for (int i = 0; i < Q; ++i) {
            if (m_out) m_out[k * Q + i] = basis(k, i);
            if (minv_out) minv_out[k * Q + i] = inv[k][i];
        }
    return LBM_OK;
}

int lbm_moment16_calibrate(lbm_lattice* h, int32_t n_steps, double margin, double* lo, double* hi)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (n_steps < 1 || !lo || !hi || !(margin >= 0.0)) return fail(LBM_ERR_INVALID, "need n_steps >= 1, margin >= 0 and outputs");
    if ((rc = check_force_ready(h))) return rc;
    if (h->storage != LBM_STORAGE_F64 && h->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_UNSUPPORTED, "calibration runs on an f64 or f32 lattice");
    double* part = nullptr;
    CK(cudaMalloc((void**)&part, sizeof(double) * 2 * Q * ENV_GRID), "envelope scratch");
    std::vector<double> host((size_t)2 * Q * ENV_GRID);
    for (int k = 0; k < Q; ++k) {
        lo[k] = 1e300;
        hi[k] = -1e300;
    }
    const uint8_t* flags = h->has_flags ? h->flags : nullptr;
    for (int32_t s = 0; s < n_steps && rc == LBM_OK; ++s) {
        if ((rc = advance(h, nullptr, nullptr, nullptr))) break;
        const int grid = ENV_GRID;
        if (h->storage == LBM_STORAGE_F64)
            k_me_envelope<double><<<grid, 256, 0, h->stream>>>(h->n, flags, (const double*)h->buf[h->cur], part);
        else
            k_me_envelope<float><<<grid, 256, 0, h->stream>>>(h->n, flags, (const float*)h->buf[h->cur], part);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host.data(), part, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "moment envelope");
            break;
        }
        for (int b = 0; b < grid; ++b)
            for (int k = 0; k < Q; ++k) {
                lo[k] = std::fmin(lo[k], host[(size_t)b * 2 * Q + k]);
                hi[k] = std::fmax(hi[k], host[(size_t)b * 2 * Q + Q + k]);
            }
    }
    cudaFree(part);
    if (rc) return rc;
    for (int k = 0; k < Q; ++k) {
        double span = hi[k] - lo[k];
        if (span < 1e-12) span = 1e-12;
        lo[k] -= margin * span;
        hi[k] += margin * span;
    }
    return LBM_OK;
}

int lbm_moment16_step(lbm_lattice* h, const double* lo, const double* hi, int32_t n_steps)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (n_steps < 0 || !lo || !hi) return fail(LBM_ERR_INVALID, "need n_steps >= 0 and ranges");
    if (h->storage != LBM_STORAGE_F32)
        return fail(LBM_ERR_UNSUPPORTED, "the moment-encoded state steps with an f32 lattice's kernels");
    if ((rc = check_force_ready(h))) return rc;
    if (n_steps == 0) return LBM_OK;
    MomentCodec C;
    if ((rc = codec_from_ranges(lo, hi, C))) return rc;
    if (!h->me_codes) CK(cudaMalloc((void**)&h->me_codes, sizeof(uint16_t) * Q * (size_t)h->n), "code allocation");
    const int n = h->n;
    const int grid = grid_for(n, 256);
    int32_t s = 0;
    if (h->pre) {  // the first step collides the set state; its result is encoded
        if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
        ++s;
    }
    k_me_encode<<<grid, 256, 0, h->stream>>>(n, C, (const float*)h->buf[h->cur], h->me_codes);
    CK(cudaGetLastError(), "moment encode");
    for (; s < n_steps; ++s) {
        k_me_decode<<<grid, 256, 0, h->stream>>>(n, C, h->me_codes, (float*)h->buf[h->cur]);
        CK(cudaGetLastError(), "moment decode");
        if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
        k_me_encode<<<grid, 256, 0, h->stream>>>(n, C, (const float*)h->buf[h->cur], h->me_codes);
        CK(cudaGetLastError(), "moment encode");
    }
    // the lattice holds the encoded state, for readback and further steps
    k_me_decode<<<grid, 256, 0, h->stream>>>(n, C, h->me_codes, (float*)h->buf[h->cur]);
    CK(cudaGetLastError(), "moment decode");
    return LBM_OK;
}

}  // extern "C"
