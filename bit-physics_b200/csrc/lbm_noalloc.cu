// lbm_noalloc.cu -- FP64 conservation sums over caller-owned device memory
// with no device allocation of any kind.
//
// lbm_conservation() reduces through per-block partial sums that live in
// scratch memory the lattice handle allocated at creation.  Some callers
// cannot allocate device memory at the point where they want these sums:
// code running inside another framework whose caching allocator already
// holds the device's memory (a fresh cudaMalloc can fail there, or force
// that allocator to release its cache), and monitoring code in a
// latency-critical step loop, where cudaMalloc / cudaFree may synchronise the
// whole device and stall the pipeline.  For them, this entry point keeps its
// scratch in a fixed file-scope device array instead.
//
// Limits and sharing:
//   * the array holds the partial sums of at most LBM_NOALLOC_MAX_CELLS / 256
//     blocks, so lattices above LBM_NOALLOC_MAX_CELLS cells are rejected;
//   * it is one array per GPU for the life of the process, shared by every
//     call on that GPU: two calls whose kernels overlap on the GPU (different
//     streams, or different host threads) race on it and both results are
//     undefined -- serialise them;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "lbm_d3q19.h"
#include "lbm_kernels.cuh"
#include "lbm_launch.h"

namespace lbm {
namespace {

constexpr int NOALLOC_BLOCK = 256;
constexpr int NOALLOC_MAX_BLOCKS = (int)(LBM_NOALLOC_MAX_CELLS / NOALLOC_BLOCK);

// Per-block partials (5 doubles each) followed by the 5 final sums.  Every
// call overwrites all entries it reads, so nothing needs clearing.
static __device__ __align__(256) double g_noalloc_scratch[(size_t)NOALLOC_MAX_BLOCKS * 5 + 5];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
double* g_scratch_addr[MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(double** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = (double*)p;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// The 5 final sums -> the caller's 4 outputs {sum rho, sum m_x, sum m_y, sum m_z}.
__global__ void k_noalloc_publish(const double* __restrict__ sums5, double* __restrict__ out4)
{
    if (threadIdx.x < 4) out4[threadIdx.x] = sums5[threadIdx.x];
}

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" int lbm_conservation_noalloc(const double* f, const uint8_t* flags, int32_t nx, int32_t ny, int32_t nz,
                                        double* out4, void* stream)
{
    if (!f || !out4) return set_error(LBM_ERR_INVALID, "lbm_conservation_noalloc: null population or output pointer");
    if (nx < 1 || ny < 1 || nz < 1) return set_error(LBM_ERR_INVALID, "lbm_conservation_noalloc: dimensions must be >= 1");
    const long long n = (long long)nx * ny * nz;
    if (n > LBM_NOALLOC_MAX_CELLS) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "lbm_conservation_noalloc: %lld cells exceed the fixed scratch limit of %lld cells "
                      "(use lbm_conservation on a lattice handle instead)",
                      n, (long long)LBM_NOALLOC_MAX_CELLS);
        return set_error(LBM_ERR_INVALID, msg);
    }
    double* scratch = nullptr;
    cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    Params P;
    std::memset(&P, 0, sizeof(P));
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.n = (int)n;
    P.nynz = ny * nz;
    P.div_nz.init((uint32_t)nz);
    P.div_ny.init((uint32_t)ny);
    P.periodic = 7;
    P.has_flags = flags ? 1 : 0;
    P.flags = flags;
    const int grid = grid_for(n, NOALLOC_BLOCK);
    double* partials = scratch;
    double* sums5 = scratch + (size_t)NOALLOC_MAX_BLOCKS * 5;
    cudaStream_t s = (cudaStream_t)stream;
    Outputs<double> out{nullptr, nullptr, partials};
    k_observe<ModeExact, FORCE_NONE>
        <<<grid, NOALLOC_BLOCK, 0, s>>>(P, make_streams<double>(f, nullptr, P.n), false, nullptr, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    if ((e = launch_reduce_partials(partials, grid, sums5, s)) != cudaSuccess)
        return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    k_noalloc_publish<<<1, 32, 0, s>>>(sums5, out4);
    if ((e = cudaGetLastError()) != cudaSuccess) return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    return LBM_OK;
}
