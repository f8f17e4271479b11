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
//   * the array holds the partial sums of at most LBM_NOALLOC_MAX_CELLS / 128
//     blocks (5.2 MB per GPU), so lattices above LBM_NOALLOC_MAX_CELLS cells
//     are rejected;
//   * it is one array per GPU for the life of the process, shared by every
//     call on that GPU: two calls whose kernels overlap on the GPU (different
//     streams, or different host threads) race on it and both results are
//     undefined -- serialise them;
//   * every call looks up the array's device address (cudaGetSymbolAddress,
//     not a stream operation) with the caller's device current, so the
//     address stays right after cudaDeviceReset reloads the module; the first
//     call on a device loads the module, so make it before any stream capture
//     begins;
//   * the blocks are 128 threads, the default block of a lattice handle, so
//     the sums are bit-identical to lbm_conservation of a default lattice
//     holding f as its uploaded state.
#include <cstdio>
#include <cstring>

#include "lbm_d3q19.h"
#include "lbm_kernels.cuh"
#include "lbm_launch.h"

namespace lbm {
namespace {

constexpr int NOALLOC_BLOCK = 128;
constexpr int NOALLOC_MAX_BLOCKS = (int)(LBM_NOALLOC_MAX_CELLS / NOALLOC_BLOCK);

// Per-block partials (5 doubles each) followed by the 5 final sums.  Every
// call overwrites all entries it reads, so nothing needs clearing.
static __device__ __align__(256) double g_noalloc_scratch[(size_t)NOALLOC_MAX_BLOCKS * 5 + 5];

// Device address of the scratch array on the current device.
cudaError_t scratch_address(double** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = (double*)p;
    return cudaSuccess;
}

// LBM_OK when p is device (or managed) memory of the current device; a host
// pointer handed to the kernels would fault the GPU instead of failing here.
int check_dev(const void* p, const char* what)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    cudaPointerAttributes attr{};
    e = cudaPointerGetAttributes(&attr, p);
    char msg[160];
    if (e != cudaSuccess) {
        cudaGetLastError();
        std::snprintf(msg, sizeof(msg), "lbm_conservation_noalloc: %s is not a CUDA pointer", what);
        return set_error(LBM_ERR_INVALID, msg);
    }
    const bool ok = attr.type == cudaMemoryTypeManaged || (attr.type == cudaMemoryTypeDevice && attr.device == dev);
    if (!ok) {
        std::snprintf(msg, sizeof(msg), "lbm_conservation_noalloc: %s must be device memory of GPU %d", what, dev);
        return set_error(LBM_ERR_INVALID, msg);
    }
    return LBM_OK;
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
    int rc = check_dev(f, "f");
    if (rc == LBM_OK) rc = check_dev(out4, "out4");
    if (rc == LBM_OK && flags) rc = check_dev(flags, "flags");
    if (rc != LBM_OK) return rc;
    double* scratch = nullptr;
    cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) return set_error(LBM_ERR_CUDA, cudaGetErrorString(e));
    Params P;
    std::memset(&P, 0, sizeof(P));
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.n = (int)n;
    P.cell0 = 0;
    P.cell_end = P.n;
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
