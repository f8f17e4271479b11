// lbm_api.cu -- the C ABI of include/lbm_d3q19.h: lattice handles, state
// transfer, the step loop and the stateless reference functions.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <utility>
#include <string>
#include <vector>


#include "lbm_d3q19.h"
#include "lbm_handle.h"
#include "lbm_launch.h"

using namespace lbm;
using namespace lbm::api;

namespace {
thread_local std::string g_err;
}  // namespace

int lbm::set_error(int code, const char* message)
{
    g_err = message ? message : "";
    return code;
}

namespace lbm {
namespace api {

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(LBM_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(e));
    }
    return fail(LBM_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace api
}  // namespace lbm

namespace {

size_t storage_bytes(int storage)
{
    switch (storage) {
    case LBM_STORAGE_F64: return 8;
    case LBM_STORAGE_F32: return 4;
    case LBM_STORAGE_F16_SHIFT:
    case LBM_STORAGE_BF16_SHIFT: return 2;
    default: return 0;
    }
}

// Host f64 constants with the reference's expressions (constants.py:50-57,
// d3q19_warp.py:51-54).  volatile keeps them runtime IEEE operations.
void fill_constants(Params& P)
{
    volatile double one = 1.0, two = 2.0, three = 3.0, eighteen = 18.0, thirtysix = 36.0;
    P.cs2 = one / three;
    P.inv_cs2 = one / P.cs2;
    P.inv_cs4 = one / (P.cs2 * P.cs2);
    P.inv_two_cs4 = one / (two * P.cs2 * P.cs2);
    P.inv_two_cs2 = one / (two * P.cs2);
    P.w[0] = one / three;
    for (int i = 1; i <= 6; ++i) P.w[i] = one / eighteen;
    for (int i = 7; i < Q; ++i) P.w[i] = one / thirtysix;
}

void init_geometry(Params& P, int nx, int ny, int nz)
{
    std::memset(&P, 0, sizeof(P));
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.n = nx * ny * nz;
    P.cell0 = 0;  // the step kernels' window: every cell
    P.cell_end = P.n;
    P.nynz = ny * nz;
    P.div_nz.init((uint32_t)nz);
    P.div_ny.init((uint32_t)ny);
    P.periodic = 7;
    P.wall_sum_pairwise = (long long)nx * nz == 1;
    fill_constants(P);
    P.tau = 1.0;
}

bool dims_ok(long long nx, long long ny, long long nz)
{
    if (nx < 1 || ny < 1 || nz < 1) return false;
    long long n = nx * ny * nz;
    return n < (1LL << 31) / 1 && n * 1 > 0;
}

}  // namespace


namespace {

void rebuild_params(lbm_lattice* h)
{
    h->params_version += 1;  // any captured step graph is stale now
    Params& P = h->P;
    const lbm_desc& d = h->desc;
    init_geometry(P, d.nx, d.ny, d.nz);
    P.periodic = d.periodic & 7;
    for (int a = 0; a < 3; ++a) P.walled[a] = (P.periodic >> a) & 1 ? 0u : 1u;
    P.has_flags = h->has_flags ? 1 : 0;
    P.flags = h->flags;
    P.bbmask = h->bbmask;
    P.err = h->err;
    P.force = h->force;
    P.porosity = h->poro;
    P.tau = d.tau;
    for (int f = 0; f < 6; ++f)
        for (int a = 0; a < 3; ++a) {
            P.wall_u[f][a] = d.wall_velocity[f][a];
            P.wall_uf[f][a] = (float)d.wall_velocity[f][a];
        }
    for (int a = 0; a < 3; ++a) {
        P.body_force[a] = d.body_force[a];
        P.body_force_f[a] = (float)d.body_force[a];
    }
    P.drag_k = d.drag_k;
    P.drag_kf = (float)d.drag_k;
    // Inflow equilibrium, reciprocal form of equilibrium.py:310-322.
    const double ux = d.inflow_u[0], uy = d.inflow_u[1], uz = d.inflow_u[2];
    const double u_sq = ux * ux + uy * uy + uz * uz;
    for (int q = 0; q < Q; ++q) {
        double cu = (double)cx(q) * ux + (double)cy(q) * uy + (double)cz(q) * uz;
        P.inflow_f[q] = P.w[q] * d.inflow_rho *
                        (1.0 + cu * P.inv_cs2 + cu * cu * P.inv_two_cs4 - u_sq * P.inv_two_cs2);
        P.inflow_h[q] = (float)(P.inflow_f[q] - P.w[q]);
    }
    P.omega = (float)(1.0 / d.tau);
    P.pref = (float)(1.0 - 0.5 / d.tau);
    // 16-bit storage reference: feq(1, storage_ref_u) - w, reciprocal form.
    const bool storage16 = h->storage == LBM_STORAGE_F16_SHIFT || h->storage == LBM_STORAGE_BF16_SHIFT;
    const double rx = d.storage_ref_u[0], ry = d.storage_ref_u[1], rz = d.storage_ref_u[2];
    const double r_sq = rx * rx + ry * ry + rz * rz;
    for (int q = 0; q < Q; ++q) {
        double cu = (double)cx(q) * rx + (double)cy(q) * ry + (double)cz(q) * rz;
        const double feq = P.w[q] * 1.0 * (1.0 + cu * P.inv_cs2 + cu * cu * P.inv_two_cs4 - r_sq * P.inv_two_cs2);
        P.shift_h[q] = storage16 ? (float)(feq - P.w[q]) : 0.0f;
    }
    // The shift's constants of ModeFast::collide2s (f32, as the kernels use them).
    float sum = 0.0f, m[3] = {0.0f, 0.0f, 0.0f};
    for (int q = 0; q < Q; ++q) {
        sum += P.shift_h[q];
        m[0] += (float)cx(q) * P.shift_h[q];
        m[1] += (float)cy(q) * P.shift_h[q];
        m[2] += (float)cz(q) * P.shift_h[q];
        P.inflow_s[q] = P.inflow_h[q] - P.shift_h[q];
    }
    P.sh_sum = sum;
    for (int a = 0; a < 3; ++a) P.sh_m[a] = m[a];
    P.sh_c0 = -P.omega * P.shift_h[0];
    for (int q = 1; q < Q; q += 2) {
        P.sh_csym[q >> 1] = -P.omega * (0.5f * (P.shift_h[q] + P.shift_h[q + 1]));
        P.sh_casym[q >> 1] = -P.omega * (0.5f * (P.shift_h[q] - P.shift_h[q + 1]));
    }
}

}  // namespace

cudaError_t lbm::api::launch(lbm_lattice* h, int kernel, const void* src, void* dst, bool post, double* f_out,
                             void* rho, void* u, double* partials, int* grid_used, const PendingSums* prev)
{
    LaunchArgs a;
    a.P = h->P;
    a.src = src;
    a.dst = dst;
    a.post = post;
    a.f_out = f_out;
    a.rho = rho;
    a.u = u;
    a.partials = partials;
    a.prev_partials = partials && prev ? prev->partials : nullptr;
    a.prev_count = partials && prev ? prev->count : 0;
    a.prev_sums = partials && prev ? prev->sums : nullptr;
    a.first = 0;
    a.count = -1;
    a.block = h->block;
    a.vec = kernel == KERNEL_STEP ? h->vec : 1;
    a.stream = h->stream;
    a.grid_used = grid_used;
    a.tma_grid = 0;
    a.pipe_grid = kernel == KERNEL_STEP ? h->pipe_grid : 0;
    a.sums_grid = kernel == KERNEL_STEP ? h->sums_grid : 0;
    a.rule_quads = h->rule_quads;
    for (int k = 0; k < QUAD_KINDS; ++k) a.rule_counts[k] = h->rule_counts[k];
    a.rules_grid = h->rules_grid;
    if (kernel == KERNEL_STEP && !rho && !u && !partials) a.P.order = h->order;
    if (kernel == KERNEL_STEP && h->use_tma) {
        a.tma_grid = h->tma_grid;
        a.tile = h->tile;
        return launch_tma_step(h->storage, h->desc.force_mode, a);
    }
    if (h->storage == LBM_STORAGE_F64) return launch_exact(kernel, h->desc.force_mode, a);
    return launch_fast(h->storage, kernel, h->desc.force_mode, a);
}

namespace {

// The quads k_step4's plain path leaves to its leading blocks, from the
// current flags and walled faces (four-cell lattices only), and the number
// of those blocks.
int refresh_rule_quads(lbm_lattice* h)
{
    if (h->vec != 4) return LBM_OK;
    const int cap = h->n / 4;
    int* counts = h->rule_quads + (size_t)QUAD_KINDS * cap;
    CK(launch_list_rule_quads(h->P, h->rule_quads, cap, counts, h->stream), "rule quad lists");
    CK(cudaMemcpyAsync(h->rule_counts, counts, sizeof(int) * QUAD_KINDS, cudaMemcpyDeviceToHost, h->stream),
       "rule quad counts");
    CK(cudaStreamSynchronize(h->stream), "rule quad sync");
    // The lists come out in the order of the listing kernel's atomics; in
    // lattice order, the consecutive tasks of a warp step neighbouring quads,
    // whose gathers share cache lines.
    std::vector<int> list;
    for (int k = 0; k < QUAD_KINDS; ++k) {
        if (h->rule_counts[k] < 2) continue;
        int* dev = h->rule_quads + (size_t)k * cap;
        list.resize(h->rule_counts[k]);
        CK(cudaMemcpy(list.data(), dev, sizeof(int) * list.size(), cudaMemcpyDeviceToHost), "rule quad list");
        std::sort(list.begin(), list.end());
        CK(cudaMemcpy(dev, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice), "rule quad list");
    }
    // Leading blocks of k_step4: about 0.7 rule tasks per thread for each
    // wave of resident blocks (4 of 128 threads per SM) the plain quads take,
    // so that the rule blocks finish within the plain ones' time.  Sphere
    // channel (23,930 rule quads, f16): 38 blocks; measured 58.4 / 58.2 /
    // 58.5 us at 32 / 36 / 40, 61.0 at 28, 66.1 at 24, 60.2 at 48.  The same
    // spheres without inflow / outflow (19,834): 32 blocks, 57.5 us.
    const long long total = (long long)h->rule_counts[0] + h->rule_counts[1] + h->rule_counts[2];
    const long long plain = (long long)cap - total > 0 ? (long long)cap - total : 1;
    const long long want = (2 * total * 11 * h->sms + 2 * plain - 1) / (2 * plain);
    h->rules_grid = total > 0 ? (int)(want < 1 ? 1 : (want > 4 * h->sms ? 4 * h->sms : want)) : 0;
    if (h->rules_grid_set > 0) h->rules_grid = h->rules_grid_set;
    h->params_version += 1;  // a captured step graph holds the old count
    return LBM_OK;
}

// Calls that change the state or the parameters wait for an open
// plane-range step to be committed.
int check_no_open_step(const lbm_lattice* h)
{
    if (h->open_step) return fail(LBM_ERR_STATE, "a plane-range step is open (lbm_step_commit ends it)");
    return LBM_OK;
}

int ensure_staging(lbm_lattice* h)
{
    if (h->staging) return LBM_OK;
    CK(cudaMalloc((void**)&h->staging, sizeof(double) * Q * (size_t)h->n), "staging allocation");
    return LBM_OK;
}

}  // namespace

int lbm::api::check_handle(const lbm_lattice* h)
{
    if (!h) return fail(LBM_ERR_INVALID, "null lattice handle");
    CK(cudaSetDevice(h->desc.device), "cudaSetDevice");
    return LBM_OK;
}

// Advance one step; rho/u/partials receive the readback of the state
// before the step (optional); *blocks (optional) the number of partials written.
int lbm::api::advance(lbm_lattice* h, void* rho, void* u, double* partials, int* blocks, const PendingSums* prev)
{
    const void* src = h->buf[h->cur];
    void* dst = h->buf[h->cur ^ 1];
    cudaError_t e = launch(h, h->pre ? KERNEL_COLLIDE_LOCAL : KERNEL_STEP, src, dst, false, nullptr, rho, u, partials,
                           blocks, prev);
    if (e != cudaSuccess) return cuda_fail(e, "step kernel launch");
    h->cur ^= 1;
    h->pre = false;
    h->steps += 1;
    return LBM_OK;
}

namespace {

// Copy a device readback pair (C = double or float) into host f64 arrays.
// The caller's arrays are used as they are: no paging advice or other change
// is applied to memory the library does not own.
int readback_to_host(lbm_lattice* h, const void* drho, const void* du, double* rho, double* u)
{
    const size_t n = (size_t)h->n;
    // f32 values widened to f64 on the device (in the population staging
    // buffer, 19 n doubles) and copied straight into the caller's arrays.
    const bool staged = h->storage != LBM_STORAGE_F64 && (h->staging || ensure_staging(h) == LBM_OK);
    if (h->storage != LBM_STORAGE_F64 && !staged) cudaGetLastError();  // no room: convert on the host below
    if (staged) {
        if (rho) CK(launch_widen((const float*)drho, h->staging, n, h->stream), "rho widen");
        if (u) CK(launch_widen((const float*)du, h->staging + n, 3 * n, h->stream), "u widen");
        if (rho) CK(cudaMemcpyAsync(rho, h->staging, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream), "rho copy");
        if (u) CK(cudaMemcpyAsync(u, h->staging + n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream),
                  "u copy");
        CK(cudaStreamSynchronize(h->stream), "readback sync");
        return LBM_OK;
    }
    if (h->storage == LBM_STORAGE_F64) {
        if (rho) CK(cudaMemcpyAsync(rho, drho, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream), "rho copy");
        if (u) CK(cudaMemcpyAsync(u, du, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, h->stream), "u copy");
        CK(cudaStreamSynchronize(h->stream), "readback sync");
        return LBM_OK;
    }
    std::vector<float> tmp(4 * n);
    CK(cudaMemcpyAsync(tmp.data(), drho, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream), "rho copy");
    CK(cudaMemcpyAsync(tmp.data() + n, du, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, h->stream), "u copy");
    CK(cudaStreamSynchronize(h->stream), "readback sync");
    if (rho)
        for (size_t i = 0; i < n; ++i) rho[i] = (double)tmp[i];
    if (u)
        for (size_t i = 0; i < 3 * n; ++i) u[i] = (double)tmp[n + i];
    return LBM_OK;
}

}  // namespace

int lbm::api::check_device_ptr(const lbm_lattice* h, const void* p, const char* what)
{
    if (!p) return LBM_OK;
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(LBM_ERR_INVALID, "%s is not a CUDA pointer", what);
    }
    const bool dev = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    if (!dev || (attr.type == cudaMemoryTypeDevice && attr.device != h->desc.device))
        return fail(LBM_ERR_INVALID, "%s must be device memory of GPU %d", what, h->desc.device);
    return LBM_OK;
}

int lbm::api::observe_rho_u(lbm_lattice* h, void* drho, void* du)
{
    cudaError_t e = launch(h, KERNEL_OBSERVE, h->buf[h->cur], nullptr, !h->pre, nullptr, drho, du, nullptr);
    if (e != cudaSuccess) return cuda_fail(e, "observe kernel launch");
    return LBM_OK;
}


extern "C" {

int lbm_version(void) { return 10000; }

const char* lbm_last_error(void) { return g_err.c_str(); }

int lbm_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int lbm_desc_init(lbm_desc* d)
{
    if (!d) return fail(LBM_ERR_INVALID, "null descriptor");
    std::memset(d, 0, sizeof(*d));
    d->nx = d->ny = d->nz = 1;
    d->storage = LBM_STORAGE_F64;
    d->periodic = LBM_PERIODIC_X | LBM_PERIODIC_Y | LBM_PERIODIC_Z;
    d->force_mode = LBM_FORCE_NONE;
    d->tau = 1.0;
    d->inflow_rho = 1.0;
    return LBM_OK;
}

int lbm_create(const lbm_desc* desc, lbm_lattice** out)
{
    if (!desc || !out) return fail(LBM_ERR_INVALID, "null argument to lbm_create");
    *out = nullptr;
    if (!dims_ok(desc->nx, desc->ny, desc->nz))
        return fail(LBM_ERR_INVALID, "invalid lattice dimensions %d x %d x %d (need >= 1 and < 2^31 cells)",
                    desc->nx, desc->ny, desc->nz);
    if (storage_bytes(desc->storage) == 0) return fail(LBM_ERR_INVALID, "unknown storage %d", desc->storage);
    if (desc->force_mode < LBM_FORCE_NONE || desc->force_mode > LBM_FORCE_DRAG)
        return fail(LBM_ERR_INVALID, "unknown force mode %d", desc->force_mode);
    if (!(desc->tau > 0.5)) return fail(LBM_ERR_INVALID, "tau must be > 0.5 (got %g)", desc->tau);
    if (desc->periodic < 0 || desc->periodic > 7) return fail(LBM_ERR_INVALID, "periodic mask must be 0..7");
    for (int a = 0; a < 3; ++a)
        if (!(desc->storage_ref_u[a] > -0.5 && desc->storage_ref_u[a] < 0.5))
            return fail(LBM_ERR_INVALID, "storage_ref_u components must lie in (-0.5, 0.5)");
    if (desc->block_size != 0 && (desc->block_size % 32 != 0 || desc->block_size < 32 || desc->block_size > 256))
        return fail(LBM_ERR_INVALID, "block_size must be 0 or a multiple of 32 in [32, 256]");
    if (desc->cells_per_thread < 0 || desc->cells_per_thread > 4 || desc->cells_per_thread == 3)
        return fail(LBM_ERR_INVALID, "cells_per_thread must be 0 (auto), 1, 2 or 4");
    if (desc->staging < LBM_STAGING_AUTO || desc->staging > LBM_STAGING_PERSISTENT)
        return fail(LBM_ERR_INVALID, "staging must be LBM_STAGING_AUTO, _REGISTERS, _TMA, _PIPELINED or _PERSISTENT");
    if (desc->cells_per_thread == 2 && (desc->storage == LBM_STORAGE_F64 || desc->nz % 2 != 0))
        return fail(LBM_ERR_UNSUPPORTED, "cells_per_thread = 2 needs f32/f16/bf16 storage and an even nz");
    const bool storage16 = desc->storage == LBM_STORAGE_F16_SHIFT || desc->storage == LBM_STORAGE_BF16_SHIFT;
    if (desc->cells_per_thread == 4 && (!storage16 || desc->nz % 4 != 0))
        return fail(LBM_ERR_UNSUPPORTED, "cells_per_thread = 4 needs f16/bf16 storage and nz a multiple of 4");
    if (desc->cells_per_thread == 4 && desc->staging != LBM_STAGING_AUTO && desc->staging != LBM_STAGING_REGISTERS)
        return fail(LBM_ERR_UNSUPPORTED, "cells_per_thread = 4 runs with register staging only");
    int ndev = lbm_device_count();
    if (ndev == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device available");
    if (desc->device < 0 || desc->device >= ndev) return fail(LBM_ERR_INVALID, "device %d out of range", desc->device);
    CK(cudaSetDevice(desc->device), "cudaSetDevice");

    lbm_lattice* h = new lbm_lattice();
    h->desc = *desc;
    h->storage = desc->storage;
    h->n = desc->nx * desc->ny * desc->nz;
    h->elem = storage_bytes(desc->storage);
    // 128-thread blocks: on the 256x128x128 sphere channel f32 39.5 against
    // 38.9 GLUPS with 256, f16 (pipelined) 59.1 against 58.4 (192: 38.7 /
    // 52.4), f64 17.1 against 16.5.
    h->block = desc->block_size ? desc->block_size : 128;
    // Two cells per thread (packed f32x2 arithmetic) cuts the instructions
    // per cell; measured on the 256x128x128 sphere channel: f16 41 -> 50
    // GLUPS, f32 unchanged (bandwidth-bound).  Needs an even nz.  The 16-bit
    // storages take four (k_step4) when nz is a multiple of 4 and the staging
    // is the default: 78.6 against 66.0 GLUPS (f16, 256x128x128 without flags).
    if (desc->cells_per_thread)
        h->vec = desc->cells_per_thread;
    else if (storage16 && desc->nz % 4 == 0 && (desc->staging == LBM_STAGING_AUTO || desc->staging == LBM_STAGING_REGISTERS))
        h->vec = 4;
    else
        h->vec = desc->storage != LBM_STORAGE_F64 && desc->nz % 2 == 0 ? 2 : 1;
    auto cleanup = [&](int code) {
        lbm_destroy(h);
        return code;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "stream creation"));
    h->own_stream = true;
    const size_t pop_bytes = h->elem * Q * (size_t)h->n;
    for (int b = 0; b < 2; ++b) {
        e = cudaMalloc(&h->buf[b], pop_bytes);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "population allocation"));
    }
    const size_t cbytes = h->storage == LBM_STORAGE_F64 ? sizeof(double) : sizeof(float);
    e = cudaMalloc(&h->rho, cbytes * (size_t)h->n);
    if (e == cudaSuccess) e = cudaMalloc(&h->u, cbytes * 3 * (size_t)h->n);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "readback allocation"));
    // TMA-staged step (on request): shared-memory pipeline for f32-arithmetic
    // storages whose rows are multiples of 16 bytes.  Not the default: on the
    // 256x128x128 sphere channel it measured 26 / 34 GLUPS (f32 / f16) against
    // 37 / 50 for the register-staged kernels.  Planned before the reduction
    // scratch is sized: its persistent grid writes one partial per block.
    if (desc->staging == LBM_STAGING_TMA) {
        int grid = 0;
        TileCfg G = plan_tma(h->storage, desc->nx, desc->ny, desc->nz, &grid, desc->device);
        if (G.stages >= 2 && grid > 0) {
            h->use_tma = true;
            h->tile = G;
            h->tma_grid = grid;
        }
    }
    // Pipelined two-cell step (on request): on the 256x128x128 sphere channel
    // f16 58.6-59.1 GLUPS against 60.5-60.7 for k_step2 in 128-thread blocks
    // at 96 registers, which is therefore the default.
    const bool pipe_ok = (h->storage == LBM_STORAGE_F16_SHIFT || h->storage == LBM_STORAGE_BF16_SHIFT) && h->vec == 2;
    if (desc->staging == LBM_STAGING_PIPELINED && !pipe_ok)
        return cleanup(fail(LBM_ERR_UNSUPPORTED, "pipelined staging needs f16/bf16 storage, two cells per "
                                                 "thread and an even nz"));
    if (desc->staging == LBM_STAGING_PIPELINED) {
        h->pipe_grid = pipe_grid_fast(h->storage, desc->force_mode, h->block);
        if (h->pipe_grid <= 0) return cleanup(fail(LBM_ERR_CUDA, "pipelined step: no resident blocks"));
    }
    // Steps with FP64 sums (two cells per thread) run one block per resident
    // slot, each thread looping over pairs: one partial row per block.
    if (h->storage != LBM_STORAGE_F64 && h->vec >= 2) {
        h->sums_grid = sums_grid_fast(h->storage, desc->force_mode, h->block);
        if (h->sums_grid <= 0) return cleanup(fail(LBM_ERR_CUDA, "step with sums: no resident blocks"));
    }
    if (desc->staging == LBM_STAGING_TMA && !h->use_tma)
        return cleanup(fail(LBM_ERR_UNSUPPORTED, "TMA staging needs f32/f16/bf16 storage, two cells per thread, "
                                                 "an even nz and nz * element size a multiple of 16 bytes"));
    // Room for the partial rows of any launch: one per block of a per-cell
    // grid, of the TMA grid or of the resident sums grid (which exceeds the
    // per-cell grid on small lattices).
    h->partial_blocks = grid_for(h->n, h->block);
    if (h->partial_blocks < h->tma_grid) h->partial_blocks = h->tma_grid;
    if (h->partial_blocks < h->sums_grid) h->partial_blocks = h->sums_grid;
    e = cudaMalloc((void**)&h->partials, sizeof(double) * 2 * 5 * (size_t)h->partial_blocks);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->sums, sizeof(double) * 5);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->err, 0, sizeof(int));
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "reduction scratch allocation"));
    if (desc->staging == LBM_STAGING_PERSISTENT) {
        int coop = 0;
        if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, desc->device) != cudaSuccess || !coop) {
            cudaGetLastError();
            return cleanup(fail(LBM_ERR_UNSUPPORTED, "persistent staging needs cooperative launch support"));
        }
        e = cudaMalloc((void**)&h->bar, sizeof(GridBarrier));
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "grid barrier allocation"));
        h->persist = true;
    }
    if (h->vec == 4) {
        e = cudaMalloc((void**)&h->rule_quads, sizeof(int) * ((size_t)QUAD_KINDS * (h->n / 4) + QUAD_KINDS));
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "four-cell step set-up"));
        if (cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, desc->device) != cudaSuccess ||
            h->sms < 1)
            h->sms = 1;
    }
    rebuild_params(h);
    if (int rc2 = refresh_rule_quads(h)) return cleanup(rc2);
    // Visit order of the plain one- and two-cell steps on a lattice with
    // walls: the items on the walled faces first, then the interior (fixed
    // by the periodicity, which does not change after creation).
    if (h->vec <= 2 && desc->periodic != 7) {
        const size_t items = (size_t)h->n / h->vec;
        e = cudaMalloc((void**)&h->order, sizeof(int) * (items + 1));
        if (e == cudaSuccess) e = launch_face_order(h->P, h->vec, h->order, h->order + items, h->stream);
        int faces = -1;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&faces, h->order + items, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cleanup(cuda_fail(e, "face order"));
        const long long bx = desc->nx - 2 * (int)h->P.walled[0], by = desc->ny - 2 * (int)h->P.walled[1],
                        bz = desc->nz / h->vec - 2 * (int)h->P.walled[2];
        const long long inner = bx > 0 && by > 0 && bz > 0 ? bx * by * bz : 0;
        if (faces != (long long)items - inner) return cleanup(fail(LBM_ERR_CUDA, "face order incomplete"));
        if (faces > 1) {  // the face items into lattice order
            std::vector<int> list(faces);
            e = cudaMemcpy(list.data(), h->order, sizeof(int) * list.size(), cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) {
                std::sort(list.begin(), list.end());
                e = cudaMemcpy(h->order, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice);
            }
            if (e != cudaSuccess) return cleanup(cuda_fail(e, "face order"));
        }
    }
    // Rest state f = w_i (rho = 1, u = 0).
    e = launch_feq_init(h->storage, h->P, nullptr, nullptr, h->buf[0], h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "initial state"));
    h->cur = 0;
    h->pre = true;
    *out = h;
    return LBM_OK;
}

int lbm_destroy(lbm_lattice* h)
{
    if (!h) return LBM_OK;
    cudaSetDevice(h->desc.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    void* ptrs[] = {h->buf[0], h->buf[1], h->flags, h->bbmask, h->force, h->poro, h->rho,
                    h->u, h->partials, h->sums, h->staging, h->monitor, h->err, h->diag, h->rule_quads, h->bar,
                    h->me_codes, h->order};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LBM_OK;
}

int lbm_set_stream(lbm_lattice* h, void* stream)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    CK(cudaStreamSynchronize(h->stream), "stream sync");
    if (h->own_stream) CK(cudaStreamDestroy(h->stream), "stream destroy");
    h->own_stream = false;
    if (stream) {
        h->stream = (cudaStream_t)stream;
    } else {
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream creation");
        h->own_stream = true;
    }
    return LBM_OK;
}

// Device error word raised by a kernel (a bounded pipeline wait that ran out).
static int check_device_error(lbm_lattice* h)
{
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "error word read");
    CK(cudaStreamSynchronize(h->stream), "stream sync");
    if (flag) {
        cudaMemsetAsync(h->err, 0, sizeof(int), h->stream);
        return fail(LBM_ERR_CUDA, "a step kernel's bounded wait (shared-memory pipeline or grid barrier) timed out; "
                                  "the state is invalid");
    }
    return LBM_OK;
}

int lbm_synchronize(lbm_lattice* h)
{
    int rc = check_handle(h);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream), "stream sync");
    return check_device_error(h);
}

int lbm_set_populations(lbm_lattice* h, const double* f)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!f) return fail(LBM_ERR_INVALID, "null population array");
    const size_t bytes = sizeof(double) * Q * (size_t)h->n;
    if (h->storage == LBM_STORAGE_F64) {
        CK(cudaMemcpyAsync(h->buf[h->cur], f, bytes, cudaMemcpyHostToDevice, h->stream), "population upload");
    } else {
        if ((rc = ensure_staging(h))) return rc;
        CK(cudaMemcpyAsync(h->staging, f, bytes, cudaMemcpyHostToDevice, h->stream), "population upload");
        CK(launch_store_f64(h->storage, h->P, h->staging, h->buf[h->cur], h->stream), "population store");
    }
    CK(cudaStreamSynchronize(h->stream), "population upload sync");
    h->pre = true;
    return LBM_OK;
}

int lbm_get_populations(lbm_lattice* h, double* f)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!f) return fail(LBM_ERR_INVALID, "null population array");
    const size_t bytes = sizeof(double) * Q * (size_t)h->n;
    if (h->pre && h->storage == LBM_STORAGE_F64) {
        CK(cudaMemcpyAsync(f, h->buf[h->cur], bytes, cudaMemcpyDeviceToHost, h->stream), "population download");
    } else {
        if ((rc = ensure_staging(h))) return rc;
        if (h->pre) {
            CK(launch_load_f64(h->storage, h->P, h->buf[h->cur], h->staging, h->stream), "population load");
        } else {
            CK(launch(h, KERNEL_OBSERVE, h->buf[h->cur], nullptr, true, h->staging, nullptr, nullptr, nullptr),
               "population rebuild");
        }
        CK(cudaMemcpyAsync(f, h->staging, bytes, cudaMemcpyDeviceToHost, h->stream), "population download");
    }
    CK(cudaStreamSynchronize(h->stream), "population download sync");
    return LBM_OK;
}

int lbm_set_equilibrium(lbm_lattice* h, const double* rho, const double* u)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    double* drho = nullptr;
    double* du = nullptr;
    const size_t n = (size_t)h->n;
    if (rho || u) {
        if ((rc = ensure_staging(h))) return rc;
        drho = rho ? h->staging : nullptr;
        du = u ? h->staging + n : nullptr;
        if (rho) CK(cudaMemcpyAsync(drho, rho, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream), "rho upload");
        if (u) CK(cudaMemcpyAsync(du, u, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream), "u upload");
    }
    CK(launch_feq_init(h->storage, h->P, drho, du, h->buf[h->cur], h->stream), "equilibrium init");
    CK(cudaStreamSynchronize(h->stream), "equilibrium sync");
    h->pre = true;
    return LBM_OK;
}

int lbm_set_flags(lbm_lattice* h, const uint8_t* flags)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!flags) {
        h->has_flags = false;
        rebuild_params(h);
        return refresh_rule_quads(h);
    }
    const size_t n = (size_t)h->n;
    for (size_t i = 0; i < n; ++i)
        if (flags[i] > LBM_CELL_OUTFLOW)
            return fail(LBM_ERR_INVALID, "flag value %u at cell %zu is not a cell type (0..3)", flags[i], i);
    // A state held as P_{n-1} was built under the old flags; rebuild f_n
    // under them first so that the change applies from the next step on.
    if (!h->pre) {
        if ((rc = ensure_staging(h))) return rc;
        CK(launch(h, KERNEL_OBSERVE, h->buf[h->cur], nullptr, true, h->staging, nullptr, nullptr, nullptr),
           "state rebuild");
    }
    if (!h->flags) CK(cudaMalloc((void**)&h->flags, n), "flag allocation");
    if (!h->bbmask) CK(cudaMalloc((void**)&h->bbmask, sizeof(uint32_t) * n), "mask allocation");
    CK(cudaMemcpyAsync(h->flags, flags, n, cudaMemcpyHostToDevice, h->stream), "flag upload");
    h->has_flags = true;
    rebuild_params(h);
    CK(launch_mark_near_solid(h->P, h->flags, h->bbmask, h->stream), "flag marking");
    if (!h->pre) {
        CK(launch_store_f64(h->storage, h->P, h->staging, h->buf[h->cur], h->stream), "state store");
        h->pre = true;
    }
    CK(cudaStreamSynchronize(h->stream), "flag sync");
    return refresh_rule_quads(h);
}

int lbm_set_force_field(lbm_lattice* h, const double* force)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!force) return fail(LBM_ERR_INVALID, "null force field");
    if (h->desc.force_mode != LBM_FORCE_FIELD)
        return fail(LBM_ERR_STATE, "lattice was not created with LBM_FORCE_FIELD");
    const size_t cnt = 3 * (size_t)h->n;
    if (h->storage == LBM_STORAGE_F64) {
        if (!h->force) CK(cudaMalloc(&h->force, sizeof(double) * cnt), "force allocation");
        CK(cudaMemcpyAsync(h->force, force, sizeof(double) * cnt, cudaMemcpyHostToDevice, h->stream), "force upload");
        CK(cudaStreamSynchronize(h->stream), "force sync");
    } else {
        std::vector<float> tmp(cnt);
        for (size_t i = 0; i < cnt; ++i) tmp[i] = (float)force[i];
        if (!h->force) CK(cudaMalloc(&h->force, sizeof(float) * cnt), "force allocation");
        CK(cudaMemcpyAsync(h->force, tmp.data(), sizeof(float) * cnt, cudaMemcpyHostToDevice, h->stream),
           "force upload");
        CK(cudaStreamSynchronize(h->stream), "force sync");
    }
    rebuild_params(h);
    return LBM_OK;
}

int lbm_set_porosity(lbm_lattice* h, const float* alpha)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!alpha) return fail(LBM_ERR_INVALID, "null porosity field");
    if (h->desc.force_mode != LBM_FORCE_DRAG)
        return fail(LBM_ERR_STATE, "lattice was not created with LBM_FORCE_DRAG");
    const size_t n = (size_t)h->n;
    for (size_t i = 0; i < n; ++i)
        if (!(alpha[i] >= 0.0f && alpha[i] <= 1.0f))
            return fail(LBM_ERR_INVALID, "porosity at cell %zu is outside [0, 1]", i);
    if (!h->poro) CK(cudaMalloc((void**)&h->poro, sizeof(float) * n), "porosity allocation");
    CK(cudaMemcpyAsync(h->poro, alpha, sizeof(float) * n, cudaMemcpyHostToDevice, h->stream), "porosity upload");
    CK(cudaStreamSynchronize(h->stream), "porosity sync");
    rebuild_params(h);
    return LBM_OK;
}

int lbm_set_tau(lbm_lattice* h, double tau)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!(tau > 0.5)) return fail(LBM_ERR_INVALID, "tau must be > 0.5 (got %g)", tau);
    h->desc.tau = tau;
    rebuild_params(h);
    return LBM_OK;
}

int lbm_set_wall_velocity(lbm_lattice* h, int32_t face, const double* u3)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (face < 0 || face > 5 || !u3) return fail(LBM_ERR_INVALID, "bad face index or null velocity");
    for (int a = 0; a < 3; ++a) h->desc.wall_velocity[face][a] = u3[a];
    rebuild_params(h);
    return LBM_OK;
}

int lbm_set_body_force(lbm_lattice* h, const double* f3)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!f3) return fail(LBM_ERR_INVALID, "null body force");
    for (int a = 0; a < 3; ++a) h->desc.body_force[a] = f3[a];
    rebuild_params(h);
    return LBM_OK;
}

}  // extern "C"

int lbm::api::check_force_ready(lbm_lattice* h)
{
    if (h->desc.force_mode == LBM_FORCE_FIELD && !h->force)
        return fail(LBM_ERR_STATE, "LBM_FORCE_FIELD lattice has no force field (lbm_set_force_field)");
    if (h->desc.force_mode == LBM_FORCE_DRAG && !h->poro)
        return fail(LBM_ERR_STATE, "LBM_FORCE_DRAG lattice has no porosity field (lbm_set_porosity)");
    return LBM_OK;
}

extern "C" {

// Capture the two steady-state steps from the current buffer into a graph.
static int capture_step_graph(lbm_lattice* h)
{
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "graph capture begin");
    const int c = h->cur;
    cudaError_t e0 = launch(h, KERNEL_STEP, h->buf[c], h->buf[c ^ 1], false, nullptr, nullptr, nullptr, nullptr);
    cudaError_t e1 = launch(h, KERNEL_STEP, h->buf[c ^ 1], h->buf[c], false, nullptr, nullptr, nullptr, nullptr);
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
    if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(e0 != cudaSuccess ? e0 : (e1 != cudaSuccess ? e1 : e2), "step graph capture");
    }
    cudaError_t e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "step graph instantiate");
    h->graph_cur = c;
    h->graph_version = h->params_version;
    return LBM_OK;
}

int lbm_step(lbm_lattice* h, int32_t n_steps)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (n_steps < 0) return fail(LBM_ERR_INVALID, "negative step count");
    if ((rc = check_force_ready(h))) return rc;
    int32_t s = 0;
    if (h->persist && n_steps >= 2) {
        if (h->pre) {
            if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
            ++s;
        }
        const int32_t k = n_steps - s;
        if (k > 0) {
            LaunchArgs a;
            a.P = h->P;
            a.src = h->buf[h->cur];
            a.dst = h->buf[h->cur ^ 1];
            a.block = 256;
            a.vec = h->vec;
            a.stream = h->stream;
            CK(launch_persistent(h->storage, h->desc.force_mode, a, k, h->bar, h->persist_missing,
                                 h->persist_timeout_ns, nullptr),
               "persistent step launch");
            h->cur ^= (k & 1);
            h->steps += k;
        }
        return LBM_OK;
    }
    // Launch-bound small lattices gain from replaying steady-state steps
    // (two per replay) from a captured CUDA graph.  Any call of three or more
    // steps captures it (a short warm-up call then leaves the capture and
    // instantiation behind it, outside a caller's timed loop).
    if (n_steps >= 3) {
        while (s < n_steps && (h->pre || (h->graph && h->graph_version == h->params_version && h->cur != h->graph_cur))) {
            if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
            ++s;
        }
        if (n_steps - s >= 2) {
            if (!h->graph || h->graph_version != h->params_version || h->cur != h->graph_cur)
                if ((rc = capture_step_graph(h))) return rc;
            for (; s + 1 < n_steps; s += 2) {
                CK(cudaGraphLaunch(h->graph, h->stream), "step graph launch");
                h->steps += 2;
            }
        }
    }
    for (; s < n_steps; ++s)
        if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
    return LBM_OK;
}

int lbm_step_planes(lbm_lattice* h, int32_t x_begin, int32_t x_end)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (h->pre) return fail(LBM_ERR_STATE, "plane-range steps need a stepped state (take the first step with lbm_step)");
    if (x_begin < 0 || x_end > h->desc.nx || x_begin >= x_end)
        return fail(LBM_ERR_INVALID, "plane range [%d, %d) outside [0, %d) or empty", x_begin, x_end, h->desc.nx);
    if ((rc = check_force_ready(h))) return rc;
    // The register-staged kernel of the lattice's storage and cells per
    // thread, without outputs, over the window's cells.
    LaunchArgs a;
    a.P = h->P;
    a.P.cell0 = x_begin * h->desc.ny * h->desc.nz;
    a.P.cell_end = x_end * h->desc.ny * h->desc.nz;
    a.src = h->buf[h->cur];
    a.dst = h->buf[h->cur ^ 1];
    a.post = false;
    a.f_out = nullptr;
    a.rho = a.u = nullptr;
    a.partials = nullptr;
    a.prev_partials = nullptr;
    a.prev_count = 0;
    a.prev_sums = nullptr;
    a.first = 0;
    a.count = -1;
    a.block = h->block;
    a.vec = h->vec;
    a.stream = h->stream;
    a.grid_used = nullptr;
    a.tma_grid = 0;
    a.rule_quads = h->rule_quads;
    for (int k = 0; k < QUAD_KINDS; ++k) a.rule_counts[k] = h->rule_counts[k];
    a.rules_grid = h->rules_grid;
    cudaError_t e = h->storage == LBM_STORAGE_F64 ? launch_exact(KERNEL_STEP, h->desc.force_mode, a)
                                                  : launch_fast(h->storage, KERNEL_STEP, h->desc.force_mode, a);
    if (e != cudaSuccess) return cuda_fail(e, "plane-range step launch");
    h->open_step = true;
    return LBM_OK;
}

int lbm_step_commit(lbm_lattice* h)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->open_step) return fail(LBM_ERR_STATE, "no plane-range step is open");
    h->cur ^= 1;
    h->steps += 1;
    h->open_step = false;
    return LBM_OK;
}

int lbm_set_rule_blocks(lbm_lattice* h, int32_t blocks)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (blocks < 0 || blocks > 65536) return fail(LBM_ERR_INVALID, "rule blocks must be in [0, 65536]");
    if (h->vec != 4) return fail(LBM_ERR_STATE, "the lattice does not step four cells per thread");
    h->rules_grid_set = blocks;
    return refresh_rule_quads(h);
}

int lbm_get_rule_blocks(const lbm_lattice* h, int32_t* blocks, int32_t* rule_quads)
{
    if (!h) return fail(LBM_ERR_INVALID, "null lattice handle");
    if (blocks) *blocks = h->rules_grid;
    if (rule_quads) *rule_quads = h->rule_counts[0] + h->rule_counts[1] + h->rule_counts[2];
    return LBM_OK;
}

int64_t lbm_step_count(const lbm_lattice* h) { return h ? h->steps : -1; }

int lbm_test_barrier_limit(lbm_lattice* h, int32_t missing_arrivals, int64_t timeout_ns)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!h->persist) return fail(LBM_ERR_STATE, "the lattice was not created with LBM_STAGING_PERSISTENT");
    if (missing_arrivals < 0) return fail(LBM_ERR_INVALID, "missing_arrivals must be >= 0");
    h->persist_missing = (unsigned)missing_arrivals;
    h->persist_timeout_ns = timeout_ns > 0 ? (unsigned long long)timeout_ns : 2000000000ull;
    return LBM_OK;
}

int lbm_get_rho_u(lbm_lattice* h, double* rho, double* u)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_force_ready(h))) return rc;
    if ((rc = observe_rho_u(h, h->rho, h->u))) return rc;
    return readback_to_host(h, h->rho, h->u, rho, u);
}

int lbm_get_rho_u_dev(lbm_lattice* h, double* rho, double* u)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_force_ready(h))) return rc;
    if (!rho && !u) return LBM_OK;
    if ((rc = check_device_ptr(h, rho, "rho")) || (rc = check_device_ptr(h, u, "u"))) return rc;
    const size_t n = (size_t)h->n;
    if (h->storage == LBM_STORAGE_F64) {
        // the readback kernel writes both fields; borrow the handle's buffer
        // for the one not asked for
        return observe_rho_u(h, rho ? rho : h->rho, u ? u : h->u);
    }
    if ((rc = observe_rho_u(h, h->rho, h->u))) return rc;
    if (rho) CK(launch_widen((const float*)h->rho, rho, n, h->stream), "rho widen");
    if (u) CK(launch_widen((const float*)h->u, u, 3 * n, h->stream), "u widen");
    return LBM_OK;
}

int lbm_set_porosity_dev(lbm_lattice* h, const float* alpha)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (!alpha) return fail(LBM_ERR_INVALID, "null porosity field");
    if (h->desc.force_mode != LBM_FORCE_DRAG)
        return fail(LBM_ERR_STATE, "lattice was not created with LBM_FORCE_DRAG");
    if ((rc = check_device_ptr(h, alpha, "alpha"))) return rc;
    const size_t n = (size_t)h->n;
    // range check on the device; the 5-double sum scratch holds the flag
    int* bad = (int*)h->sums;
    int flag = 0;
    CK(cudaMemsetAsync(bad, 0, sizeof(int), h->stream), "flag clear");
    CK(launch_check_unit_interval(alpha, h->n, bad, h->stream), "porosity check");
    CK(cudaMemcpyAsync(&flag, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "flag read");
    CK(cudaStreamSynchronize(h->stream), "porosity check sync");
    if (flag) return fail(LBM_ERR_INVALID, "porosity outside [0, 1] (or NaN)");
    if (!h->poro) CK(cudaMalloc((void**)&h->poro, sizeof(float) * n), "porosity allocation");
    CK(cudaMemcpyAsync(h->poro, alpha, sizeof(float) * n, cudaMemcpyDeviceToDevice, h->stream), "porosity copy");
    rebuild_params(h);
    return LBM_OK;
}

int lbm_run_capture(lbm_lattice* h, int32_t n_steps, int32_t every, double* rho_frames, double* u_frames)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (n_steps < 0 || every < 1) return fail(LBM_ERR_INVALID, "need n_steps >= 0 and every >= 1");
    if (!rho_frames || !u_frames) return fail(LBM_ERR_INVALID, "null frame buffer");
    if ((rc = check_force_ready(h))) return rc;
    const size_t n = (size_t)h->n;
    int frame = 0;
    for (int32_t s = 0; s <= n_steps; ++s) {
        const bool need = (s % every == 0) || (s == n_steps);
        if (s < n_steps) {
            // The step kernel reads back the state it advances from (step s).
            if ((rc = advance(h, need ? h->rho : nullptr, need ? h->u : nullptr, nullptr))) return rc;
        } else if (need) {
            if ((rc = observe_rho_u(h, h->rho, h->u))) return rc;
        }
        if (need) {
            rc = readback_to_host(h, h->rho, h->u, rho_frames + frame * n, u_frames + frame * 3 * n);
            if (rc) return rc;
            ++frame;
        }
    }
    return LBM_OK;
}

int lbm_step_monitor(lbm_lattice* h, int32_t n_steps, double* sums)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_no_open_step(h))) return rc;
    if (n_steps < 0) return fail(LBM_ERR_INVALID, "negative step count");
    if (n_steps > 0 && !sums) return fail(LBM_ERR_INVALID, "null sums array");
    if ((rc = check_force_ready(h))) return rc;
    if (n_steps == 0) return LBM_OK;
    if (h->monitor_cap < n_steps) {
        if (h->monitor) CK(cudaFree(h->monitor), "monitor free");
        h->monitor = nullptr;
        h->monitor_cap = 0;
        CK(cudaMalloc((void**)&h->monitor, sizeof(double) * 5 * (size_t)n_steps), "monitor allocation");
        h->monitor_cap = n_steps;
    }
    // Step s writes its per-block partials into one of two buffers; block 0 of
    // step s + 1 reduces them into monitor row s; one reduction launch ends it.
    PendingSums pend{nullptr, 0, nullptr};
    for (int32_t s = 0; s < n_steps; ++s) {
        double* part = h->partials + (size_t)(s & 1) * 5 * h->partial_blocks;
        int blocks = 0;
        if ((rc = advance(h, nullptr, nullptr, part, &blocks, s > 0 ? &pend : nullptr))) return rc;
        pend = PendingSums{part, blocks, h->monitor + 5 * (size_t)s};
    }
    CK(launch_reduce_partials(pend.partials, pend.count, pend.sums, h->stream), "partial reduction");
    std::vector<double> tmp(5 * (size_t)n_steps);
    CK(cudaMemcpyAsync(tmp.data(), h->monitor, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, h->stream),
       "monitor copy");
    CK(cudaStreamSynchronize(h->stream), "monitor sync");
    for (int32_t s = 0; s < n_steps; ++s) {
        const double* v = tmp.data() + 5 * (size_t)s;
        sums[4 * s + 0] = h->storage == LBM_STORAGE_F64 ? v[0] : v[0] + v[4];
        sums[4 * s + 1] = v[1];
        sums[4 * s + 2] = v[2];
        sums[4 * s + 3] = v[3];
    }
    return LBM_OK;
}

int lbm_conservation(lbm_lattice* h, double* out4)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!out4) return fail(LBM_ERR_INVALID, "null output");
    if ((rc = check_force_ready(h))) return rc;
    cudaError_t e = launch(h, KERNEL_OBSERVE, h->buf[h->cur], nullptr, !h->pre, nullptr, nullptr, nullptr, h->partials);
    if (e != cudaSuccess) return cuda_fail(e, "conservation kernel");
    // the rows the observe launch wrote (one per block of its per-cell grid)
    CK(launch_reduce_partials(h->partials, grid_for(h->n, h->block), h->sums, h->stream), "partial reduction");
    double s[5];
    CK(cudaMemcpyAsync(s, h->sums, sizeof(s), cudaMemcpyDeviceToHost, h->stream), "sum copy");
    CK(cudaStreamSynchronize(h->stream), "sum sync");
    // f32-arithmetic storages sum density deviations; add the cell count back.
    out4[0] = h->storage == LBM_STORAGE_F64 ? s[0] : s[0] + s[4];
    out4[1] = s[1];
    out4[2] = s[2];
    out4[3] = s[3];
    return LBM_OK;
}

int lbm_conservation_planes(lbm_lattice* h, int32_t x0, int32_t x1, double* out4)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!out4) return fail(LBM_ERR_INVALID, "null output");
    if (x0 < 0 || x1 > h->desc.nx || x0 >= x1) return fail(LBM_ERR_INVALID, "plane range [%d, %d) invalid", x0, x1);
    if ((rc = check_force_ready(h))) return rc;
    const int nynz = h->desc.ny * h->desc.nz;
    LaunchArgs a{};
    a.P = h->P;
    a.src = h->buf[h->cur];
    a.post = !h->pre;
    a.partials = h->partials;
    a.block = h->block;
    a.vec = 1;
    a.stream = h->stream;
    a.first = x0 * nynz;
    a.count = (x1 - x0) * nynz;
    const cudaError_t e = h->storage == LBM_STORAGE_F64 ? launch_exact(KERNEL_OBSERVE, h->desc.force_mode, a)
                                                        : launch_fast(h->storage, KERNEL_OBSERVE, h->desc.force_mode, a);
    if (e != cudaSuccess) return cuda_fail(e, "conservation kernel");
    CK(launch_reduce_partials(h->partials, grid_for(a.count, h->block), h->sums, h->stream), "partial reduction");
    double s5[5];
    CK(cudaMemcpyAsync(s5, h->sums, sizeof(s5), cudaMemcpyDeviceToHost, h->stream), "sum copy");
    CK(cudaStreamSynchronize(h->stream), "sum sync");
    out4[0] = h->storage == LBM_STORAGE_F64 ? s5[0] : s5[0] + s5[4];
    out4[1] = s5[1];
    out4[2] = s5[2];
    out4[3] = s5[3];
    return LBM_OK;
}

// Plane x of the stored array, directions in dir_mask, to or from a device
// buffer (direction-major in increasing d, ny * nz elements each).
static int plane_copy(lbm_lattice* h, int32_t x, uint32_t dir_mask, void* dev, bool get)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dev) return fail(LBM_ERR_INVALID, "null plane buffer");
    if (x < 0 || x >= h->desc.nx) return fail(LBM_ERR_INVALID, "plane %d outside [0, %d)", x, h->desc.nx);
    if (dir_mask == 0 || dir_mask >= (1u << Q)) return fail(LBM_ERR_INVALID, "direction mask 0x%x invalid", dir_mask);
    if ((rc = check_device_ptr(h, dev, "plane buffer"))) return rc;
    const size_t plane = (size_t)h->desc.ny * h->desc.nz * h->elem;
    CK(launch_plane_copy(h->buf[h->cur], (size_t)h->n * h->elem, (size_t)x * plane, plane, dir_mask, dev, get,
                         h->stream),
       "plane copy");
    return LBM_OK;
}

int lbm_plane_get(lbm_lattice* h, int32_t x, uint32_t dir_mask, void* dst) { return plane_copy(h, x, dir_mask, dst, true); }

int lbm_plane_put(lbm_lattice* h, int32_t x, uint32_t dir_mask, const void* src)
{
    return plane_copy(h, x, dir_mask, const_cast<void*>(src), false);
}

int lbm_diagnostics(lbm_lattice* h, double dx_phys, double* out6)
{
    int rc = check_handle(h);
    if (rc) return rc;
    if (!out6) return fail(LBM_ERR_INVALID, "null output");
    if (!(dx_phys > 0.0)) return fail(LBM_ERR_INVALID, "dx_phys must be > 0");
    if ((rc = check_force_ready(h))) return rc;
    if (!h->diag) CK(cudaMalloc((void**)&h->diag, sizeof(double) * (DIAG_SCRATCH + 6)), "diagnostics scratch");
    if ((rc = observe_rho_u(h, h->rho, h->u))) return rc;
    const double* rho = (const double*)h->rho;
    const double* u = (const double*)h->u;
    if (h->storage != LBM_STORAGE_F64) {
        // the f32 readback widened to f64, as lbm_get_rho_u hands it out
        if ((rc = ensure_staging(h))) return rc;
        const size_t n = (size_t)h->n;
        CK(launch_widen((const float*)h->rho, h->staging, n, h->stream), "rho widen");
        CK(launch_widen((const float*)h->u, h->staging + n, 3 * n, h->stream), "u widen");
        rho = h->staging;
        u = h->staging + n;
    }
    CK(launch_diagnostics(h->P, rho, u, dx_phys, h->diag, h->diag + DIAG_SCRATCH, h->stream), "diagnostics");
    CK(cudaMemcpyAsync(out6, h->diag + DIAG_SCRATCH, sizeof(double) * 6, cudaMemcpyDeviceToHost, h->stream),
       "diagnostics copy");
    CK(cudaStreamSynchronize(h->stream), "diagnostics sync");
    return LBM_OK;
}

int lbm_check_health(lbm_lattice* h)
{
    double s[4];
    int rc = lbm_conservation(h, s);
    if (rc) return rc;
    if ((rc = check_device_error(h))) return rc;
    for (double v : s)
        if (!(v == v) || v == 1.0 / 0.0 || v == -1.0 / 0.0)
            return fail(LBM_ERR_NONFINITE, "non-finite density or momentum in the lattice");
    return LBM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Stateless reference functions
// ---------------------------------------------------------------------------
namespace {

struct Workspace {
    std::mutex mu;
    int device = -1;
    double* ptr = nullptr;
    size_t cap = 0;  // doubles
};
Workspace g_ws;

// Device scratch for the host-array functions: holds inputs and outputs.
int workspace(size_t doubles, double** out)
{
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    if (g_ws.ptr && (g_ws.cap < doubles || g_ws.device != dev)) {
        cudaFree(g_ws.ptr);
        g_ws.ptr = nullptr;
        g_ws.cap = 0;
    }
    if (!g_ws.ptr) {
        CK(cudaMalloc((void**)&g_ws.ptr, sizeof(double) * doubles), "workspace allocation");
        g_ws.cap = doubles;
        g_ws.device = dev;
    }
    *out = g_ws.ptr;
    return LBM_OK;
}

int ref_params(int nx, int ny, int nz, Params& P)
{
    if (!dims_ok(nx, ny, nz)) return fail(LBM_ERR_INVALID, "invalid lattice dimensions %d x %d x %d", nx, ny, nz);
    if (lbm_device_count() == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device available");
    init_geometry(P, nx, ny, nz);
    return LBM_OK;
}

// LBM_OK when every non-null pointer is device (or managed) memory of the
// current GPU; a host pointer or another GPU's memory handed to a kernel
// would fault the GPU instead of failing here.
int check_dev_ptrs(std::initializer_list<std::pair<const void*, const char*>> ptrs)
{
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    for (const auto& pw : ptrs) {
        if (!pw.first) continue;
        cudaPointerAttributes attr{};
        if (cudaPointerGetAttributes(&attr, pw.first) != cudaSuccess) {
            cudaGetLastError();
            return fail(LBM_ERR_INVALID, "%s is not a CUDA pointer", pw.second);
        }
        const bool ok = attr.type == cudaMemoryTypeManaged || (attr.type == cudaMemoryTypeDevice && attr.device == dev);
        if (!ok) return fail(LBM_ERR_INVALID, "%s must be device memory of GPU %d", pw.second, dev);
    }
    return LBM_OK;
}

int finish(cudaError_t e, const char* what, cudaStream_t s)
{
    if (e != cudaSuccess) return cuda_fail(e, what);
    CK(cudaStreamSynchronize(s), what);
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_release_workspace(void)
{
    std::lock_guard<std::mutex> lk(g_ws.mu);
    if (g_ws.ptr) cudaFree(g_ws.ptr);
    g_ws.ptr = nullptr;
    g_ws.cap = 0;
    return LBM_OK;
}

int lbm_feq_field_dev(const double* rho, const double* u, double* feq, int32_t nx, int32_t ny, int32_t nz,
                      void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!rho || !u || !feq) return fail(LBM_ERR_INVALID, "null pointer");
    if ((rc = check_dev_ptrs({{rho, "rho"}, {u, "u"}, {feq, "feq"}}))) return rc;
    return finish(ref_feq_field(P, rho, u, feq, (cudaStream_t)stream), "feq_field", (cudaStream_t)stream);
}

int lbm_density_field_dev(const double* f, double* rho, int32_t nx, int32_t ny, int32_t nz, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f || !rho) return fail(LBM_ERR_INVALID, "null pointer");
    if ((rc = check_dev_ptrs({{f, "f"}, {rho, "rho"}}))) return rc;
    return finish(ref_density(P, f, rho, (cudaStream_t)stream), "density_field", (cudaStream_t)stream);
}

int lbm_momentum_field_dev(const double* f, double* mom, int32_t nx, int32_t ny, int32_t nz, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f || !mom) return fail(LBM_ERR_INVALID, "null pointer");
    if ((rc = check_dev_ptrs({{f, "f"}, {mom, "mom"}}))) return rc;
    return finish(ref_momentum(P, f, mom, (cudaStream_t)stream), "momentum_field", (cudaStream_t)stream);
}

int lbm_macroscopic_velocity_dev(const double* f, const double* force, double* u, int32_t nx, int32_t ny,
                                 int32_t nz, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f || !u) return fail(LBM_ERR_INVALID, "null pointer");
    if ((rc = check_dev_ptrs({{f, "f"}, {force, "force"}, {u, "u"}}))) return rc;
    return finish(ref_macro_velocity(P, f, force, u, (cudaStream_t)stream), "macroscopic_velocity",
                  (cudaStream_t)stream);
}

int lbm_stream_dev(const double* f_post, double* f_out, int32_t nx, int32_t ny, int32_t nz, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f_post || !f_out || f_post == f_out) return fail(LBM_ERR_INVALID, "null or aliased pointer");
    if ((rc = check_dev_ptrs({{f_post, "f_post"}, {f_out, "f_out"}}))) return rc;
    return finish(ref_stream(P, f_post, f_out, (cudaStream_t)stream), "stream", (cudaStream_t)stream);
}

int lbm_bgk_step_dev(const double* f, double* f_out, double tau, const double* force, int32_t nx, int32_t ny,
                     int32_t nz, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f || !f_out || f == f_out) return fail(LBM_ERR_INVALID, "null or aliased pointer");
    if ((rc = check_dev_ptrs({{f, "f"}, {force, "force"}, {f_out, "f_out"}}))) return rc;
    P.tau = tau;
    return finish(ref_bgk_step(P, f, force, f_out, (cudaStream_t)stream), "bgk_step", (cudaStream_t)stream);
}

int lbm_bounce_back_y_walls_dev(const double* f, double* f_out, int32_t nx, int32_t ny, int32_t nz,
                                const double* top, const double* bottom, void* stream)
{
    Params P;
    int rc = ref_params(nx, ny, nz, P);
    if (rc) return rc;
    if (!f || !f_out || f == f_out) return fail(LBM_ERR_INVALID, "null or aliased pointer");
    if ((rc = check_dev_ptrs({{f, "f"}, {f_out, "f_out"}}))) return rc;
    for (int a = 0; a < 3; ++a) {
        P.wall_u[FACE_YP][a] = top ? top[a] : 0.0;
        P.wall_u[FACE_YM][a] = bottom ? bottom[a] : 0.0;
    }
    return finish(ref_bounce_y(P, f, f_out, (cudaStream_t)stream), "apply_bounce_back_y_walls", (cudaStream_t)stream);
}

// Host-array variants: copy in, run on the default stream, copy out.
#define HOST_PROLOGUE(ndoubles)                              \
    std::lock_guard<std::mutex> lk(g_ws.mu);                 \
    if (lbm_device_count() == 0) return fail(LBM_ERR_NO_DEVICE, "no CUDA device available"); \
    if (!dims_ok(nx, ny, nz)) return fail(LBM_ERR_INVALID, "invalid lattice dimensions"); \
    const size_t n = (size_t)nx * ny * nz;                   \
    double* ws = nullptr;                                    \
    int rc_ = workspace((ndoubles), &ws);                    \
    if (rc_) return rc_;

static int up(double* dst, const double* src, size_t cnt)
{
    CK(cudaMemcpy(dst, src, sizeof(double) * cnt, cudaMemcpyHostToDevice), "host-to-device copy");
    return LBM_OK;
}
static int down(double* dst, const double* src, size_t cnt)
{
    CK(cudaMemcpy(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost), "device-to-host copy");
    return LBM_OK;
}

int lbm_feq_field(const double* rho, const double* u, double* feq, int32_t nx, int32_t ny, int32_t nz)
{
    if (!rho || !u || !feq) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(23 * n)
    int rc;
    if ((rc = up(ws, rho, n)) || (rc = up(ws + n, u, 3 * n))) return rc;
    if ((rc = lbm_feq_field_dev(ws, ws + n, ws + 4 * n, nx, ny, nz, nullptr))) return rc;
    return down(feq, ws + 4 * n, 19 * n);
}

int lbm_density_field(const double* f, double* rho, int32_t nx, int32_t ny, int32_t nz)
{
    if (!f || !rho) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(20 * n)
    int rc;
    if ((rc = up(ws, f, 19 * n))) return rc;
    if ((rc = lbm_density_field_dev(ws, ws + 19 * n, nx, ny, nz, nullptr))) return rc;
    return down(rho, ws + 19 * n, n);
}

int lbm_momentum_field(const double* f, double* mom, int32_t nx, int32_t ny, int32_t nz)
{
    if (!f || !mom) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(22 * n)
    int rc;
    if ((rc = up(ws, f, 19 * n))) return rc;
    if ((rc = lbm_momentum_field_dev(ws, ws + 19 * n, nx, ny, nz, nullptr))) return rc;
    return down(mom, ws + 19 * n, 3 * n);
}

int lbm_macroscopic_velocity(const double* f, const double* force, double* u, int32_t nx, int32_t ny, int32_t nz)
{
    if (!f || !u) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(25 * n)
    int rc;
    if ((rc = up(ws, f, 19 * n))) return rc;
    if (force && (rc = up(ws + 22 * n, force, 3 * n))) return rc;
    if ((rc = lbm_macroscopic_velocity_dev(ws, force ? ws + 22 * n : nullptr, ws + 19 * n, nx, ny, nz, nullptr)))
        return rc;
    return down(u, ws + 19 * n, 3 * n);
}

int lbm_stream(const double* f_post, double* f_out, int32_t nx, int32_t ny, int32_t nz)
{
    if (!f_post || !f_out) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(38 * n)
    int rc;
    if ((rc = up(ws, f_post, 19 * n))) return rc;
    if ((rc = lbm_stream_dev(ws, ws + 19 * n, nx, ny, nz, nullptr))) return rc;
    return down(f_out, ws + 19 * n, 19 * n);
}

int lbm_bgk_step(const double* f, double* f_out, double tau, const double* force, int32_t nx, int32_t ny,
                 int32_t nz)
{
    if (!f || !f_out) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(41 * n)
    int rc;
    if ((rc = up(ws, f, 19 * n))) return rc;
    if (force && (rc = up(ws + 38 * n, force, 3 * n))) return rc;
    if ((rc = lbm_bgk_step_dev(ws, ws + 19 * n, tau, force ? ws + 38 * n : nullptr, nx, ny, nz, nullptr)))
        return rc;
    return down(f_out, ws + 19 * n, 19 * n);
}

int lbm_bounce_back_y_walls(const double* f, double* f_out, int32_t nx, int32_t ny, int32_t nz, const double* top,
                            const double* bottom)
{
    if (!f || !f_out) return fail(LBM_ERR_INVALID, "null pointer");
    HOST_PROLOGUE(38 * n)
    int rc;
    if ((rc = up(ws, f, 19 * n))) return rc;
    if ((rc = lbm_bounce_back_y_walls_dev(ws, ws + 19 * n, nx, ny, nz, top, bottom, nullptr))) return rc;
    return down(f_out, ws + 19 * n, 19 * n);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches
// ---------------------------------------------------------------------------
#include "lbm_batch.cuh"

struct lbm_batch {
    int count = 0;
    int storage = 0;
    int force_mode = 0;
    int device = 0;
    std::vector<lbm_lattice*> lats;
    cudaStream_t stream = nullptr;
    void* records = nullptr;       // count BatchLattice records (layout independent of T)
    std::vector<BatchLattice<float>> host_records;
    BatchItem* items = nullptr;
    int nitems = 0;
    int items_cap = 0;
    int sched = SCHED_SINGLE;
    int block = 256;
    int grid = 0;
    int sms = 1;
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;
    // SCHED_BRANCHES: `grid` streams; lattice i steps on branches[branch_of[i]]
    // (largest lattices first, each to the branch with the fewest cells).  The
    // two-step graph holds every lattice's buffers and parameters: it is
    // recaptured when a lattice's buffer parity or parameters differ from
    // the capture's.
    std::vector<cudaStream_t> branches;
    std::vector<cudaEvent_t> branch_done;
    cudaEvent_t root = nullptr;
    std::vector<int> branch_of, branch_order;
    std::vector<int> graph_cur, graph_params;
};

namespace {

int batch_span(const lbm_batch* b) { return b->block * (b->sched == SCHED_SINGLE ? 1 : 2); }

int batch_build_items(lbm_batch* b)
{
    const int span = batch_span(b);
    // Lattices by kind (even nz, which the pair schedules step with vector
    // access, before odd nz), then by size: neighbouring blocks run items
    // of one kind at a time.
    std::vector<int> order(b->count);
    for (int i = 0; i < b->count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) {
        const int oi = b->lats[i]->desc.nz % 2, oj = b->lats[j]->desc.nz % 2;
        return oi != oj ? oi < oj : b->lats[i]->n > b->lats[j]->n;
    });
    std::vector<BatchItem> items;
    for (int i : order)
        for (int c = 0; c < b->lats[i]->n; c += span) items.push_back(BatchItem{i, c});
    if ((int)items.size() > b->items_cap) {
        if (b->items) CK(cudaFree(b->items), "batch items free");
        b->items = nullptr;
        b->items_cap = 0;
        CK(cudaMalloc((void**)&b->items, sizeof(BatchItem) * items.size()), "batch items allocation");
        b->items_cap = (int)items.size();
    }
    CK(cudaMemcpy(b->items, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice), "items upload");
    b->nitems = (int)items.size();
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->graph_valid = false;
    return LBM_OK;
}

int batch_grid(const lbm_batch* b)
{
    if (b->sched == SCHED_BRANCHES) return b->grid > 0 ? b->grid : 8;
    const int g = b->grid > 0 ? b->grid : 4 * b->sms;
    return g < b->nitems ? g : b->nitems;
}

void batch_free_branches(lbm_batch* b)
{
    for (cudaStream_t s : b->branches) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->branch_done) cudaEventDestroy(e);
    b->branches.clear();
    b->branch_done.clear();
}

// Streams, events and the lattice -> branch assignment of SCHED_BRANCHES.
int batch_build_branches(lbm_batch* b, int nb)
{
    if ((int)b->branches.size() != nb) {
        CK(cudaStreamSynchronize(b->stream), "batch sync");
        batch_free_branches(b);
        for (int k = 0; k < nb; ++k) {
            cudaStream_t s = nullptr;
            cudaEvent_t e = nullptr;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "branch stream");
            b->branches.push_back(s);
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "branch event");
            b->branch_done.push_back(e);
        }
    }
    if (!b->root) CK(cudaEventCreateWithFlags(&b->root, cudaEventDisableTiming), "root event");
    b->branch_order.resize(b->count);
    for (int i = 0; i < b->count; ++i) b->branch_order[i] = i;
    std::stable_sort(b->branch_order.begin(), b->branch_order.end(),
                     [&](int i, int j) { return b->lats[i]->n > b->lats[j]->n; });
    std::vector<long long> load(nb, 0);
    b->branch_of.assign(b->count, 0);
    for (int i : b->branch_order) {
        int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->branch_of[i] = k;
        load[k] += b->lats[i]->n;
    }
    return LBM_OK;
}

// One step of every lattice (phase 0: buf[cur] -> buf[cur ^ 1], phase 1 the
// reverse) with each lattice's own kernels on its branch, forked from and
// joined into the batch stream.
cudaError_t batch_branch_step(lbm_batch* b, int phase)
{
    cudaError_t e;
    if ((e = cudaEventRecord(b->root, b->stream)) != cudaSuccess) return e;
    const int nb = (int)b->branches.size();
    for (int k = 0; k < nb; ++k)
        if ((e = cudaStreamWaitEvent(b->branches[k], b->root, 0)) != cudaSuccess) return e;
    for (int i : b->branch_order) {
        lbm_lattice* h = b->lats[i];
        const int c = h->cur ^ phase;
        cudaStream_t own = h->stream;
        h->stream = b->branches[b->branch_of[i]];
        e = launch(h, KERNEL_STEP, h->buf[c], h->buf[c ^ 1], false, nullptr, nullptr, nullptr, nullptr);
        h->stream = own;
        if (e != cudaSuccess) return e;
    }
    for (int k = 0; k < nb; ++k) {
        if ((e = cudaEventRecord(b->branch_done[k], b->branches[k])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(b->stream, b->branch_done[k], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

bool batch_branch_graph_current(const lbm_batch* b)
{
    if (!b->graph_valid || (int)b->graph_cur.size() != b->count) return false;
    for (int i = 0; i < b->count; ++i)
        if (b->graph_cur[i] != b->lats[i]->cur || b->graph_params[i] != b->lats[i]->params_version) return false;
    return true;
}

// Records for the next steps: phase 0 reads buf[cur], phase 1 the other.
int batch_upload_records(lbm_batch* b)
{
    for (int i = 0; i < b->count; ++i) {
        lbm_lattice* h = b->lats[i];
        BatchLattice<float>& r = b->host_records[i];
        r.P = h->P;
        r.S[0] = make_streams<float>(nullptr, nullptr, h->n);
        // the pointer layout does not depend on T: fill as bytes of the storage
        for (int d = 0; d < Q; ++d) {
            const char* a = (const char*)h->buf[h->cur] + (size_t)d * h->n * h->elem;
            const char* c = (const char*)h->buf[h->cur ^ 1] + (size_t)d * h->n * h->elem;
            r.S[0].src[d] = (const float*)a;
            r.S[0].dst[d] = (float*)c;
            r.S[1].src[d] = (const float*)c;
            r.S[1].dst[d] = (float*)a;
        }
        r.vec = (h->storage != LBM_STORAGE_F64 && h->desc.nz % 2 == 0) ? 2 : 1;
    }
    CK(cudaMemcpyAsync(b->records, b->host_records.data(), sizeof(BatchLattice<float>) * b->count,
                       cudaMemcpyHostToDevice, b->stream),
       "records upload");
    return LBM_OK;
}

void batch_advance_bookkeeping(lbm_batch* b, int steps)
{
    for (lbm_lattice* h : b->lats) {
        if (steps % 2) h->cur ^= 1;
        h->pre = false;
        h->steps += steps;
    }
}

cudaError_t batch_launch(lbm_batch* b, bool collide, int phase)
{
    return launch_batch_step(b->storage, b->force_mode, b->sched, collide, b->records, b->items, b->nitems,
                             batch_span(b), phase, batch_grid(b), b->block, b->stream);
}

int batch_check(lbm_batch* b)
{
    if (!b) return fail(LBM_ERR_INVALID, "null batch handle");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    for (lbm_lattice* h : b->lats) {
        int rc = check_force_ready(h);
        if (rc) return rc;
    }
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_batch_create(const lbm_desc* descs, int32_t count, lbm_batch** out)
{
    if (!descs || !out || count < 1) return fail(LBM_ERR_INVALID, "need descriptors, count >= 1 and an output");
    *out = nullptr;
    for (int i = 1; i < count; ++i)
        if (descs[i].storage != descs[0].storage || descs[i].force_mode != descs[0].force_mode ||
            descs[i].device != descs[0].device)
            return fail(LBM_ERR_INVALID, "lattices of a batch share storage, force model and device");
    lbm_batch* b = new lbm_batch();
    b->count = count;
    b->storage = descs[0].storage;
    b->force_mode = descs[0].force_mode;
    b->device = descs[0].device;
    auto cleanup = [&](int code) {
        lbm_batch_destroy(b);
        return code;
    };
    int rc;
    for (int i = 0; i < count; ++i) {
        lbm_lattice* h = nullptr;
        if ((rc = lbm_create(&descs[i], &h))) return cleanup(rc);
        b->lats.push_back(h);
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "batch stream"));
    for (lbm_lattice* h : b->lats)
        if ((rc = lbm_set_stream(h, b->stream))) return cleanup(rc);
    b->host_records.resize(count);
    e = cudaMalloc(&b->records, sizeof(BatchLattice<float>) * count);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "batch records"));
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    if (b->sms < 1) b->sms = 1;
    if ((rc = batch_build_items(b))) return cleanup(rc);
    *out = b;
    return LBM_OK;
}

int lbm_batch_destroy(lbm_batch* b)
{
    if (!b) return LBM_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    batch_free_branches(b);
    if (b->root) cudaEventDestroy(b->root);
    for (lbm_lattice* h : b->lats) {
        h->stream = nullptr;  // the batch owns the stream
        h->own_stream = false;
        lbm_destroy(h);
    }
    if (b->records) cudaFree(b->records);
    if (b->items) cudaFree(b->items);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return LBM_OK;
}

int lbm_batch_count(const lbm_batch* b) { return b ? b->count : -1; }

int lbm_batch_lattice(lbm_batch* b, int32_t i, lbm_lattice** out)
{
    if (!b || !out || i < 0 || i >= b->count) return fail(LBM_ERR_INVALID, "bad batch index");
    *out = b->lats[i];
    return LBM_OK;
}

int lbm_batch_set_schedule(lbm_batch* b, int32_t sched, int32_t block, int32_t grid)
{
    if (!b) return fail(LBM_ERR_INVALID, "null batch handle");
    if (sched < SCHED_SINGLE || sched > SCHED_BRANCHES) return fail(LBM_ERR_INVALID, "unknown schedule %d", sched);
    if ((sched == SCHED_PAIR_SCALAR || sched == SCHED_PAIR_MIXED) &&
        (b->storage == LBM_STORAGE_F64 || b->force_mode == LBM_FORCE_FIELD || b->force_mode == LBM_FORCE_DRAG))
        return fail(LBM_ERR_UNSUPPORTED, "two-cell schedules need f32/f16/bf16 storage and no per-cell force");
    if (block < 32 || block > 256 || block % 32) return fail(LBM_ERR_INVALID, "block must be a multiple of 32 <= 256");
    if (grid < 0) return fail(LBM_ERR_INVALID, "negative grid");
    if (sched == SCHED_BRANCHES && grid > 64) return fail(LBM_ERR_INVALID, "at most 64 branches");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    b->sched = sched;
    b->block = block;
    b->grid = grid;
    int rc;
    if (sched == SCHED_BRANCHES && (rc = batch_build_branches(b, batch_grid(b)))) return rc;
    return batch_build_items(b);
}

int lbm_batch_get_schedule(const lbm_batch* b, int32_t* sched, int32_t* block, int32_t* grid)
{
    if (!b) return fail(LBM_ERR_INVALID, "null batch handle");
    if (sched) *sched = b->sched;
    if (block) *block = b->block;
    if (grid) *grid = batch_grid(b);
    return LBM_OK;
}

int lbm_batch_synchronize(lbm_batch* b)
{
    if (!b) return fail(LBM_ERR_INVALID, "null batch handle");
    CK(cudaSetDevice(b->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(b->stream), "batch sync");
    return LBM_OK;
}

int lbm_batch_step(lbm_batch* b, int32_t n_steps)
{
    int rc = batch_check(b);
    if (rc) return rc;
    if (n_steps < 0) return fail(LBM_ERR_INVALID, "negative step count");
    int done = 0;
    // First step: lattices holding f_n collide in place.  A batch whose
    // lattices are in different states takes one step lattice by lattice.
    int n_pre = 0;
    for (lbm_lattice* h : b->lats) n_pre += h->pre ? 1 : 0;
    if (n_steps > 0 && n_pre > 0) {
        if (n_pre == b->count) {
            if ((rc = batch_upload_records(b))) return rc;
            CK(batch_launch(b, true, 0), "batch collide launch");
            batch_advance_bookkeeping(b, 1);
        } else {
            for (lbm_lattice* h : b->lats)
                if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
        }
        done = 1;
    }
    const int rest = n_steps - done;
    if (rest <= 0) return LBM_OK;
    if (b->sched == SCHED_BRANCHES) {
        if (rest >= 2 && !batch_branch_graph_current(b)) {
            if (b->graph) cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
            b->graph_valid = false;
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture begin");
            cudaError_t e0 = batch_branch_step(b, 0);
            cudaError_t e1 = e0 == cudaSuccess ? batch_branch_step(b, 1) : e0;
            cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
            if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return cuda_fail(e0 != cudaSuccess ? e0 : (e1 != cudaSuccess ? e1 : e2), "branch graph capture");
            }
            cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(e, "branch graph instantiate");
            b->graph_valid = true;
            b->graph_cur.resize(b->count);
            b->graph_params.resize(b->count);
            for (int i = 0; i < b->count; ++i) {
                b->graph_cur[i] = b->lats[i]->cur;
                b->graph_params[i] = b->lats[i]->params_version;
            }
        }
        for (int k = 0; k + 1 < rest; k += 2) CK(cudaGraphLaunch(b->graph, b->stream), "branch graph launch");
        if (rest % 2) CK(batch_branch_step(b, 0), "branch step launch");
        batch_advance_bookkeeping(b, rest);
        return LBM_OK;
    }
    if ((rc = batch_upload_records(b))) return rc;
    if (rest >= 2 && !b->graph_valid) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "graph capture begin");
        cudaError_t e0 = batch_launch(b, false, 0);
        cudaError_t e1 = batch_launch(b, false, 1);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e0 != cudaSuccess || e1 != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e0 != cudaSuccess ? e0 : (e1 != cudaSuccess ? e1 : e2), "batch graph capture");
        }
        cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
        b->graph_valid = true;
    }
    for (int k = 0; k + 1 < rest; k += 2) CK(cudaGraphLaunch(b->graph, b->stream), "batch graph launch");
    if (rest % 2) CK(batch_launch(b, false, 0), "batch step launch");
    batch_advance_bookkeeping(b, rest);
    return LBM_OK;
}

int lbm_batch_step_unbatched(lbm_batch* b, int32_t n_steps)
{
    int rc = batch_check(b);
    if (rc) return rc;
    if (n_steps < 0) return fail(LBM_ERR_INVALID, "negative step count");
    for (int s = 0; s < n_steps; ++s)
        for (lbm_lattice* h : b->lats)
            if ((rc = advance(h, nullptr, nullptr, nullptr))) return rc;
    return LBM_OK;
}

int lbm_batch_autotune(lbm_batch* b, int32_t trial_steps, double* best_ms)
{
    int rc = batch_check(b);
    if (rc) return rc;
    if (trial_steps < 2) return fail(LBM_ERR_INVALID, "trial_steps must be >= 2");
    trial_steps += trial_steps % 2;  // even: every lattice returns to its buffer parity
    // Save both buffers and the state flags of every lattice.
    std::vector<void*> saved;
    for (lbm_lattice* h : b->lats) {
        const size_t bytes = h->elem * Q * (size_t)h->n;
        for (int k = 0; k < 2; ++k) {
            void* p = nullptr;
            cudaError_t e = cudaMalloc(&p, bytes);
            if (e != cudaSuccess) {
                for (void* q : saved) cudaFree(q);
                return cuda_fail(e, "autotune snapshot");
            }
            cudaMemcpyAsync(p, h->buf[k], bytes, cudaMemcpyDeviceToDevice, b->stream);
            saved.push_back(p);
        }
    }
    std::vector<int> cur0, pre0;
    std::vector<int64_t> steps0;
    for (lbm_lattice* h : b->lats) {
        cur0.push_back(h->cur);
        pre0.push_back(h->pre);
        steps0.push_back(h->steps);
    }
    const int old_sched = b->sched, old_block = b->block, old_grid = b->grid;
    // warm the lattices into the steady state once
    if ((rc = lbm_batch_step(b, 1))) goto restore;
    {
        std::vector<int> scheds = {SCHED_SINGLE};
        if (b->storage != LBM_STORAGE_F64 && (b->force_mode == LBM_FORCE_NONE || b->force_mode == LBM_FORCE_UNIFORM)) {
            scheds.push_back(SCHED_PAIR_SCALAR);
            scheds.push_back(SCHED_PAIR_MIXED);
        }
        double best = 1e30;
        int bs = old_sched, bb = old_block, bg = old_grid;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        scheds.push_back(SCHED_BRANCHES);
        for (int sc : scheds)
            for (int blk : {128, 256})
                for (int per_sm : {2, 4, 8}) {
                    // SCHED_BRANCHES: 4, 8 or 16 branches, once (the block size is each lattice's own)
                    if (sc == SCHED_BRANCHES && blk != 128) continue;
                    const int g = sc == SCHED_BRANCHES ? 2 * per_sm : per_sm * b->sms;
                    if ((rc = lbm_batch_set_schedule(b, sc, blk, g))) break;
                    if ((rc = lbm_batch_step(b, 2))) break;  // capture + warm
                    cudaEventRecord(e0, b->stream);
                    if ((rc = lbm_batch_step(b, trial_steps))) break;
                    cudaEventRecord(e1, b->stream);
                    cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    const double per = ms / trial_steps;
                    if (per < best) {
                        best = per;
                        bs = sc;
                        bb = blk;
                        bg = g;
                    }
                }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc == LBM_OK) {
            if (best_ms) *best_ms = best;
            rc = lbm_batch_set_schedule(b, bs, bb, bg);
            goto restore_state;
        }
    }
restore:
    lbm_batch_set_schedule(b, old_sched, old_block, old_grid);
restore_state:
    cudaStreamSynchronize(b->stream);
    for (int i = 0; i < b->count; ++i) {
        lbm_lattice* h = b->lats[i];
        const size_t bytes = h->elem * Q * (size_t)h->n;
        for (int k = 0; k < 2; ++k) {
            cudaMemcpyAsync(h->buf[k], saved[2 * i + k], bytes, cudaMemcpyDeviceToDevice, b->stream);
        }
        h->cur = cur0[i];
        h->pre = pre0[i];
        h->steps = steps0[i];
    }
    cudaStreamSynchronize(b->stream);
    for (void* p : saved) cudaFree(p);
    return rc;
}

}  // extern "C"
