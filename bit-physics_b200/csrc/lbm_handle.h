// lbm_handle.h -- the lattice handle behind the C ABI and the host helpers
// that the API translation units share (lbm_api.cu, lbm_tape.cu).  Internal:
// not installed, not part of include/.
#pragma once

#include <cstdint>

#include "lbm_d3q19.h"
#include "lbm_launch.h"

// The opaque lbm_lattice of include/lbm_d3q19.h.
struct lbm_lattice {
    lbm_desc desc{};
    int storage = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int n = 0;
    size_t elem = 0;
    void* buf[2] = {nullptr, nullptr};
    int cur = 0;
    bool pre = true;
    bool open_step = false;  // lbm_step_planes ran since the last commit
    uint8_t* flags = nullptr;
    uint32_t* bbmask = nullptr; // (n) bounce-back masks, allocated with the flags
    bool has_flags = false;
    void* force = nullptr;   // (3, n) double (f64 storage) or float
    float* poro = nullptr;   // (n)
    void* rho = nullptr;     // readback buffers, double (f64 storage) or float
    void* u = nullptr;
    double* partials = nullptr;  // 2 x partial_blocks rows of 5 (alternating in step_monitor)
    double* sums = nullptr;  // 5 doubles
    int partial_blocks = 0;  // rows of partials of one launch (one per block, any kernel)
    double* staging = nullptr; // (19, n) f64, allocated on first use
    double* monitor = nullptr; // (monitor_cap, 5) per-step sums of lbm_step_monitor
    double* diag = nullptr;    // DIAG_SCRATCH + 6 doubles of lbm_diagnostics, allocated on first use
    uint16_t* me_codes = nullptr; // (19, n) 16-bit moment codes of lbm_moment16_step, allocated on first use
    int monitor_cap = 0;
    int64_t steps = 0;
    int block = 256;
    int vec = 1; // cells per thread of the fused step kernel
    int* err = nullptr; // device error word (pipeline wait timeouts)
    // Two-step CUDA graph of the steady-state step (buf[graph_cur] -> other ->
    // back), valid while params_version == graph_version.
    cudaGraphExec_t graph = nullptr;
    int graph_cur = -1;
    int params_version = 0;
    int graph_version = -1;
    bool use_tma = false;
    int tma_grid = 0;
    int pipe_grid = 0;  // > 0: steps without outputs run k_step2_pipe
    int sums_grid = 0;  // > 0: steps with FP64 sums run k_step2_sums
    // Four-cell steps (vec == 4): the quads that need a boundary rule, stepped
    // by the leading rules_grid blocks of k_step4.
    int* rule_quads = nullptr;  // QUAD_KINDS lists of n / 4 entries, then the counts
    int* order = nullptr;       // Params::order of the plain one- / two-cell steps (walled lattices)
    int rule_counts[lbm::QUAD_KINDS] = {0, 0, 0};
    int rules_grid = 0;
    int rules_grid_set = 0;     // lbm_set_rule_blocks (0: sized from the lists)
    int sms = 148;              // SMs of the lattice's device
    // Many steps per cooperative launch (LBM_STAGING_PERSISTENT): barrier
    // state, the limit of one barrier wait, and arrivals added to the
    // expected count (nonzero only through lbm_test_barrier_limit).
    bool persist = false;
    lbm::GridBarrier* bar = nullptr;
    unsigned long long persist_timeout_ns = 2000000000ull;
    unsigned persist_missing = 0;
    lbm::TileCfg tile{};
    lbm::Params P{};
};

namespace lbm {
namespace api {

// Record an error message for lbm_last_error() and return code.
int fail(int code, const char* fmt, ...);
// LBM_ERR_NOMEM for allocation failures, LBM_ERR_CUDA otherwise.
int cuda_fail(cudaError_t e, const char* what);

int check_handle(const lbm_lattice* h);
// LBM_ERR_STATE when the force model's field has not been set.
int check_force_ready(lbm_lattice* h);
// One kernel of the handle's configuration (KernelKind) from src to dst.
// Partials of an earlier launch that the next launch with partials reduces
// (its block 0) into sums.
struct PendingSums {
    const double* partials;
    int count;
    double* sums;
};
cudaError_t launch(lbm_lattice* h, int kernel, const void* src, void* dst, bool post, double* f_out, void* rho,
                   void* u, double* partials, int* grid_used = nullptr, const PendingSums* prev = nullptr);
// Advance the handle by one step (rho/u/partials: optional readback of the
// state before the step; *blocks: the number of partials written; prev:
// with partials, earlier partials this step's kernel reduces as well).
int advance(lbm_lattice* h, void* rho, void* u, double* partials, int* blocks = nullptr,
            const PendingSums* prev = nullptr);
// Readback of the current state into the handle's rho/u buffers.
int observe_rho_u(lbm_lattice* h, void* drho, void* du);
// LBM_OK when p is NULL or device (or managed) memory of the handle's GPU,
// LBM_ERR_INVALID naming `what` otherwise (a host pointer would fault a kernel).
int check_device_ptr(const lbm_lattice* h, const void* p, const char* what);

}  // namespace api
}  // namespace lbm

#define CK(call, what)                                                 \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return ::lbm::api::cuda_fail(e_, what); \
    } while (0)
