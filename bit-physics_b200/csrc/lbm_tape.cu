// lbm_tape.cu -- the adjoint tape of include/lbm_d3q19.h: a forward run that
// keeps a state every `every` steps, and a backward pass that replays each
// segment with the step kernels (storing its states) and runs the adjoint
// level kernels (lbm_adjoint.cuh) over it from the last step to the first.
//
// State s_k = the lattice buffer after k steps: s_0 = f_0 (PRE), s_k = P_{k-1}.
// Memory: ceil(N / K) checkpoints + the final state + K - 1 segment states
// + two adjoint fields + the special-cell list, all in one device allocation.
#include <algorithm>
#include <vector>

#include "lbm_adjoint.cuh"
#include "lbm_handle.h"

using namespace lbm;
using namespace lbm::api;

struct lbm_tape {
    lbm_lattice* h = nullptr;
    int device = 0;
    int32_t n_steps = 0;
    int32_t every = 0;
    int params_version = 0;
    void* arena = nullptr;
    int64_t bytes = 0;
    size_t state_bytes = 0;       // exact size of one state
    std::vector<void*> ck;        // s_0, s_K, s_2K, ...
    void* final_state = nullptr;  // s_N
    std::vector<void*> seg;       // s_{jK+1} .. s_{jK+K-1} of the segment in replay
    void* lam[2] = {nullptr, nullptr};
    int* special = nullptr;       // cells of k_adjoint_special (capacity n), then a count
    int n_special = 0;
    // The special-cell kernel of a level runs on `side`, forked from and
    // joined back into the lattice's stream, beside the plain-cell kernel.
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

namespace {

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

void free_tape(lbm_tape* t)
{
    if (!t) return;
    cudaSetDevice(t->device);
    if (t->side) cudaStreamSynchronize(t->side);
    if (t->arena) cudaFree(t->arena);
    if (t->fork) cudaEventDestroy(t->fork);
    if (t->join) cudaEventDestroy(t->join);
    if (t->side) cudaStreamDestroy(t->side);
    delete t;
}

int level(lbm_tape* t, int kind, AdjointArgs& a)
{
    const bool fork = kind != ADJ_FINAL && a.n_special > 0;
    if (fork) {
        CK(cudaEventRecord(t->fork, a.stream), "fork record");
        CK(cudaStreamWaitEvent(t->side, t->fork, 0), "fork wait");
    }
    a.special_stream = fork ? t->side : nullptr;
    cudaError_t e = launch_adjoint_level(t->h->storage, t->h->desc.force_mode, kind, a);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint kernel launch");
    if (fork) {
        CK(cudaEventRecord(t->join, t->side), "join record");
        CK(cudaStreamWaitEvent(a.stream, t->join, 0), "join wait");
    }
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_tape_forward(lbm_lattice* h, int32_t n_steps, int32_t checkpoint_every, lbm_tape** out)
{
    if (!out) return fail(LBM_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int rc = check_handle(h);
    if (rc) return rc;
    if ((rc = check_force_ready(h))) return rc;
    if (n_steps < 1) return fail(LBM_ERR_INVALID, "a tape needs at least one step (got %d)", n_steps);
    if (checkpoint_every < 1) return fail(LBM_ERR_INVALID, "checkpoint_every must be >= 1");
    if (!h->pre)
        return fail(LBM_ERR_STATE, "a tape starts from populations set by lbm_set_populations / "
                                   "lbm_set_equilibrium and not stepped since");
    const int32_t every = checkpoint_every < n_steps ? checkpoint_every : n_steps;
    const int nck = (n_steps + every - 1) / every;
    lbm_tape* t = new lbm_tape();
    t->h = h;
    t->device = h->desc.device;
    t->n_steps = n_steps;
    t->every = every;
    t->state_bytes = h->elem * Q * (size_t)h->n;
    cudaError_t es = cudaStreamCreateWithFlags(&t->side, cudaStreamNonBlocking);
    if (es == cudaSuccess) es = cudaEventCreateWithFlags(&t->fork, cudaEventDisableTiming);
    if (es == cudaSuccess) es = cudaEventCreateWithFlags(&t->join, cudaEventDisableTiming);
    if (es != cudaSuccess) {
        free_tape(t);
        return cuda_fail(es, "tape stream / event creation");
    }
    const size_t sb = round_up(t->state_bytes, 256);
    const size_t lb = round_up(adjoint_elem_bytes(h->storage) * Q * (size_t)h->n, 256);
    const size_t nstates = (size_t)nck + 1 + (size_t)(every - 1);
    const size_t listb = round_up(sizeof(int) * ((size_t)h->n + 1), 256);
    const size_t total = nstates * sb + 2 * lb + listb;
    cudaError_t e = cudaMalloc(&t->arena, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_tape(t);
        return fail(e == cudaErrorMemoryAllocation ? LBM_ERR_NOMEM : LBM_ERR_CUDA,
                    "tape allocation of %.2f GB (%d checkpoints + %d segment states): %s", total / 1e9, nck,
                    every - 1, cudaGetErrorString(e));
    }
    t->bytes = (int64_t)total;
    char* p = (char*)t->arena;
    for (int j = 0; j < nck; ++j, p += sb) t->ck.push_back(p);
    t->final_state = p;
    p += sb;
    for (int i = 0; i + 1 < every; ++i, p += sb) t->seg.push_back(p);
    t->lam[0] = p;
    t->lam[1] = p + lb;
    t->special = (int*)(p + 2 * lb);
    int* count = t->special + h->n;
    e = launch_list_special(h->P, t->special, count, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&t->n_special, count, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess && t->n_special > 1) {
        // into lattice order: neighbouring cells in a warp's consecutive tasks
        std::vector<int> cells(t->n_special);
        e = cudaMemcpy(cells.data(), t->special, sizeof(int) * cells.size(), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) {
            std::sort(cells.begin(), cells.end());
            e = cudaMemcpy(t->special, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice);
        }
    }
    if (e != cudaSuccess) {
        free_tape(t);
        return cuda_fail(e, "special-cell list");
    }
    for (int j = 0; j < nck; ++j) {
        e = cudaMemcpyAsync(t->ck[j], h->buf[h->cur], t->state_bytes, cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) {
            free_tape(t);
            return cuda_fail(e, "checkpoint copy");
        }
        const int32_t steps = n_steps - j * every < every ? n_steps - j * every : every;
        if ((rc = lbm_step(h, steps))) {
            free_tape(t);
            return rc;
        }
    }
    e = cudaMemcpyAsync(t->final_state, h->buf[h->cur], t->state_bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess) {
        free_tape(t);
        return cuda_fail(e, "final state copy");
    }
    t->params_version = h->params_version;
    *out = t;
    return LBM_OK;
}

int lbm_tape_backward(lbm_tape* t, const double* grad_rho, const double* grad_u, double* grad_alpha, double* grad_f0)
{
    if (!t) return fail(LBM_ERR_INVALID, "null tape");
    lbm_lattice* h = t->h;
    int rc = check_handle(h);
    if (rc) return rc;
    if (h->params_version != t->params_version)
        return fail(LBM_ERR_STATE, "the lattice's flags, fields or parameters changed after the taped forward");
    if ((rc = check_device_ptr(h, grad_rho, "grad_rho")) || (rc = check_device_ptr(h, grad_u, "grad_u")) ||
        (rc = check_device_ptr(h, grad_alpha, "grad_alpha")) || (rc = check_device_ptr(h, grad_f0, "grad_f0")))
        return rc;
    const size_t n = (size_t)h->n;
    if (grad_alpha) CK(cudaMemsetAsync(grad_alpha, 0, sizeof(double) * n, h->stream), "gradient clear");
    const size_t lb = adjoint_elem_bytes(h->storage) * Q * n;
    CK(cudaMemsetAsync(t->lam[0], 0, lb, h->stream), "adjoint clear");
    CK(cudaMemsetAsync(t->lam[1], 0, lb, h->stream), "adjoint clear");
    AdjointArgs a{};
    a.P = h->P;
    a.stream = h->stream;
    a.dalpha = h->desc.force_mode == LBM_FORCE_DRAG ? grad_alpha : nullptr;
    a.special = t->special;
    a.n_special = t->n_special;
    // level N: the loss seeds on f_N, rebuilt from s_N
    a.src = t->final_state;
    a.Lout = t->lam[0];
    a.grad_rho = grad_rho;
    a.grad_u = grad_u;
    if ((rc = level(t, ADJ_INIT, a))) return rc;
    a.grad_rho = a.grad_u = nullptr;
    int cur = 0;
    const int nck = (int)t->ck.size();
    for (int j = nck - 1; j >= 0; --j) {
        const int32_t base = j * t->every;
        const int32_t len = t->n_steps - base < t->every ? t->n_steps - base : t->every;
        // replay s_{base+1} .. s_{base+len-1} into the segment states
        const void* prev = t->ck[j];
        for (int32_t i = 1; i < len; ++i) {
            const int kind = base + i - 1 == 0 ? KERNEL_COLLIDE_LOCAL : KERNEL_STEP;
            cudaError_t e = launch(h, kind, prev, t->seg[i - 1], false, nullptr, nullptr, nullptr, nullptr);
            if (e != cudaSuccess) return cuda_fail(e, "segment replay");
            prev = t->seg[i - 1];
        }
        // levels base+len-1 .. base+1 over the segment, then level base
        for (int32_t k = base + len - 1; k > base; --k) {
            a.src = t->seg[k - base - 1];
            a.Lin = t->lam[cur];
            a.Lout = t->lam[cur ^ 1];
            if ((rc = level(t, ADJ_STEP, a))) return rc;
            cur ^= 1;
        }
        a.src = t->ck[j];
        a.Lin = t->lam[cur];
        if (base == 0) {
            a.Lout = nullptr;
            a.grad_f0 = grad_f0;
            if ((rc = level(t, ADJ_FINAL, a))) return rc;
        } else {
            a.Lout = t->lam[cur ^ 1];
            if ((rc = level(t, ADJ_STEP, a))) return rc;
            cur ^= 1;
        }
    }
    return LBM_OK;
}

int64_t lbm_tape_bytes(const lbm_tape* t) { return t ? t->bytes : -1; }

int lbm_tape_destroy(lbm_tape* t)
{
    if (!t) return LBM_OK;
    free_tape(t);
    return LBM_OK;
}

}  // extern "C"
