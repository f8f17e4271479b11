// lbm_launch.h -- host-side launch entry points of the kernel translation
// units (lbm_exact.cu: f64 reference-order arithmetic, built --fmad=false;
// lbm_fast.cu: f32 arithmetic for f32 / f16 / bf16 storage).
#pragma once

#include <cuda_runtime.h>

#include "lbm_device.cuh"
#include "lbm_kernels.cuh"

namespace lbm {

enum StorageKind : int { STORAGE_F64 = 0, STORAGE_F32 = 1, STORAGE_F16 = 2, STORAGE_BF16 = 3 };
enum KernelKind : int { KERNEL_STEP = 0, KERNEL_COLLIDE_LOCAL = 1, KERNEL_OBSERVE = 2 };

struct LaunchArgs {
    Params P;
    const void* src;
    void* dst;          // KERNEL_STEP / KERNEL_COLLIDE_LOCAL
    bool post;          // KERNEL_OBSERVE: rebuild from a POST buffer
    double* f_out;      // KERNEL_OBSERVE: optional f64 populations
    void* rho;          // optional readback (double for f64 storage, float otherwise)
    void* u;
    double* partials;   // optional per-block conservation partials (grid x 5)
    const double* prev_partials;  // with partials: block 0 also reduces these prev_count rows
    int prev_count;               // (the previous launch's partials) into prev_sums
    double* prev_sums;
    int first;          // KERNEL_OBSERVE: cell window [first, first + count);
    int count;          // count < 0: all cells
    int block;
    int vec;            // cells per thread of KERNEL_STEP (1, or 2 for ModeFast with nz even)
    cudaStream_t stream;
    int* grid_used;     // optional: receives the launched grid size (partial rows written)
    int tma_grid;       // > 0: KERNEL_STEP runs the TMA-staged kernel with this grid
    TileCfg tile;
    int pipe_grid = 0;  // > 0: a 16-bit two-cell KERNEL_STEP without outputs runs
                        // k_step2_pipe with this grid
    int sums_grid = 0;  // > 0: a two-cell KERNEL_STEP with partials runs
                        // k_step2_sums with this grid
    // vec == 4 steps without outputs: the rule quads, stepped by k_step4's
    // leading blocks
    const int* rule_quads = nullptr;  // QUAD_KINDS lists of n / 4 entries
    int rule_counts[QUAD_KINDS] = {0, 0, 0};
    int rules_grid = 0;  // leading blocks (0: one task per thread)
};

// Output selection of a step launch (OUT_* bits of lbm_kernels.cuh) from the
// optional pointers: rho/u and partials are mutually exclusive for steps.
inline int out_bits(const LaunchArgs& a) { return (a.rho ? 1 : 0) | (a.partials ? 2 : 0); }

inline int grid_for(long long work, int block) { return (int)((work + block - 1) / block); }

// Stateful engine kernels.
cudaError_t launch_exact(int kernel, int force_mode, const LaunchArgs& a);
cudaError_t launch_fast(int storage, int kernel, int force_mode, const LaunchArgs& a);
// Grids of the grid-stride two-cell kernels for this storage / force model /
// block size on the current device (resident blocks per SM x SMs); 0 where
// the kernel does not apply.  k_step2_pipe: f16 / bf16; k_step2_sums: f32 /
// f16 / bf16.
int pipe_grid_fast(int storage, int force_mode, int block);
int sums_grid_fast(int storage, int force_mode, int block);
cudaError_t launch_store_f64(int storage, const Params& P, const double* f, void* dst, cudaStream_t s);
cudaError_t launch_load_f64(int storage, const Params& P, const void* src, double* f, cudaStream_t s);
cudaError_t launch_feq_init(int storage, const Params& P, const double* rho, const double* u, void* dst,
                            cudaStream_t s);
cudaError_t launch_mark_near_solid(const Params& P, uint8_t* flags, uint32_t* bbmask, cudaStream_t s);
// The quads of a lattice (nz a multiple of 4) that k_step4's plain path
// leaves to its leading blocks, by kind into lists + kind * cap (in no
// order); their numbers into counts[QUAD_KINDS] (device).
cudaError_t launch_list_rule_quads(const Params& P, int* lists, int cap, int* counts, cudaStream_t s);
// Params::order for items of vec (1 or 2) cells; *face_count (device)
// receives the number of items on the walled faces.
cudaError_t launch_face_order(const Params& P, int vec, int* order, int* face_count, cudaStream_t s);
cudaError_t launch_reduce_partials(const double* partials, int nblocks, double* out5, cudaStream_t s);
// Tier-1 / Tier-2 diagnostics of f64 rho (n) / u (3, n) device arrays into
// out6 (device): {check_health, rho_min, rho_max, u_max_lat,
// check_divergence_free, check_circulation}; scratch: DIAG_SCRATCH doubles.
constexpr int DIAG_MAX_BLOCKS = 1184;
constexpr size_t DIAG_SCRATCH = (size_t)DIAG_MAX_BLOCKS * 6;
cudaError_t launch_diagnostics(const Params& P, const double* rho, const double* u, double dx_phys, double* scratch,
                               double* out6, cudaStream_t s);
// x-slab exchange: plane (plane_off bytes into each direction, plane_bytes
// long, directions dir_stride bytes apart) of the directions in mask to
// (get) or from the packed buffer, one launch.
cudaError_t launch_plane_copy(void* base, size_t dir_stride, size_t plane_off, size_t plane_bytes, uint32_t mask,
                              void* buf, bool get, cudaStream_t s);

// Batched step (one launch for many lattices): records and items in device
// memory, see lbm_batch.cuh.  `records` points to BatchLattice<T> for the
// storage's element type.
// sched: BatchSched (the pair schedules need f32/f16/bf16 storage and the
// force-free or uniform force model); collide != 0 runs the in-place collide
// of the first step, with items of `span` cells.
cudaError_t launch_batch_step(int storage, int force_mode, int sched, bool collide, const void* records,
                              const void* items, int nitems, int span, int phase, int grid, int block,
                              cudaStream_t s);
size_t batch_record_bytes(int storage);

// `steps` steps from POST in one cooperative launch (k_step_persistent;
// a.src / a.dst: the buffers of the first step, which alternate).  The grid
// is every block that fits on the device at once; a barrier wait gives up
// after timeout_ns (raising *a.P.err), and `missing` arrivals are added to
// the expected count (nonzero only to test that path).  *grid_out: the grid.
cudaError_t launch_persistent(int storage, int force_mode, const LaunchArgs& a, int steps, GridBarrier* bar,
                              unsigned missing, unsigned long long timeout_ns, int* grid_out);

// The cooperative launch of k_step_persistent<M, FM, VEC> (see launch_persistent).
template <class M, int FM, int VEC>
inline cudaError_t persistent_t(const LaunchArgs& a, int steps, GridBarrier* bar, unsigned missing,
                         unsigned long long timeout_ns, int* grid_out)
{
    using T = typename M::T;
    auto kern = k_step_persistent<M, FM, VEC>;
    const int block = 256;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    const int items = VEC == 2 ? a.P.n / 2 : a.P.n;
    int grid = sms * per_sm;
    const int need = (items + block - 1) / block;
    if (grid > need) grid = need;  // no block without work
    Params P = a.P;
    Streams<T> S0 = make_streams<T>(a.src, a.dst, a.P.n);
    Streams<T> S1 = make_streams<T>(a.dst, const_cast<void*>(a.src), a.P.n);
    unsigned expected = (unsigned)grid + missing;
    void* args[] = {&P, &S0, &S1, &steps, &bar, &expected, &timeout_ns};
    if ((e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), a.stream)) != cudaSuccess) return e;
    e = cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(block), args, 0, a.stream);
    if (grid_out) *grid_out = grid;
    return e;
}

// TMA-staged step (lbm_tma.cu): tile plan for a lattice (stages == 0 when the
// path does not apply) and the launch.
TileCfg plan_tma(int storage, int nx, int ny, int nz, int* grid, int device);
cudaError_t launch_tma_step(int storage, int force_mode, const LaunchArgs& a);

// Adjoint (lbm_adjoint.cu): one level over n cells.  Lambda buffers are
// (19, n) of adjoint_elem_bytes(storage) elements (double for f64 storage,
// float otherwise); level: AdjointLevel of lbm_adjoint.cuh.
struct AdjointArgs {
    Params P;
    const void* src;         // stored state of the level
    const void* Lin;         // Lambda_{k+1}
    void* Lout;              // Lambda_k
    const double* grad_rho;  // INIT seeds (nullable)
    const double* grad_u;
    double* dalpha;          // accumulated dL/dalpha (nullable)
    double* grad_f0;         // FINAL: dL/df_0 (nullable)
    const int* special;      // the cells k_adjoint_special handles (launch_list_special)
    int n_special;
    cudaStream_t stream;
    cudaStream_t special_stream;  // where k_adjoint_special runs (NULL: stream); the
                                  // caller orders the two (they touch disjoint cells)
};
cudaError_t launch_adjoint_level(int storage, int force_mode, int level, const AdjointArgs& a);
size_t adjoint_elem_bytes(int storage);
// Compact the special cells of a lattice into list (capacity n), *count on the device.
cudaError_t launch_list_special(const Params& P, int* list, int* count, cudaStream_t s);
cudaError_t launch_widen(const float* in, double* out, size_t count, cudaStream_t s);
cudaError_t launch_check_unit_interval(const float* a, int n, int* flag, cudaStream_t s);

// Record the calling thread's error message (lbm_last_error) and return code.
int set_error(int code, const char* message);

// Stateless reference functions (f64, bit-exact), device pointers.
cudaError_t ref_feq_field(const Params& P, const double* rho, const double* u, double* feq, cudaStream_t s);
cudaError_t ref_density(const Params& P, const double* f, double* rho, cudaStream_t s);
cudaError_t ref_momentum(const Params& P, const double* f, double* mom, cudaStream_t s);
cudaError_t ref_macro_velocity(const Params& P, const double* f, const double* force, double* u,
                               cudaStream_t s);
cudaError_t ref_stream(const Params& P, const double* fin, double* fout, cudaStream_t s);
cudaError_t ref_bgk_step(const Params& P, const double* f, const double* force, double* fout, cudaStream_t s);
cudaError_t ref_bounce_y(const Params& P, const double* f, double* fout, cudaStream_t s);

}  // namespace lbm
