/*
 * lbm_d3q19.h -- C ABI of the B200 D3Q19 BGK lattice-Boltzmann engine
 * (liblbm_d3q19.so, built from bit-physics_b200/csrc).
 *
 * Conventions
 *   - Every function returns int status: LBM_OK (0) or a negative LBM_ERR_*
 *     code; lbm_last_error() gives the calling thread's last message.  No
 *     function aborts the process.
 *   - Population arrays are structure-of-arrays f64 (19, nx, ny, nz), C order
 *     (x slowest, z fastest), direction index in the reference's lex D3Q19
 *     order (0 rest; 1-6 +-x,+-y,+-z; 7-10 xy; 11-14 xz; 15-18 yz).
 *     rho is (nx, ny, nz); u and force fields are (3, nx, ny, nz).
 *   - Host pointers are borrowed for the duration of the call.  A handle owns
 *     its device memory.  Handles are not thread-safe: one thread per handle.
 *
 * Reference interface replaced (Bit-Physics, package
 * packages/lattice-boltzmann-d3q19-stack-e/lattice_boltzmann_d3q19_stack_e/):
 * the Python surface re-exported by reference/__init__.py:12-68 and the
 * evolve loops of sim.py:119-190.  Each declaration cites the function it
 * stands in for.
 */
#ifndef LBM_D3Q19_H
#define LBM_D3Q19_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define LBM_OK 0
#define LBM_ERR_INVALID (-1)     /* bad argument (shape, pointer, tau <= 0.5, ...) */
#define LBM_ERR_CUDA (-2)        /* CUDA runtime error (message in lbm_last_error) */
#define LBM_ERR_NOMEM (-3)       /* device or host allocation failed */
#define LBM_ERR_STATE (-4)       /* call not valid in the handle's current state */
#define LBM_ERR_NONFINITE (-5)   /* health check found a non-finite density */
#define LBM_ERR_UNSUPPORTED (-6) /* combination not implemented */
#define LBM_ERR_NO_DEVICE (-7)   /* no CUDA device / driver */

/* ---- storage formats of the population arrays on the device ------------ */
#define LBM_STORAGE_F64 0        /* f64, reference operation order (bit-exact)   */
#define LBM_STORAGE_F32 1        /* f32 populations, f32 arithmetic               */
#define LBM_STORAGE_F16_SHIFT 2  /* binary16 f_i - feq_i(1, storage_ref_u) (f_i - w_i
                                    by default), f32 arithmetic                     */
#define LBM_STORAGE_BF16_SHIFT 3 /* bfloat16, the same deviation, f32 arithmetic  */

/* ---- periodicity bits; a non-periodic axis has two walled faces -------- */
#define LBM_PERIODIC_X 1
#define LBM_PERIODIC_Y 2
#define LBM_PERIODIC_Z 4

/* ---- domain faces (index into lbm_desc.wall_velocity) ------------------ */
#define LBM_FACE_XM 0
#define LBM_FACE_XP 1
#define LBM_FACE_YM 2 /* the reference's bottom wall, y = 0      */
#define LBM_FACE_YP 3 /* the reference's top wall,    y = ny - 1 */
#define LBM_FACE_ZM 4
#define LBM_FACE_ZP 5

/* ---- cell types of the flag grid (uint8, one per cell) ----------------- */
#define LBM_CELL_FLUID 0
#define LBM_CELL_SOLID 1   /* static obstacle, half-way bounce-back            */
#define LBM_CELL_INFLOW 2  /* post-stream state := feq(inflow_rho, inflow_u)   */
#define LBM_CELL_OUTFLOW 3 /* post-stream state := that of cell (x-1, y, z)    */

/* ---- body-force models -------------------------------------------------- */
#define LBM_FORCE_NONE 0    /* force-free collision (bgk.py:72-85 path)          */
#define LBM_FORCE_UNIFORM 1 /* F = body_force in every cell (Guo forcing)        */
#define LBM_FORCE_FIELD 2   /* F from a per-cell (3, n) field (lbm_set_force_field) */
#define LBM_FORCE_DRAG 3    /* F = body_force - beta(alpha) m, porosity alpha    */

typedef struct lbm_desc {
    int32_t nx, ny, nz;
    int32_t storage;     /* LBM_STORAGE_*                                    */
    int32_t periodic;    /* LBM_PERIODIC_* bits; default all periodic        */
    int32_t force_mode;  /* LBM_FORCE_*                                      */
    double tau;          /* BGK relaxation time, > 0.5                       */
    double wall_velocity[6][3]; /* per face, used where the axis is walled   */
    double body_force[3];
    double drag_k;       /* drag coefficient k for LBM_FORCE_DRAG            */
    double inflow_rho;   /* inflow cell density (default 1)                  */
    double inflow_u[3];  /* inflow cell velocity                             */
    int32_t device;      /* CUDA device ordinal                              */
    int32_t block_size;  /* threads per block for the step kernels; 0 = auto */
    int32_t cells_per_thread; /* step kernel: 1; 2 (f32/f16/bf16 storage,
                                 nz even); 4 (f16/bf16 storage, nz a
                                 multiple of 4, register staging); 0 = auto */
    int32_t staging;     /* step kernel input staging: LBM_STAGING_*         */
    double storage_ref_u[3]; /* f16/bf16 storage: populations are held as the
                                16-bit deviation from feq(1, storage_ref_u)
                                (default 0: f - w_i); a reference velocity
                                near the flow's keeps the deviations small,
                                so the rounding error is small           */
} lbm_desc;

/* Step-kernel staging (lbm_desc.staging). */
#define LBM_STAGING_AUTO 0      /* the fastest measured: registers               */
#define LBM_STAGING_REGISTERS 1 /* loads straight into registers                  */
#define LBM_STAGING_TMA 2       /* TMA bulk copies into a shared-memory ring: two
                                   cells per thread, f32/f16/bf16 storage, nz even
                                   and nz * element size a multiple of 16 bytes   */
#define LBM_STAGING_PIPELINED 3 /* registers, with the next pair's loads issued
                                   before the current pair's collision (grid-stride
                                   loop): two cells per thread, f16/bf16 storage;
                                   steps with readback or sums run the two-cell
                                   kernel                                         */
#define LBM_STAGING_PERSISTENT 4 /* lbm_step runs all its steady-state steps in
                                    one cooperative launch, every block stepping
                                    its share of the cells and a grid barrier
                                    between steps (lattices that stay in L2, where
                                    a launch per step costs more than the step);
                                    loads of populations cached in L2 only       */

typedef struct lbm_lattice lbm_lattice;

/* Fill a descriptor with defaults: 1x1x1, f64, all periodic, tau 1, no force. */
int lbm_desc_init(lbm_desc* desc);

/* ---- stateful engine ----------------------------------------------------
 * Replaces the evolve loop of sim.py:119-190: state stays resident on the
 * GPU; each step is one fused pull-stream + boundary + collide kernel. */

/* Create a lattice handle; populations start at the rest equilibrium w_i. */
int lbm_create(const lbm_desc* desc, lbm_lattice** out);
int lbm_destroy(lbm_lattice* h);
/* Use a caller-owned cudaStream_t (NULL: the handle's own stream). */
int lbm_set_stream(lbm_lattice* h, void* cuda_stream);
int lbm_synchronize(lbm_lattice* h);

/* State in / out: stands in for the f array that the reference's loop
 * carries between bgk_step and apply_bounce_back_y_walls (sim.py:140-142). */
int lbm_set_populations(lbm_lattice* h, const double* f);
int lbm_get_populations(lbm_lattice* h, double* f);
/* Set f = feq(rho, u) on the device; rho may be NULL (1) and u NULL (0).
 * Stands in for feq_field + the initial state (sim.py:112-116). */
int lbm_set_equilibrium(lbm_lattice* h, const double* rho, const double* u);

/* Boundary and forcing inputs. */
int lbm_set_flags(lbm_lattice* h, const uint8_t* flags);     /* NULL clears */
int lbm_set_force_field(lbm_lattice* h, const double* force); /* (3, n)     */
int lbm_set_porosity(lbm_lattice* h, const float* alpha);     /* (n), [0,1] */
int lbm_set_tau(lbm_lattice* h, double tau);
int lbm_set_wall_velocity(lbm_lattice* h, int32_t face, const double* u3);
int lbm_set_body_force(lbm_lattice* h, const double* f3);

/* Advance n_steps: bgk_step + apply_bounce_back_y_walls per step
 * (d3q19_warp.py:321-368, :386-415), generalised to the flag grid. */
int lbm_step(lbm_lattice* h, int32_t n_steps);
int64_t lbm_step_count(const lbm_lattice* h);

/* One step split over several launches (no reference counterpart: the
 * reference steps one whole lattice per call).  lbm_step_planes advances
 * the x-planes [x_begin, x_end) of the current step into the next state;
 * lbm_step_commit ends the step and makes the next state current.  Until the
 * commit the current state is the step's source: readbacks and
 * lbm_plane_get / lbm_plane_put act on it (a halo plane filled by
 * lbm_plane_put before the planes next to it are advanced is what they
 * pull), and calls that change the state or the parameters return
 * LBM_ERR_STATE.  Planes left out hold unspecified values after the
 * commit.  Needs a stepped state (LBM_ERR_STATE right after a state upload:
 * take that step with lbm_step).  Runs the register-staged kernel of the
 * lattice's storage and cells per thread on its stream: the advanced planes
 * are bit-identical to lbm_step's result under automatic, register or
 * pipelined staging. */
int lbm_step_planes(lbm_lattice* h, int32_t x_begin, int32_t x_end);
int lbm_step_commit(lbm_lattice* h);

/* Four-cell lattices (16-bit storage, nz % 4 == 0): the quads that need a
 * boundary rule are stepped by the leading blocks of each step launch.
 * lbm_set_rule_blocks fixes their number (0: sized from the rule-quad count,
 * the default); lbm_get_rule_blocks reports it and the number of rule quads.
 * Results do not depend on it.  LBM_ERR_STATE for other lattices. */
int lbm_set_rule_blocks(lbm_lattice* h, int32_t blocks);
int lbm_get_rule_blocks(const lbm_lattice* h, int32_t* blocks, int32_t* rule_quads);

/* rho and u of the current state: density_field + macroscopic_velocity
 * (d3q19_warp.py:283-292, :371-383).  Either pointer may be NULL. */
int lbm_get_rho_u(lbm_lattice* h, double* rho, double* u);

/* Run n_steps and read back rho/u every `every` steps, plus the start and
 * final states (sim.py:140-153 with capture_interval = every).  Frame k
 * holds step k*every (the last frame step n_steps).  rho_frames holds
 * n_frames*n, u_frames n_frames*3n doubles, n_frames = n_steps/every + 1
 * (+1 when every does not divide n_steps). */
int lbm_run_capture(lbm_lattice* h, int32_t n_steps, int32_t every, double* rho_frames,
                    double* u_frames);

/* Advance n_steps and return, per step, the FP64 sums {sum rho, sum m_x,
 * sum m_y, sum m_z} over non-solid cells of the state that step advanced
 * from (sums: n_steps x 4 doubles).  The sums are reduced on the GPU inside
 * the step kernels and copied to the host once, after the last step: the
 * global mass / momentum drift check of a run (sim.py:89-96 health check). */
int lbm_step_monitor(lbm_lattice* h, int32_t n_steps, double* sums);

/* FP64 sums over non-solid cells of the current state:
 * out = {sum rho, sum m_x, sum m_y, sum m_z}. */
int lbm_conservation(lbm_lattice* h, double* out4);

/* Stateful health check: LBM_ERR_NONFINITE if any density is non-finite
 * (the check_health diagnostic of sim.py:89-96). */
int lbm_check_health(lbm_lattice* h);

/* ---- stateless functions on host arrays ---------------------------------
 * Same inputs, outputs and arithmetic as the reference's pure functions
 * (f64, bit-exact); data is copied to the GPU and back on every call. */
int lbm_feq_field(const double* rho, const double* u, double* feq, int32_t nx, int32_t ny,
                  int32_t nz);                                        /* d3q19_warp.py:253 */
int lbm_density_field(const double* f, double* rho, int32_t nx, int32_t ny,
                      int32_t nz);                                    /* d3q19_warp.py:283 */
int lbm_momentum_field(const double* f, double* mom, int32_t nx, int32_t ny,
                       int32_t nz);                                   /* d3q19_warp.py:295 */
int lbm_macroscopic_velocity(const double* f, const double* force, double* u, int32_t nx,
                             int32_t ny, int32_t nz);                 /* d3q19_warp.py:371 */
int lbm_stream(const double* f_post, double* f_out, int32_t nx, int32_t ny,
               int32_t nz);                                           /* d3q19_warp.py:308 */
int lbm_bgk_step(const double* f, double* f_out, double tau, const double* force, int32_t nx,
                 int32_t ny, int32_t nz);                             /* d3q19_warp.py:321 */
int lbm_bounce_back_y_walls(const double* f, double* f_out, int32_t nx, int32_t ny, int32_t nz,
                            const double* wall_velocity_top,
                            const double* wall_velocity_bottom);      /* d3q19_warp.py:386 */

/* ---- the same functions on device pointers (no copies; stream may be NULL) */
int lbm_feq_field_dev(const double* rho, const double* u, double* feq, int32_t nx, int32_t ny,
                      int32_t nz, void* stream);
int lbm_density_field_dev(const double* f, double* rho, int32_t nx, int32_t ny, int32_t nz,
                          void* stream);
int lbm_momentum_field_dev(const double* f, double* mom, int32_t nx, int32_t ny, int32_t nz,
                           void* stream);
int lbm_macroscopic_velocity_dev(const double* f, const double* force, double* u, int32_t nx,
                                 int32_t ny, int32_t nz, void* stream);
int lbm_stream_dev(const double* f_post, double* f_out, int32_t nx, int32_t ny, int32_t nz,
                   void* stream);
int lbm_bgk_step_dev(const double* f, double* f_out, double tau, const double* force, int32_t nx,
                     int32_t ny, int32_t nz, void* stream);
int lbm_bounce_back_y_walls_dev(const double* f, double* f_out, int32_t nx, int32_t ny,
                                int32_t nz, const double* wall_velocity_top,
                                const double* wall_velocity_bottom, void* stream);

/* ---- batches: many independent lattices, one launch per step -----------
 * The batched ensemble the reference does not have: lattices of different
 * sizes and parameters (same storage and force model) advanced together by
 * one persistent kernel launch per step, replayed from a CUDA graph.  Each
 * lattice is an ordinary handle (lbm_batch_lattice) for state transfer and
 * readback; the batch owns them and their stream. */
typedef struct lbm_batch lbm_batch;

#define LBM_SCHED_SINGLE 0      /* one cell per thread                              */
#define LBM_SCHED_PAIR_SCALAR 1 /* two cells per thread, f32x2 collision            */
#define LBM_SCHED_PAIR_MIXED 2  /* as 1, vector memory access where nz is even      */
#define LBM_SCHED_BRANCHES 3    /* no batched kernel: every lattice's own step
                                   kernels on `grid` parallel streams (0: 8),
                                   largest lattices first, each to the stream with
                                   the fewest cells; two steps per captured graph  */

int lbm_batch_create(const lbm_desc* descs, int32_t count, lbm_batch** out);
int lbm_batch_destroy(lbm_batch* b);
int lbm_batch_count(const lbm_batch* b);
/* Borrowed handle of lattice i (valid until lbm_batch_destroy). */
int lbm_batch_lattice(lbm_batch* b, int32_t i, lbm_lattice** out);
/* Work schedule: sched LBM_SCHED_*, threads per block (multiple of 32, <= 256),
 * grid = blocks of the persistent launch (0: 4 per SM); for
 * LBM_SCHED_BRANCHES grid is the number of streams (<= 64) and block is
 * unused. */
int lbm_batch_set_schedule(lbm_batch* b, int32_t sched, int32_t block, int32_t grid);
int lbm_batch_get_schedule(const lbm_batch* b, int32_t* sched, int32_t* block, int32_t* grid);
/* Advance every lattice n_steps: one launch per step (LBM_SCHED_BRANCHES:
 * one graph of per-lattice launches per two steps), steady-state steps
 * replayed from a captured two-step CUDA graph. */
int lbm_batch_step(lbm_batch* b, int32_t n_steps);
/* The same with one launch per lattice and step (for comparison). */
int lbm_batch_step_unbatched(lbm_batch* b, int32_t n_steps);
/* Time every schedule on trial_steps steps, keep the fastest (ms per step in
 * *best_ms); the lattices' states are saved before and restored after. */
int lbm_batch_autotune(lbm_batch* b, int32_t trial_steps, double* best_ms);
int lbm_batch_synchronize(lbm_batch* b);

/* ---- device-pointer transfers (for callers whose fields live on the GPU) --
 * rho (n) and u (3, n) of the current state as f64 into device memory,
 * enqueued on the lattice's stream (either pointer may be NULL). */
int lbm_get_rho_u_dev(lbm_lattice* h, double* rho, double* u);
/* lbm_set_porosity from device memory (n floats in [0, 1], checked). */
int lbm_set_porosity_dev(lbm_lattice* h, const float* alpha);

/* ---- x-slab decomposition --------------------------------------------------
 * No counterpart in the reference (single-device).  A lattice split in x over
 * several handles (x-slabs with one halo plane per side, periodic in x)
 * exchanges, before each step, the populations that cross a slab face: plane
 * x of the stored array (after a step: the post-collision populations) for
 * the directions in dir_mask (bit d = direction d), to / from a device buffer
 * of popcount(dir_mask) * ny * nz storage elements, direction-major in
 * increasing d.  Enqueued on the lattice's stream. */
int lbm_plane_get(lbm_lattice* h, int32_t x, uint32_t dir_mask, void* dst);
int lbm_plane_put(lbm_lattice* h, int32_t x, uint32_t dir_mask, const void* src);
/* FP64 {sum rho, sum m} over the cells of the x-planes [x0, x1) (a slab's
 * owned planes); as lbm_conservation otherwise. */
int lbm_conservation_planes(lbm_lattice* h, int32_t x0, int32_t x1, double* out4);

/* ---- adjoint: gradients through taped steps -------------------------------
 * The differentiable run the reference does not have (its Warp kernels are
 * not taped).  lbm_tape_forward runs n_steps from the lattice's current PRE
 * state (populations set by lbm_set_populations / lbm_set_equilibrium /
 * lbm_set_flags and not stepped since), exactly as lbm_step would, and keeps
 * a copy of the state every checkpoint_every steps plus the final one.
 * lbm_tape_backward takes the gradient of a loss L(rho_N, u_N) of the final
 * readback -- dL/drho (n) and dL/du (3, n), f64 device arrays, either may be
 * NULL for zero -- and runs the discrete adjoint of every step back to the
 * start, recomputing the states between checkpoints with the step kernels.
 * Outputs (f64 device arrays, overwritten; either may be NULL):
 *   grad_alpha (n)     dL/dalpha for the drag model (zero for other models)
 *   grad_f0 (19, n)    dL/df_0 of the initial populations
 * The tape borrows the lattice: the lattice must outlive it, and a backward
 * after a change of the lattice's flags, fields or parameters returns
 * LBM_ERR_STATE.  Work is enqueued on the lattice's stream. */
typedef struct lbm_tape lbm_tape;
int lbm_tape_forward(lbm_lattice* h, int32_t n_steps, int32_t checkpoint_every, lbm_tape** out);
int lbm_tape_backward(lbm_tape* t, const double* grad_rho, const double* grad_u, double* grad_alpha,
                      double* grad_f0);
/* Device bytes the tape holds (checkpoints, segment states, adjoint fields). */
int64_t lbm_tape_bytes(const lbm_tape* t);
int lbm_tape_destroy(lbm_tape* t);

/* Tier-1 / Tier-2 diagnostics of the current state, reduced on the GPU
 * (replaces the NumPy diagnostics of Stack-E sim.py:89-109 after a full host
 * readback): out6 = {check_health (0 all finite, 1 otherwise), rho_min,
 * rho_max, u_max_lat = max |u|, check_divergence_free = max |div u| on the
 * z = 0 slice by periodic central differences with spacing dx_phys,
 * check_circulation = sum of u_x over that slice * dx_phys^2}, of the rho /
 * u that lbm_get_rho_u would return (solid cells read back as 0).  Equal to
 * the reference's expressions on those arrays bit for bit, except the
 * circulation sum's order of summation. */
int lbm_diagnostics(lbm_lattice* h, double dx_phys, double* out6);

/* ---- 16-bit moment-encoded state ---------------------------------------
 * The frontier variant's compressed state (packages/lattice-boltzmann-d3q19-
 * frontier-moment-encoded/src/lbm_me.cpp:71-138, :212-250): 19 monomial
 * moments per cell (m = M f) quantised to 16 bits over per-moment ranges
 * [lo_k, hi_k], code = round((m - lo) / (hi - lo) * 65535) clamped.
 * lbm_moment16_basis: M and M^-1 (19 x 19, row-major; either may be NULL).
 * lbm_moment16_calibrate: run n_steps on h (f64 or f32 storage) and return
 * the envelope of every post-collision state's moments over the non-solid
 * cells, each range widened by margin * its span on both sides.
 * lbm_moment16_step: advance an f32 lattice n_steps with the persistent
 * state held as moment codes: each step decodes the codes, runs the fused
 * step and encodes its result; afterwards the lattice holds the decoded
 * codes (readbacks and later steps see the encoded state).  No counterpart
 * in the reference's Stack-E API. */
int lbm_moment16_basis(double* m_out, double* minv_out);
int lbm_moment16_calibrate(lbm_lattice* h, int32_t n_steps, double margin, double* lo, double* hi);
int lbm_moment16_step(lbm_lattice* h, const double* lo, const double* hi, int32_t n_steps);

/* Test hook of the persistent step's bounded grid barrier: the next
 * cooperative launches of h expect `missing_arrivals` more blocks than they
 * launch (so no barrier opens) and give up each wait after timeout_ns
 * (<= 0: the default, 2 s).  The launch then ends by itself with the error
 * word raised; lbm_synchronize reports LBM_ERR_CUDA and the state is
 * invalid until new populations are set.  (0, 0) restores the defaults. */
int lbm_test_barrier_limit(lbm_lattice* h, int32_t missing_arrivals, int64_t timeout_ns);

/* ---- without device allocation ----------------------------------------- */
/* No counterpart in the reference.  FP64 sums {sum rho, sum m_x, sum m_y,
 * sum m_z} of a population array f (19, nx, ny, nz, f64, device memory) over
 * its non-solid cells (flags: optional device uint8 cell types), written to
 * out4 (4 doubles, device memory), enqueued on `stream` (NULL: the legacy
 * default stream).  f, flags and out4 must be device memory of the current
 * GPU (LBM_ERR_INVALID otherwise).  The result is bit-identical to
 * lbm_conservation of an f64 lattice with the default block size holding f
 * as its uploaded state (same 128-cell blocks, same reduction order), and
 * equal up to FP64 rounding for other block sizes.  It allocates nothing: its
 * scratch is one fixed device array per GPU, for callers that cannot call
 * cudaMalloc where they need the sums (another allocator owns the device
 * memory, or a step loop must not be stalled by an allocation).  At most
 * LBM_NOALLOC_MAX_CELLS cells; calls that overlap on one GPU race on the
 * shared array.  The first call on a device loads the module that holds the
 * array and should come before any stream capture. */
#define LBM_NOALLOC_MAX_CELLS 16777216LL
int lbm_conservation_noalloc(const double* f, const uint8_t* flags, int32_t nx, int32_t ny, int32_t nz,
                             double* out4, void* stream);

/* ---- library ------------------------------------------------------------ */
const char* lbm_last_error(void);
int lbm_version(void);
/* Number of visible CUDA devices (0 when there is no driver or device). */
int lbm_device_count(void);
/* Release the device workspace that the host-array functions cache. */
int lbm_release_workspace(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_D3Q19_H */
