/*
 * lbm_oracle.c -- CPU oracle for the D3Q19 BGK lattice-Boltzmann hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file:
 * only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and
 * the --impl reference arm) load it, as the checker and as the CPU baseline.
 *
 * Two layers:
 *
 * 1. Reference-exact f64 functions.  A plain-C restatement of the Stack-E
 *    Warp module packages/lattice-boltzmann-d3q19-stack-e/
 *    lattice_boltzmann_d3q19_stack_e/reference/d3q19_warp.py (kernels
 *    :87-212, host glue :253-415), whose arithmetic is byte-identical to the
 *    Phase-1 NumPy module packages/lattice-boltzmann-d3q19/
 *    lattice_boltzmann_d3q19/reference/{bgk.py,equilibrium.py}.  Every
 *    floating-point operation is issued in the reference's order; the file
 *    is compiled with -ffp-contract=off so no FMA is formed.  Pinned
 *    bit-exactly against golden vectors produced by the NumPy reference.
 *
 * 2. A generalised step ("engine") with the boundary semantics the reference
 *    lacks (flag grid with solid / inflow / outflow cells, walls on any
 *    non-periodic domain face, porosity drag, reduced-precision storage).
 *    With only the y axis walled and no flags it reduces exactly to
 *    bgk_step followed by apply_bounce_back_y_walls; beyond that the rules
 *    are this project's own and parity with the reference is unpinned.
 *
 * Threading: loops over x planes are OpenMP-parallel; every cell's result
 * depends only on the inputs, so the output is independent of thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define Q 19

/* Lex D3Q19 velocity order: constants.py:27-47 (VELOCITIES). */
static const int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
/* Opposite map: d3q19_warp.py:61-64 (_OPP). */
static const int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

static double W[Q];
static double CS2, INV_CS2, INV_CS4, INV_TWO_CS4, INV_TWO_CS2;
static int g_init = 0;

/* constants.py:50-57 (WEIGHTS, CS2) and d3q19_warp.py:51-54 (host reciprocals). */
static void init_constants(void)
{
    if (g_init) return;
    volatile double one = 1.0, three = 3.0, eighteen = 18.0, thirtysix = 36.0, two = 2.0;
    W[0] = one / three;
    for (int i = 1; i <= 6; ++i) W[i] = one / eighteen;
    for (int i = 7; i < Q; ++i) W[i] = one / thirtysix;
    CS2 = one / three;
    INV_CS2 = one / CS2;
    INV_CS4 = one / (CS2 * CS2);
    INV_TWO_CS4 = one / (two * CS2 * CS2);
    INV_TWO_CS2 = one / (two * CS2);
    g_init = 1;
}

void orc_constants(double* w19, double* cs)
{
    init_constants();
    for (int i = 0; i < Q; ++i) w19[i] = W[i];
    cs[0] = CS2; cs[1] = INV_CS2; cs[2] = INV_CS4; cs[3] = INV_TWO_CS4; cs[4] = INV_TWO_CS2;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

static inline int64_t cidx(int x, int y, int z, int ny, int nz)
{
    return ((int64_t)x * ny + y) * nz + z;
}

static inline int wrap(int v, int n)
{
    /* Positive modulus, d3q19_warp.py:209-211. */
    return ((v % n) + n) % n;
}

/* np.maximum(rho, 1e-30): NaN propagates (bgk.py:73). */
static inline double rho_safe(double r)
{
    if (isnan(r)) return r;
    return r > 1e-30 ? r : 1e-30;
}

/* ------------------------------------------------------------------------- */
/* Layer 1: reference-exact f64 functions                                     */
/* ------------------------------------------------------------------------- */

/* feq_field: equilibrium.py:295-322 == d3q19_warp.py:87-108 (reciprocal form). */
void orc_feq_field(const double* rho, const double* u, double* feq, int nx, int ny, int nz)
{
    init_constants();
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double ux = u[c], uy = u[n + c], uz = u[2 * n + c];
        double usq = ux * ux + uy * uy + uz * uz;
        double r = rho[c];
        for (int d = 0; d < Q; ++d) {
            double cu = (double)CX[d] * ux + (double)CY[d] * uy + (double)CZ[d] * uz;
            feq[d * n + c] = W[d] * r * (1.0 + cu * INV_CS2 + cu * cu * INV_TWO_CS4 - usq * INV_TWO_CS2);
        }
    }
}

/* density_field: d3q19_warp.py:111-120 (lex sum seeded 0.0). */
void orc_density_field(const double* f, double* rho, int nx, int ny, int nz)
{
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double acc = 0.0;
        for (int d = 0; d < Q; ++d) acc = acc + f[d * n + c];
        rho[c] = acc;
    }
}

/* momentum_field: d3q19_warp.py:123-140. */
void orc_momentum_field(const double* f, double* mom, int nx, int ny, int nz)
{
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double mx = 0.0, my = 0.0, mz = 0.0;
        for (int d = 0; d < Q; ++d) {
            double fd = f[d * n + c];
            mx = mx + (double)CX[d] * fd;
            my = my + (double)CY[d] * fd;
            mz = mz + (double)CZ[d] * fd;
        }
        mom[c] = mx; mom[n + c] = my; mom[2 * n + c] = mz;
    }
}

/* macroscopic_velocity: d3q19_warp.py:371-383 ((m [+ 0.5 F]) / max(rho, 1e-30)). */
void orc_macroscopic_velocity(const double* f, const double* force, double* u, int nx, int ny, int nz)
{
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double r = 0.0, m[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < Q; ++d) {
            double fd = f[d * n + c];
            r = r + fd;
            m[0] = m[0] + (double)CX[d] * fd;
            m[1] = m[1] + (double)CY[d] * fd;
            m[2] = m[2] + (double)CZ[d] * fd;
        }
        double rs = rho_safe(r);
        for (int a = 0; a < 3; ++a) {
            double ma = m[a];
            if (force) ma = ma + 0.5 * force[a * n + c];
            u[a * n + c] = ma / rs;
        }
    }
}

/*
 * Per-cell BGK collision with optional Guo forcing, reference operation order.
 * force == NULL: the NumPy force-free path (bgk.py:72-85, no Guo term).
 * force != NULL: d3q19_warp.py:156-195 (== bgk.py:81-110 with a force array).
 */
static inline void collide_exact(const double* f, double* out, const double* F, double tau)
{
    double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    for (int d = 0; d < Q; ++d) {
        double fd = f[d];
        r = r + fd;
        mx = mx + (double)CX[d] * fd;
        my = my + (double)CY[d] * fd;
        mz = mz + (double)CZ[d] * fd;
    }
    double rs = rho_safe(r);
    double ux, uy, uz;
    if (F) {
        ux = mx / rs + 0.5 * F[0] / rs;
        uy = my / rs + 0.5 * F[1] / rs;
        uz = mz / rs + 0.5 * F[2] / rs;
    } else {
        ux = mx / rs; uy = my / rs; uz = mz / rs;
    }
    double usq = ux * ux + uy * uy + uz * uz;
    double pref = 1.0 - 0.5 / tau;
    for (int d = 0; d < Q; ++d) {
        double cd0 = (double)CX[d], cd1 = (double)CY[d], cd2 = (double)CZ[d];
        double cu = cd0 * ux + cd1 * uy + cd2 * uz;
        double feq = W[d] * r * (1.0 + cu * INV_CS2 + cu * cu * INV_TWO_CS4 - usq * INV_TWO_CS2);
        double fd = f[d];
        double relaxed = fd - (fd - feq) / tau;
        if (F) {
            double tx = (cd0 - ux) * INV_CS2 + cu * cd0 * INV_CS4;
            double ty = (cd1 - uy) * INV_CS2 + cu * cd1 * INV_CS4;
            double tz = (cd2 - uz) * INV_CS2 + cu * cd2 * INV_CS4;
            double force_i = pref * W[d] * (tx * F[0] + ty * F[1] + tz * F[2]);
            out[d] = relaxed + force_i;
        } else {
            out[d] = relaxed;
        }
    }
}

/* _k_collide_guo over a whole lattice: d3q19_warp.py:143-195. */
void orc_collide(const double* f, double* fpost, const double* force, double tau, int nx, int ny, int nz)
{
    init_constants();
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double fl[Q], o[Q], F[3];
        for (int d = 0; d < Q; ++d) fl[d] = f[d * n + c];
        if (force) { F[0] = force[c]; F[1] = force[n + c]; F[2] = force[2 * n + c]; }
        collide_exact(fl, o, force ? F : NULL, tau);
        for (int d = 0; d < Q; ++d) fpost[d * n + c] = o[d];
    }
}

/* _k_stream: d3q19_warp.py:198-212 (out[d,x] = in[d, (x - c_d) mod n]). */
void orc_stream(const double* fin, double* fout, int nx, int ny, int nz)
{
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z)
                for (int d = 0; d < Q; ++d) {
                    int sx = wrap(x - CX[d], nx), sy = wrap(y - CY[d], ny), sz = wrap(z - CZ[d], nz);
                    fout[d * n + cidx(x, y, z, ny, nz)] = fin[d * n + cidx(sx, sy, sz, ny, nz)];
                }
}

/* bgk_step: collide then stream (d3q19_warp.py:321-368). */
void orc_bgk_step(const double* f, double* fout, double tau, const double* force, int nx, int ny, int nz)
{
    const int64_t n = (int64_t)nx * ny * nz;
    double* tmp = (double*)malloc(sizeof(double) * Q * n);
    orc_collide(f, tmp, force, tau, nx, ny, nz);
    orc_stream(tmp, fout, nx, ny, nz);
    free(tmp);
}

/* rho_wall = sum_d f[d] of one wall cell.  bgk.py:203/:212 reduce with
 * NumPy's f[:, :, y, :].sum(axis=0): lex order when a wall row holds several
 * cells, but NumPy's 8-accumulator pairwise order when the row is a single
 * cell (nx * nz == 1) and the reduction runs along the direction axis. */
static inline double wall_sum(const double* g, int pairwise)
{
    if (!pairwise) {
        double r = 0.0;
        for (int d = 0; d < Q; ++d) r = r + g[d];
        return r;
    }
    double a[8];
    for (int j = 0; j < 8; ++j) a[j] = g[j];
    for (int j = 0; j < 8; ++j) a[j] = a[j] + g[8 + j];
    double r = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    for (int d = 16; d < Q; ++d) r = r + g[d];
    return r;
}

/* Moving-wall momentum injection, bgk.py:199-205 operation order:
 * ((-2.0 * W[i]) * rho_wall * ci_dot_uw) / CS2. */
static inline double wall_injection(int i, double rho_wall, const double* uw)
{
    double ci_dot_uw = (double)CX[i] * uw[0] + (double)CY[i] * uw[1] + (double)CZ[i] * uw[2];
    return -2.0 * W[i] * rho_wall * ci_dot_uw / CS2;
}

/* apply_bounce_back_y_walls: d3q19_warp.py:386-415 (== bgk.py:145-216). */
void orc_bounce_back_y_walls(const double* f, double* out, int nx, int ny, int nz,
                             const double* u_top, const double* u_bottom)
{
    init_constants();
    const int64_t n = (int64_t)nx * ny * nz;
    memcpy(out, f, sizeof(double) * Q * n);
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int z = 0; z < nz; ++z) {
            int64_t cb = cidx(x, 0, z, ny, nz), ct = cidx(x, ny - 1, z, ny, nz);
            double gb[Q], gt[Q];
            for (int d = 0; d < Q; ++d) { gb[d] = f[d * n + cb]; gt[d] = f[d * n + ct]; }
            const int pw = (int64_t)nx * nz == 1;
            double rb = wall_sum(gb, pw), rt = wall_sum(gt, pw);
            for (int i = 0; i < Q; ++i) {
                if (CY[i] > 0) out[i * n + cb] = f[OPP[i] * n + cb] + wall_injection(i, rb, u_bottom);
                if (CY[i] < 0) out[i * n + ct] = f[OPP[i] * n + ct] + wall_injection(i, rt, u_top);
            }
        }
}

/* ------------------------------------------------------------------------- */
/* Layer 2: generalised step (project semantics; unpinned beyond y walls)     */
/* ------------------------------------------------------------------------- */

enum { CELL_FLUID = 0, CELL_SOLID = 1, CELL_INFLOW = 2, CELL_OUTFLOW = 3 };
enum { FORCE_NONE = 0, FORCE_UNIFORM = 1, FORCE_FIELD = 2, FORCE_DRAG = 3 };
enum { STORE_F64 = 0, STORE_F32 = 1, STORE_F16_SHIFT = 2, STORE_BF16_SHIFT = 3 };
/* Face order: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+.  A direction whose source
 * lies beyond several walled faces takes the first face in this priority. */
static const int FACE_PRIORITY[6] = {3, 2, 0, 1, 4, 5};

typedef struct {
    int32_t nx, ny, nz;
    int32_t periodic;          /* bit 0 x, bit 1 y, bit 2 z */
    int32_t force_mode;
    int32_t storage;
    double tau;
    double wall_u[6][3];
    double body_force[3];
    double drag_k;
    double inflow_rho;
    double inflow_u[3];
    const uint8_t* flags;      /* (n) cell types, or NULL = all fluid */
    const double* force;       /* (3, n) for FORCE_FIELD */
    const float* porosity;     /* (n) for FORCE_DRAG */
    double storage_ref_u[3];   /* 16-bit storage reference velocity */
} orc_lattice;

/* IEEE binary16 / bfloat16 round-to-nearest-even conversions (bit-level). */
static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

uint16_t orc_f32_to_f16(float f)
{
    uint32_t x = f2u(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t absx = x & 0x7fffffffu;
    if (absx >= 0x7f800000u) {                  /* inf or nan */
        if (absx > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);
        return (uint16_t)(sign | 0x7c00u);
    }
    if (absx >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* rounds to >= 65520 -> inf */
    int e = (int)(absx >> 23) - 127;
    uint32_t mant = (absx & 0x7fffffu) | 0x800000u;
    if (e < -24) {
        /* below half the smallest subnormal: 0, except exactly-above-half handled below */
        if (e < -25 || absx == 0) return (uint16_t)sign;
    }
    if (e >= -14) {
        /* normal half: keep 10 mantissa bits, round the 13 dropped bits */
        uint32_t rem = absx & 0x1fffu;
        uint32_t h = (uint32_t)(((e + 15) << 10) | ((absx >> 13) & 0x3ffu));
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1;
        return (uint16_t)(sign | h);
    }
    /* subnormal half: value = mant * 2^(e-23) = units * 2^-24, so
     * units = mant >> (-e - 1), rounded half to even */
    int shift = -e - 1;
    uint32_t units = mant >> shift;
    uint32_t rem = mant & ((1u << shift) - 1u);
    uint32_t half = 1u << (shift - 1);
    if (rem > half || (rem == half && (units & 1u))) units += 1;
    return (uint16_t)(sign | units);
}

float orc_f16_to_f32(uint16_t h)
{
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t e = ((uint32_t)h >> 10) & 0x1fu;
    uint32_t m = (uint32_t)h & 0x3ffu;
    if (e == 0x1f) return u2f(sign | 0x7f800000u | (m << 13));
    if (e == 0) {
        if (m == 0) return u2f(sign);
        /* subnormal: m * 2^-24 */
        float v = (float)m * 5.9604644775390625e-08f;
        return sign ? -v : v;
    }
    return u2f(sign | ((e + 112u) << 23) | (m << 13));
}

uint16_t orc_f32_to_bf16(float f)
{
    uint32_t x = f2u(f);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
    uint32_t lsb = (x >> 16) & 1u;
    x += 0x7fffu + lsb;
    return (uint16_t)(x >> 16);
}

float orc_bf16_to_f32(uint16_t b) { return u2f((uint32_t)b << 16); }

/* 16-bit storage shift of each direction: (float)(feq_d(1, ref_u) - w_d),
 * reciprocal form (the GPU's Params::shift_h); zero for the other storages. */
static void storage_shift(int storage, const double* ref_u, float* sh)
{
    const int s16 = storage == STORE_F16_SHIFT || storage == STORE_BF16_SHIFT;
    const double rx = ref_u ? ref_u[0] : 0.0, ry = ref_u ? ref_u[1] : 0.0, rz = ref_u ? ref_u[2] : 0.0;
    const double r_sq = rx * rx + ry * ry + rz * rz;
    for (int d = 0; d < Q; ++d) {
        double cu = (double)CX[d] * rx + (double)CY[d] * ry + (double)CZ[d] * rz;
        double feq = W[d] * 1.0 * (1.0 + cu * INV_CS2 + cu * cu * INV_TWO_CS4 - r_sq * INV_TWO_CS2);
        sh[d] = s16 ? (float)(feq - W[d]) : 0.0f;
    }
}

/* Round a population value to what the storage format can hold.  The 16-bit
 * formats hold the binary16 / bfloat16 rounding of the f32 number
 * (float)(v - w_d) - sh_d and read back as w_d + ((float)stored + sh_d). */
static inline double store_round(int storage, float sh, int d, double v)
{
    switch (storage) {
    case STORE_F32: return (double)(float)v;
    case STORE_F16_SHIFT: {
        float dev = (float)(v - W[d]) - sh;
        return W[d] + (double)(orc_f16_to_f32(orc_f32_to_f16(dev)) + sh);
    }
    case STORE_BF16_SHIFT: {
        float dev = (float)(v - W[d]) - sh;
        return W[d] + (double)(orc_bf16_to_f32(orc_f32_to_bf16(dev)) + sh);
    }
    default: return v;
    }
}

void orc_store_round(int storage, const double* ref_u, double* f, int64_t n)
{
    init_constants();
    float sh[Q];
    storage_shift(storage, ref_u, sh);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c)
        for (int d = 0; d < Q; ++d) f[d * n + c] = store_round(storage, sh[d], d, f[d * n + c]);
}

static inline int cell_type(const orc_lattice* L, int64_t c)
{
    return L->flags ? (L->flags[c] & 3) : CELL_FLUID;
}

/* The rest state w_d a solid cell stands for, as the arithmetic sees it (f32
 * storage: w_d in f32; the deviation storages: a zero deviation). */
static inline double solid_value(const orc_lattice* L, int d)
{
    return L->storage == STORE_F32 ? (double)(float)W[d] : W[d];
}

static void feq_point(double rho, const double* u, double* out)
{
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int d = 0; d < Q; ++d) {
        double cu = (double)CX[d] * u[0] + (double)CY[d] * u[1] + (double)CZ[d] * u[2];
        out[d] = W[d] * rho * (1.0 + cu * INV_CS2 + cu * cu * INV_TWO_CS4 - usq * INV_TWO_CS2);
    }
}

/*
 * Post-stream (pre-collision) state of the cell at (gx,gy,gz) of type gtype,
 * from the stored post-collision array P.
 *   raw gather g[i] = P[i][(g - c_i) mod dims]  (reference streaming)
 *   walled face crossed by g - c_i:  f[i] = g[opp(i)] + injection(face, rho_w)
 *       rho_w = sum_d g[d] (reference apply_bounce_back_y_walls rule)
 *   source cell solid:               f[i] = P[opp(i)][g]  (half-way bounce-back)
 *   otherwise                        f[i] = g[i]
 * Inflow cells take feq(inflow_rho, inflow_u); solid cells their stored rest value.
 */
static void post_stream_state(const orc_lattice* L, const double* P, int gx, int gy, int gz, int gtype,
                              double* f)
{
    const int nx = L->nx, ny = L->ny, nz = L->nz;
    const int64_t n = (int64_t)nx * ny * nz;
    if (gtype == CELL_INFLOW) { feq_point(L->inflow_rho, L->inflow_u, f); return; }
    if (gtype == CELL_SOLID) { for (int d = 0; d < Q; ++d) f[d] = solid_value(L, d); return; }
    double g[Q];
    int face[Q];
    int any_face = 0;
    int64_t src[Q];
    for (int d = 0; d < Q; ++d) {
        int sx = gx - CX[d], sy = gy - CY[d], sz = gz - CZ[d];
        int crossed[6] = {0, 0, 0, 0, 0, 0};
        if (!(L->periodic & 1)) { crossed[0] = sx < 0; crossed[1] = sx >= nx; }
        if (!(L->periodic & 2)) { crossed[2] = sy < 0; crossed[3] = sy >= ny; }
        if (!(L->periodic & 4)) { crossed[4] = sz < 0; crossed[5] = sz >= nz; }
        face[d] = -1;
        for (int k = 0; k < 6; ++k)
            if (crossed[FACE_PRIORITY[k]]) { face[d] = FACE_PRIORITY[k]; break; }
        if (face[d] >= 0) any_face = 1;
        src[d] = cidx(wrap(sx, nx), wrap(sy, ny), wrap(sz, nz), ny, nz);
        g[d] = P[d * n + src[d]];
    }
    double rho_w = 0.0;
    if (any_face) rho_w = wall_sum(g, (int64_t)nx * nz == 1);
    const int64_t gc = cidx(gx, gy, gz, ny, nz);
    for (int d = 0; d < Q; ++d) {
        if (face[d] >= 0) {
            f[d] = g[OPP[d]] + wall_injection(d, rho_w, L->wall_u[face[d]]);
        } else if (L->flags && (L->flags[src[d]] & 3) == CELL_SOLID) {
            f[d] = P[OPP[d] * n + gc];
        } else {
            f[d] = g[d];
        }
    }
}

/* Position and type whose post-stream state cell (x,y,z) takes: outflow
 * cells copy their x-1 neighbour (zero-gradient); an outflow neighbour is
 * treated as fluid. */
static void gather_site(const orc_lattice* L, int x, int y, int z, int* gx, int* gtype)
{
    int t = cell_type(L, cidx(x, y, z, L->ny, L->nz));
    if (t == CELL_OUTFLOW) {
        int xm = wrap(x - 1, L->nx);
        int tn = cell_type(L, cidx(xm, y, z, L->ny, L->nz));
        *gx = xm;
        *gtype = tn == CELL_OUTFLOW ? CELL_FLUID : tn;
    } else {
        *gx = x;
        *gtype = t;
    }
}

/* Force acting at cell c given the post-stream momentum m. */
static inline void cell_force(const orc_lattice* L, int64_t c, int64_t n, const double* m, double* F)
{
    switch (L->force_mode) {
    case FORCE_UNIFORM:
        F[0] = L->body_force[0]; F[1] = L->body_force[1]; F[2] = L->body_force[2];
        break;
    case FORCE_FIELD:
        F[0] = L->force[c]; F[1] = L->force[n + c]; F[2] = L->force[2 * n + c];
        break;
    case FORCE_DRAG: {
        double ka = L->drag_k * (double)L->porosity[c];
        double beta = ka / (1.0 + 0.5 * ka);
        F[0] = L->body_force[0] - beta * m[0];
        F[1] = L->body_force[1] - beta * m[1];
        F[2] = L->body_force[2] - beta * m[2];
        break;
    }
    default:
        F[0] = F[1] = F[2] = 0.0;
    }
}

static inline void moments(const double* f, double* r, double* m)
{
    double rr = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    for (int d = 0; d < Q; ++d) {
        double fd = f[d];
        rr = rr + fd;
        mx = mx + (double)CX[d] * fd;
        my = my + (double)CY[d] * fd;
        mz = mz + (double)CZ[d] * fd;
    }
    *r = rr; m[0] = mx; m[1] = my; m[2] = mz;
}

/* Readback of one cell's state: rho = sum f, u = (m + 0.5 F) / max(rho,1e-30);
 * solid cells read back rho = 0, u = 0. */
static inline void readback(const orc_lattice* L, int64_t c, int64_t n, int type, const double* f,
                            double* rho, double* u)
{
    if (type == CELL_SOLID) {
        rho[c] = 0.0; u[c] = 0.0; u[n + c] = 0.0; u[2 * n + c] = 0.0;
        return;
    }
    double r, m[3], F[3];
    moments(f, &r, m);
    double rs = rho_safe(r);
    rho[c] = r;
    if (L->force_mode == FORCE_NONE) {
        for (int a = 0; a < 3; ++a) u[a * n + c] = m[a] / rs;
    } else {
        cell_force(L, c, n, m, F);
        for (int a = 0; a < 3; ++a) u[a * n + c] = (m[a] + 0.5 * F[a]) / rs;
    }
}

static inline void collide_cell(const orc_lattice* L, int64_t c, int64_t n, const double* f, double* out)
{
    if (L->force_mode == FORCE_NONE) {
        collide_exact(f, out, NULL, L->tau);
    } else {
        double r, m[3], F[3];
        moments(f, &r, m);
        cell_force(L, c, n, m, F);
        collide_exact(f, out, F, L->tau);
    }
}

/* PRE state -> stored post-collision array: P = round(C(f)); solid cells get
 * their rest value.  rho/u (optional) receive the readback of f. */
void orc_engine_collide_local(const orc_lattice* L, const double* f, double* P, double* rho, double* u)
{
    init_constants();
    float sh[Q];
    storage_shift(L->storage, L->storage_ref_u, sh);
    const int nx = L->nx, ny = L->ny, nz = L->nz;
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        int t = cell_type(L, c);
        double fl[Q], o[Q];
        for (int d = 0; d < Q; ++d) fl[d] = f[d * n + c];
        if (rho) readback(L, c, n, t, fl, rho, u);
        if (t == CELL_SOLID) {
            for (int d = 0; d < Q; ++d) P[d * n + c] = solid_value(L, d);
            continue;
        }
        collide_cell(L, c, n, fl, o);
        for (int d = 0; d < Q; ++d) P[d * n + c] = store_round(L->storage, sh[d], d, o[d]);
    }
}

/* One fused step on the stored post-collision array: Pout = round(C(B(G(Pin)))).
 * rho/u (optional) receive the readback of the reconstructed pre-collision state. */
void orc_engine_step(const orc_lattice* L, const double* Pin, double* Pout, double* rho, double* u)
{
    init_constants();
    float sh[Q];
    storage_shift(L->storage, L->storage_ref_u, sh);
    const int nx = L->nx, ny = L->ny, nz = L->nz;
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int64_t c = cidx(x, y, z, ny, nz);
                int t = cell_type(L, c);
                double f[Q], o[Q];
                if (t == CELL_SOLID) {
                    for (int d = 0; d < Q; ++d) Pout[d * n + c] = Pin[d * n + c];
                    if (rho) { rho[c] = 0.0; u[c] = u[n + c] = u[2 * n + c] = 0.0; }
                    continue;
                }
                int gx, gt;
                gather_site(L, x, y, z, &gx, &gt);
                post_stream_state(L, Pin, gx, y, z, gt, f);
                if (rho) readback(L, c, n, t, f, rho, u);
                collide_cell(L, c, n, f, o);
                for (int d = 0; d < Q; ++d) Pout[d * n + c] = store_round(L->storage, sh[d], d, o[d]);
            }
}

/* Pre-collision state f_n reconstructed from the stored array; readback optional. */
void orc_engine_reconstruct(const orc_lattice* L, const double* P, double* f, double* rho, double* u)
{
    init_constants();
    const int nx = L->nx, ny = L->ny, nz = L->nz;
    const int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int64_t c = cidx(x, y, z, ny, nz);
                int t = cell_type(L, c);
                double fl[Q];
                if (t == CELL_SOLID) {
                    for (int d = 0; d < Q; ++d) fl[d] = solid_value(L, d);
                } else {
                    int gx, gt;
                    gather_site(L, x, y, z, &gx, &gt);
                    post_stream_state(L, P, gx, y, z, gt, fl);
                }
                if (f) for (int d = 0; d < Q; ++d) f[d * n + c] = fl[d];
                if (rho) readback(L, c, n, t, fl, rho, u);
            }
}

/* Readback of a PRE-state array (f held directly). */
void orc_engine_moments_local(const orc_lattice* L, const double* f, double* rho, double* u)
{
    init_constants();
    const int64_t n = (int64_t)L->nx * L->ny * L->nz;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < n; ++c) {
        double fl[Q];
        for (int d = 0; d < Q; ++d) fl[d] = f[d * n + c];
        readback(L, c, n, cell_type(L, c), fl, rho, u);
    }
}

/* Advance n_steps from a PRE state f (in/out): f <- B(G(round(C(f)))).
 * Convenience for the CPU baseline; uses two scratch arrays. */
int orc_engine_run(const orc_lattice* L, double* f, int n_steps)
{
    init_constants();
    const int64_t n = (int64_t)L->nx * L->ny * L->nz;
    if (n_steps <= 0) return 0;
    double* a = (double*)malloc(sizeof(double) * Q * n);
    double* b = (double*)malloc(sizeof(double) * Q * n);
    if (!a || !b) { free(a); free(b); return -1; }
    orc_engine_collide_local(L, f, a, NULL, NULL);
    for (int s = 1; s < n_steps; ++s) {
        orc_engine_step(L, a, b, NULL, NULL);
        double* t = a; a = b; b = t;
    }
    orc_engine_reconstruct(L, a, f, NULL, NULL);
    free(a); free(b);
    return 0;
}

/* FP64 conservation sums over non-solid cells of a PRE-state array:
 * out = {sum rho, sum m_x, sum m_y, sum m_z}, cell order, lex moments. */
void orc_conservation(const orc_lattice* L, const double* f, double* out)
{
    const int64_t n = (int64_t)L->nx * L->ny * L->nz;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t c = 0; c < n; ++c) {
        if (cell_type(L, c) == CELL_SOLID) continue;
        double fl[Q], r, m[3];
        for (int d = 0; d < Q; ++d) fl[d] = f[d * n + c];
        moments(fl, &r, m);
        s[0] += r; s[1] += m[0]; s[2] += m[1]; s[3] += m[2];
    }
    for (int k = 0; k < 4; ++k) out[k] = s[k];
}
