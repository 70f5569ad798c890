/*
 * fdtd_oracle.c -- CPU restatement of DeepGPR's differentiable Maxwell FDTD
 * path, used ONLY as the parity checker for the CUDA library.
 *
 * TEST INFRASTRUCTURE.  Nothing in the product (deepgpr_b200/) links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg do.
 *
 * It exports the same ABI-6 entry points as the reference CPU backend
 * (src/DeepGPR/lib/deepgpr.h:89-152) so both libraries can be driven with the
 * identical argument list and compared bit for bit.  The arithmetic follows
 * the reference step by step (operation order included), restated here as a
 * per-cell "base update + CPML correction" pass:
 *
 *   coefficients        src/DeepGPR/lib/deepgpr_cpu.c:547-584
 *   staggered stencils  src/DeepGPR/lib/deepgpr_cpu.c:287-407
 *   E / H updates       src/DeepGPR/lib/deepgpr_cpu.c:670-717, 886-933
 *   CPML E / H          src/DeepGPR/lib/deepgpr_cpu.c:722-883, 939-1100
 *   sources, receivers  src/DeepGPR/lib/deepgpr_cpu.c:600-668, 1479-1534
 *   histories           src/DeepGPR/lib/deepgpr_cpu.c:1559-1633
 *   imaging condition   src/DeepGPR/lib/deepgpr_cpu.c:1659-1745
 *   adjoint E / H       src/DeepGPR/lib/deepgpr_cpu.c:1112-1459, 409-527
 *   drivers             src/DeepGPR/lib/deepgpr_cpu.c:1782-1934, 1975-2111
 *
 * Reorganisation relative to the reference (result-preserving): the CPML
 * correction of a cell is applied right after that cell's base update (no
 * other cell reads the corrected value inside the same half step), and the
 * adjoint keeps only the CPML part of the transposed-curl weights in scratch;
 * the interior part (coefficient * lambda) is recomputed at gather time.
 * Both evaluate the same floating-point expressions in the same order.
 *
 * Build: see oracle/Makefile (gcc -std=c99 -O3, no FMA contraction).
 */
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_API __attribute__((visibility("default")))

/* Constants of the reference header (src/DeepGPR/lib/deepgpr.h:21-33). */
static const float kEps0 = 8.8541878128e-12f;
static const float kMu0 = 1.25663706212e-06f;
static const float kPecSigma = 100.0f;

/* storage_type bits (src/DeepGPR/config/constants.py:128-187). */
#define ST_KIND_MASK 0x0f
#define ST_F32 0
#define ST_F16 1
#define ST_BF16 2
#define ST_RHS_FROM_E (1 << 4)
#define ST_PHYSICAL (1 << 5)
#define ST_DISABLED (1 << 26)

static __thread char g_error[512];

static void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

ORACLE_API int deepgpr_supports_error_reporting(void) { return 1; }
ORACLE_API const char* deepgpr_last_error(void) { return g_error; }
ORACLE_API void deepgpr_clear_last_error(void) { g_error[0] = '\0'; }
ORACLE_API int deepgpr_deterministic_adjoint(void) { return 1; }
ORACLE_API int deepgpr_abi_version(void) { return 6; }
ORACLE_API int deepgpr_supports_external_pml(void) { return 1; }
ORACLE_API int deepgpr_supports_pml_material_gradients(void) { return 1; }
ORACLE_API int deepgpr_supports_rhs_reconstruction(void) { return 1; }
ORACLE_API int deepgpr_supports_physical_history(void) { return 1; }

static int g_order = 2;
ORACLE_API void set_fdtd_order(int order) { g_order = (order == 4 || order == 8) ? order : 2; }

/* ------------------------------------------------------------------------ */
/* 16-bit history encodings: IEEE round-to-nearest-even.                     */
/* ------------------------------------------------------------------------ */

static uint16_t enc_f16(float v)
{
    uint32_t x;
    memcpy(&x, &v, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ex = (x >> 23) & 0xffu;
    uint32_t man = x & 0x7fffffu;
    if (ex == 0xffu) return (uint16_t)(sign | (man ? 0x7e00u : 0x7c00u));
    int e = (int)ex - 112; /* rebias 127 -> 15 */
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t full = man | 0x800000u;
        int sh = 14 - e;
        uint32_t q = full >> sh;
        uint32_t rem = full & ((1u << sh) - 1u);
        uint32_t half = 1u << (sh - 1);
        if (rem > half || (rem == half && (q & 1u))) q += 1u;
        return (uint16_t)(sign | q);
    }
    uint32_t q = ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q += 1u; /* carries into the exponent */
    if ((q >> 10) >= 31u) return (uint16_t)(sign | 0x7c00u);
    return (uint16_t)(sign | q);
}

static float dec_f16(uint16_t h)
{
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t ex = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    float out;
    if (ex == 0) {
        out = ldexpf((float)man, -24);
        uint32_t b;
        memcpy(&b, &out, 4);
        b |= sign;
        memcpy(&out, &b, 4);
        return out;
    }
    uint32_t b = ex == 0x1fu ? (sign | 0x7f800000u | (man << 13)) : (sign | ((ex + 112u) << 23) | (man << 13));
    memcpy(&out, &b, 4);
    return out;
}

static uint16_t enc_bf16(float v)
{
    uint32_t x;
    memcpy(&x, &v, 4);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u); /* quiet NaN */
    uint32_t lsb = (x >> 16) & 1u;
    x += 0x7fffu + lsb;
    return (uint16_t)(x >> 16);
}

static float dec_bf16(uint16_t h)
{
    uint32_t b = (uint32_t)h << 16;
    float out;
    memcpy(&out, &b, 4);
    return out;
}

static size_t kind_bytes(int kind) { return kind == ST_F32 ? 4u : 2u; }

static void hist_put(void* base, long long i, float v, int kind)
{
    if (kind == ST_F16) ((uint16_t*)base)[i] = enc_f16(v);
    else if (kind == ST_BF16) ((uint16_t*)base)[i] = enc_bf16(v);
    else ((float*)base)[i] = v;
}

static float hist_get(const void* base, long long i, int kind)
{
    if (kind == ST_F16) return dec_f16(((const uint16_t*)base)[i]);
    if (kind == ST_BF16) return dec_bf16(((const uint16_t*)base)[i]);
    return ((const float*)base)[i];
}

static const void* hist_at(const void* base, long long elems, int kind)
{
    return (const void*)((const unsigned char*)base + elems * (long long)kind_bytes(kind));
}

/* ------------------------------------------------------------------------ */
/* Grid description and staggered stencils.                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
    int NX, NY, NZ;      /* field extents = extended cells + 1 (Yee halo) */
    long long sy, sx;    /* element strides of the y and x axes */
    long long cells;     /* NX * NY * NZ (one shot) */
    int nshot;
    float dx, dy, dz;
    int R;               /* requested stencil radius 1, 2 or 4 */
    int p[6];            /* CPML thickness x0, xm, y0, ym, z0, zm */
} Geom;

static int radius_of(int order) { return order >= 8 ? 4 : (order >= 4 ? 2 : 1); }

/* Coefficient r (1-based) of the staggered stencil of radius `rad`
 * (src/DeepGPR/lib/deepgpr_cpu.c:271-289). */
static float taps(int rad, int r)
{
    static const float t4[4] = {1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f, -5.0f / 7168.0f};
    static const float t3[3] = {75.0f / 64.0f, -25.0f / 384.0f, 3.0f / 640.0f};
    static const float t2[2] = {9.0f / 8.0f, -1.0f / 24.0f};
    if (rad >= 4) return t4[r - 1];
    if (rad == 3) return t3[r - 1];
    if (rad == 2) return t2[r - 1];
    return 1.0f;
}

/* Radius actually usable at `c` on an axis of `n` points (deepgpr_cpu.c:329-353). */
static int rad_back(long long c, long long n, int R)
{
    int r = R;
    while (r > 1 && (c < r || c + r - 1 >= n)) --r;
    return r;
}

static int rad_fwd(long long c, long long n, int R)
{
    int r = R;
    while (r > 1 && (c - r + 1 < 0 || c + r >= n)) --r;
    return r;
}

/* Backward difference: sum_r a_r (f[c+(r-1)] - f[c-r]). */
static float d_back(const float* f, long long id, long long s, long long c, long long n, int R)
{
    if (R == 1) return f[id] - f[id - s];
    int rr = rad_back(c, n, R);
    float acc = 0.0f;
    for (int r = 1; r <= rr; ++r)
        acc += taps(rr, r) * (f[id + (long long)(r - 1) * s] - f[id - (long long)r * s]);
    return acc;
}

/* Forward difference: sum_r a_r (f[c+r] - f[c-(r-1)]). */
static float d_fwd(const float* f, long long id, long long s, long long c, long long n, int R)
{
    if (R == 1) return f[id + s] - f[id];
    int rr = rad_fwd(c, n, R);
    float acc = 0.0f;
    for (int r = 1; r <= rr; ++r)
        acc += taps(rr, r) * (f[id + (long long)r * s] - f[id - (long long)(r - 1) * s]);
    return acc;
}

/* Weight of a transposed-curl channel at a source point, supplied by caller. */
typedef float (*WeightFn)(const void* ctx, long long id);

/* Transpose of d_back gathered at target t (deepgpr_cpu.c:429-467). */
static float t_back(WeightFn w, const void* ctx, long long t, long long s, long long c, long long n, int R)
{
    if (R == 1) {
        float acc = w(ctx, t);
        if (c + 1 < n) acc -= w(ctx, t + s);
        return acc;
    }
    float acc = 0.0f;
    if (c >= 2 * R - 1 && c + 2 * R - 1 < n) {
        for (int r = 1; r <= R; ++r) {
            float a = taps(R, r);
            acc += a * w(ctx, t - (long long)(r - 1) * s);
            acc -= a * w(ctx, t + (long long)r * s);
        }
        return acc;
    }
    for (int r = 1; r <= R; ++r) {
        long long up = c - (r - 1);
        if (up >= 0) {
            int rr = rad_back(up, n, R);
            if (r <= rr) acc += taps(rr, r) * w(ctx, t - (long long)(r - 1) * s);
        }
        long long dn = c + r;
        if (dn < n) {
            int rr = rad_back(dn, n, R);
            if (r <= rr) acc -= taps(rr, r) * w(ctx, t + (long long)r * s);
        }
    }
    return acc;
}

/* Transpose of d_fwd gathered at target t (deepgpr_cpu.c:470-507). */
static float t_fwd(WeightFn w, const void* ctx, long long t, long long s, long long c, long long n, int R)
{
    if (R == 1) {
        float acc = 0.0f;
        if (c >= 1) acc += w(ctx, t - s);
        acc -= w(ctx, t);
        return acc;
    }
    float acc = 0.0f;
    if (c >= 2 * R - 1 && c + 2 * R <= n) {
        for (int r = 1; r <= R; ++r) {
            float a = taps(R, r);
            acc += a * w(ctx, t - (long long)r * s);
            acc -= a * w(ctx, t + (long long)(r - 1) * s);
        }
        return acc;
    }
    for (int r = 1; r <= R; ++r) {
        long long up = c - r;
        if (up >= 0) {
            int rr = rad_fwd(up, n, R);
            if (r <= rr) acc += taps(rr, r) * w(ctx, t - (long long)r * s);
        }
        long long dn = c + (r - 1);
        if (dn < n) {
            int rr = rad_fwd(dn, n, R);
            if (r <= rr) acc -= taps(rr, r) * w(ctx, t + (long long)(r - 1) * s);
        }
    }
    return acc;
}

/* Which Yee components the base update advances (deepgpr_cpu.c:697-699, 913-915). */
static int upd_ex(const Geom* g, long long i, long long j, long long k)
{
    return (g->NY - 1 != 1 || g->NZ - 1 != 1) && i < g->NX - 1 && j > 0 && j < g->NY - 1 && k > 0 && k < g->NZ - 1;
}
static int upd_ey(const Geom* g, long long i, long long j, long long k)
{
    return (g->NX - 1 != 1 || g->NZ - 1 != 1) && i > 0 && i < g->NX - 1 && j < g->NY - 1 && k > 0 && k < g->NZ - 1;
}
static int upd_ez(const Geom* g, long long i, long long j, long long k)
{
    return (g->NX - 1 != 1 || g->NY - 1 != 1) && i > 0 && i < g->NX - 1 && j > 0 && j < g->NY - 1 && k < g->NZ - 1;
}
static int upd_hx(const Geom* g, long long i, long long j, long long k)
{
    return g->NX - 1 != 1 && i > 0 && i < g->NX - 1 && j < g->NY - 1 && k < g->NZ - 1;
}
static int upd_hy(const Geom* g, long long i, long long j, long long k)
{
    return g->NY - 1 != 1 && i < g->NX - 1 && j > 0 && j < g->NY - 1 && k < g->NZ - 1;
}
static int upd_hz(const Geom* g, long long i, long long j, long long k)
{
    return g->NZ - 1 != 1 && i < g->NX - 1 && j < g->NY - 1 && k > 0 && k < g->NZ - 1;
}

/* ------------------------------------------------------------------------ */
/* CPML faces.                                                               */
/* ------------------------------------------------------------------------ */

/* One CPML face of one field (E or H): coefficients and its two psi arrays. */
typedef struct {
    const float* R; /* (4, p): RA, RB, RE, RF */
    float* psi1;
    float* psi2;
    int p;
} Face;

typedef struct {
    float ra1, rb, re, rf; /* RA - 1, RB, RE, RF */
} Prof;

static Prof prof_at(const Face* f, long long q)
{
    Prof pr;
    pr.ra1 = f->R[q] - 1.0f;
    pr.rb = f->R[f->p + q];
    pr.re = f->R[2 * f->p + q];
    pr.rf = f->R[3 * f->p + q];
    return pr;
}

/* Slab position q of a cell on each face, or -1 when outside.
 * E faces (deepgpr_cpu.c:754-760): x0 = 1..p, q = p - i; xm = n-1-p .. n-2.
 * H faces (deepgpr_cpu.c:965-971): x0 = 0..p-1, q = p - 1 - i.            */
static long long q_low_e(int p, long long c) { return (p > 0 && c > 0 && c <= p) ? p - c : -1; }
static long long q_low_h(int p, long long c) { return (p > 0 && c < p) ? p - 1 - c : -1; }
static long long q_high(int p, long long c, long long n) { return (p > 0 && c >= n - 1 - p && c < n - 1) ? c - (n - 1 - p) : -1; }

/* psi element index for each (face axis, psi slot, E/H) layout
 * (src/DeepGPR/solver/pml.py:310-348, deepgpr_cpu.c:773-878, 986-1096). */
typedef struct {
    long long a, b, c; /* extents of the three psi axes */
} Box3;

static long long at3(Box3 b, long long s, long long u, long long v, long long w)
{
    return ((s * b.a + u) * b.b + v) * b.c + w;
}

/* ------------------------------------------------------------------------ */
/* Forward half steps.                                                       */
/* ------------------------------------------------------------------------ */

typedef struct {
    float *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    const float *ce_hist, *ce_curl, *ce_rhs, *ch_hist, *ch_curl, *ch_rhs;
    Face eF[6], hF[6];
} State;

/* H half step: base update then CPML correction, one cell at a time. */
static void h_half_step(const Geom* g, State* st)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long s = w / g->cells, idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        const float* Ex = st->Ex; const float* Ey = st->Ey; const float* Ez = st->Ez;
        float hx = st->Hx[w], hy = st->Hy[w], hz = st->Hz[w];
        const float c0 = st->ch_hist[idx], c1 = st->ch_curl[idx];
        const float cy = g->dy == g->dx ? c1 : c1 * g->dx / g->dy;
        const float cz = g->dz == g->dx ? c1 : c1 * g->dx / g->dz;
        if (upd_hx(g, i, j, k)) {
            float a = d_fwd(Ez, w, NZ, j, NY, g->R), b = d_fwd(Ey, w, 1, k, NZ, g->R);
            hx = c0 * hx - cy * a + cz * b;
        }
        if (upd_hy(g, i, j, k)) {
            float a = d_fwd(Ex, w, 1, k, NZ, g->R), b = d_fwd(Ez, w, g->sx, i, NX, g->R);
            hy = c0 * hy - cz * a + c1 * b;
        }
        if (upd_hz(g, i, j, k)) {
            float a = d_fwd(Ey, w, g->sx, i, NX, g->R), b = d_fwd(Ex, w, NZ, j, NY, g->R);
            hz = c0 * hz - c1 * a + cy * b;
        }
        const float up = st->ch_rhs[idx];
        for (int f = 0; f < 6; ++f) {
            const Face* F = &st->hF[f];
            const int axis = f / 2;
            const long long c = axis == 0 ? i : (axis == 1 ? j : k);
            const long long n = axis == 0 ? NX : (axis == 1 ? NY : NZ);
            const long long q = (f % 2 == 0) ? q_low_h(F->p, c) : q_high(F->p, c, n);
            if (q < 0) continue;
            const Prof pr = prof_at(F, q);
            if (axis == 0) {
                if (k < NZ - 1) { /* psi1 -> Hy from dEz/dx */
                    Box3 b = {F->p, NY, NZ - 1};
                    long long pi = at3(b, s, q, j, k);
                    float d = d_fwd(Ez, w, g->sx, i, NX, g->R) / g->dx;
                    float ph = F->psi1[pi];
                    hy += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (j < NY - 1) { /* psi2 -> Hz from dEy/dx */
                    Box3 b = {F->p, NY - 1, NZ};
                    long long pi = at3(b, s, q, j, k);
                    float d = d_fwd(Ey, w, g->sx, i, NX, g->R) / g->dx;
                    float ph = F->psi2[pi];
                    hz -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            } else if (axis == 1) {
                if (k < NZ - 1) { /* psi1 -> Hx from dEz/dy */
                    Box3 b = {NX, F->p, NZ - 1};
                    long long pi = at3(b, s, i, q, k);
                    float d = d_fwd(Ez, w, NZ, j, NY, g->R) / g->dy;
                    float ph = F->psi1[pi];
                    hx -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (i < NX - 1) { /* psi2 -> Hz from dEx/dy */
                    Box3 b = {NX - 1, F->p, NZ};
                    long long pi = at3(b, s, i, q, k);
                    float d = d_fwd(Ex, w, NZ, j, NY, g->R) / g->dy;
                    float ph = F->psi2[pi];
                    hz += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            } else {
                if (j < NY - 1) { /* psi1 -> Hx from dEy/dz */
                    Box3 b = {NX, NY - 1, F->p};
                    long long pi = at3(b, s, i, j, q);
                    float d = d_fwd(Ey, w, 1, k, NZ, g->R) / g->dz;
                    float ph = F->psi1[pi];
                    hx += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (i < NX - 1) { /* psi2 -> Hy from dEx/dz */
                    Box3 b = {NX - 1, NY, F->p};
                    long long pi = at3(b, s, i, j, q);
                    float d = d_fwd(Ex, w, 1, k, NZ, g->R) / g->dz;
                    float ph = F->psi2[pi];
                    hy -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            }
        }
        st->Hx[w] = hx;
        st->Hy[w] = hy;
        st->Hz[w] = hz;
    }
}

/* E half step: base update then CPML correction, one cell at a time. */
static void e_half_step(const Geom* g, State* st)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long s = w / g->cells, idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        const float* Hx = st->Hx; const float* Hy = st->Hy; const float* Hz = st->Hz;
        float ex = st->Ex[w], ey = st->Ey[w], ez = st->Ez[w];
        const float c0 = st->ce_hist[idx], c1 = st->ce_curl[idx];
        const float cy = g->dy == g->dx ? c1 : c1 * g->dx / g->dy;
        const float cz = g->dz == g->dx ? c1 : c1 * g->dx / g->dz;
        if (upd_ex(g, i, j, k)) {
            float a = d_back(Hz, w, NZ, j, NY, g->R), b = d_back(Hy, w, 1, k, NZ, g->R);
            ex = c0 * ex + cy * a - cz * b;
        }
        if (upd_ey(g, i, j, k)) {
            float a = d_back(Hx, w, 1, k, NZ, g->R), b = d_back(Hz, w, g->sx, i, NX, g->R);
            ey = c0 * ey + cz * a - c1 * b;
        }
        if (upd_ez(g, i, j, k)) {
            float a = d_back(Hy, w, g->sx, i, NX, g->R), b = d_back(Hx, w, NZ, j, NY, g->R);
            ez = c0 * ez + c1 * a - cy * b;
        }
        const float up = st->ce_rhs[idx];
        for (int f = 0; f < 6; ++f) {
            const Face* F = &st->eF[f];
            const int axis = f / 2;
            const long long c = axis == 0 ? i : (axis == 1 ? j : k);
            const long long n = axis == 0 ? NX : (axis == 1 ? NY : NZ);
            const long long q = (f % 2 == 0) ? q_low_e(F->p, c) : q_high(F->p, c, n);
            if (q < 0 || c == 0) continue;
            const Prof pr = prof_at(F, q);
            if (axis == 0) {
                if (j < NY - 1) { /* psi1 -> Ey from dHz/dx */
                    Box3 b = {F->p + 1, NY - 1, NZ};
                    long long pi = at3(b, s, q, j, k);
                    float d = d_back(Hz, w, g->sx, i, NX, g->R) / g->dx;
                    float ph = F->psi1[pi];
                    ey -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (k < NZ - 1) { /* psi2 -> Ez from dHy/dx */
                    Box3 b = {F->p + 1, NY, NZ - 1};
                    long long pi = at3(b, s, q, j, k);
                    float d = d_back(Hy, w, g->sx, i, NX, g->R) / g->dx;
                    float ph = F->psi2[pi];
                    ez += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            } else if (axis == 1) {
                if (i < NX - 1) { /* psi1 -> Ex from dHz/dy */
                    Box3 b = {NX - 1, F->p + 1, NZ};
                    long long pi = at3(b, s, i, q, k);
                    float d = d_back(Hz, w, NZ, j, NY, g->R) / g->dy;
                    float ph = F->psi1[pi];
                    ex += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (k < NZ - 1) { /* psi2 -> Ez from dHx/dy */
                    Box3 b = {NX, F->p + 1, NZ - 1};
                    long long pi = at3(b, s, i, q, k);
                    float d = d_back(Hx, w, NZ, j, NY, g->R) / g->dy;
                    float ph = F->psi2[pi];
                    ez -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            } else {
                if (i < NX - 1) { /* psi1 -> Ex from dHy/dz */
                    Box3 b = {NX - 1, NY, F->p + 1};
                    long long pi = at3(b, s, i, j, q);
                    float d = d_back(Hy, w, 1, k, NZ, g->R) / g->dz;
                    float ph = F->psi1[pi];
                    ex -= up * (pr.ra1 * d + pr.rb * ph);
                    F->psi1[pi] = pr.re * ph - pr.rf * d;
                }
                if (j < NY - 1) { /* psi2 -> Ey from dHx/dz */
                    Box3 b = {NX, NY - 1, F->p + 1};
                    long long pi = at3(b, s, i, j, q);
                    float d = d_back(Hx, w, 1, k, NZ, g->R) / g->dz;
                    float ph = F->psi2[pi];
                    ey += up * (pr.ra1 * d + pr.rb * ph);
                    F->psi2[pi] = pr.re * ph - pr.rf * d;
                }
            }
        }
        st->Ex[w] = ex;
        st->Ey[w] = ey;
        st->Ez[w] = ez;
    }
}

/* ------------------------------------------------------------------------ */
/* Coefficients, sources and receivers.                                      */
/* ------------------------------------------------------------------------ */

static void build_coefficients(const Geom* g, const float* eps, const float* sig, const float* mu,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs, float dt)
{
    long long idx;
#pragma omp parallel for schedule(static)
    for (idx = 0; idx < g->cells; ++idx) {
        long long i = idx / g->sx, j = (idx % g->sx) / g->NZ, k = idx % g->NZ;
        if (i >= g->NX - 1 || j >= g->NY - 1 || k >= g->NZ - 1) continue; /* halo keeps 0 */
        float ha = kMu0 * mu[idx] / dt;
        ch_hist[idx] = 1.0f;
        ch_curl[idx] = (1.0f / g->dx) / ha;
        ch_rhs[idx] = 1.0f / ha;
        if (sig[idx] > kPecSigma) {
            ce_hist[idx] = 0.0f;
            ce_curl[idx] = 0.0f;
            ce_rhs[idx] = 0.0f;
        } else {
            float e = kEps0 * eps[idx] / dt;
            float h = 0.5f * sig[idx];
            float a = e + h, b = e - h;
            ce_hist[idx] = b / a;
            ce_curl[idx] = (1.0f / g->dx) / a;
            ce_rhs[idx] = 1.0f / a;
        }
    }
}

static long long cell_of(const Geom* g, const int* loc)
{
    return (long long)loc[0] * g->sx + (long long)loc[1] * g->NZ + loc[2];
}

static float* comp_of(State* st, int c) { return c == 0 ? st->Ex : (c == 1 ? st->Ey : st->Ez); }

static void inject(const Geom* g, State* st, int it, int nt, int nsrc, const int* loc, const float* wave, int comp)
{
    if (comp < 0 || comp > 2) return;
    float* E = comp_of(st, comp);
    const float dl = comp == 0 ? g->dx : (comp == 1 ? g->dy : g->dz);
    for (int s = 0; s < g->nshot; ++s) {
        for (int m = 0; m < nsrc; ++m) {
            float scale = wave[(long long)m * nt + it] * dl / (g->dx * g->dy * g->dz);
            long long c = cell_of(g, loc + ((long long)s * nsrc + m) * 3);
            E[(long long)s * g->cells + c] -= st->ce_rhs[c] * scale;
        }
    }
}

static void sample(const Geom* g, State* st, int it, int nt, int nrx, const int* loc, float* out, int comp)
{
    const float* E = comp == 0 ? st->Ex : (comp == 1 ? st->Ey : st->Ez);
    for (int s = 0; s < g->nshot; ++s)
        for (int r = 0; r < nrx; ++r)
            out[((long long)s * nt + it) * nrx + r] = E[(long long)s * g->cells + cell_of(g, loc + ((long long)s * nrx + r) * 3)];
}

/* ------------------------------------------------------------------------ */
/* Histories.                                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
    int x0, y0, z0, nx, ny, nz;
} HBox;

static HBox make_box(const Geom* g, int physical)
{
    HBox b;
    if (physical) {
        b.x0 = g->p[0]; b.y0 = g->p[2]; b.z0 = g->p[4];
        b.nx = g->NX - 1 - g->p[0] - g->p[1];
        b.ny = g->NY - 1 - g->p[2] - g->p[3];
        b.nz = g->NZ - 1 - g->p[4] - g->p[5];
    } else {
        b.x0 = b.y0 = b.z0 = 0;
        b.nx = g->NX - 1; b.ny = g->NY - 1; b.nz = g->NZ - 1;
    }
    return b;
}

static long long box_cells(HBox b) { return (long long)b.nx * b.ny * b.nz; }

static long long box_field_index(const Geom* g, HBox b, long long s, long long h)
{
    long long hi = h / ((long long)b.ny * b.nz), rem = h % ((long long)b.ny * b.nz);
    long long hj = rem / b.nz, hk = rem % b.nz;
    return s * g->cells + (hi + b.x0) * g->sx + (hj + b.y0) * g->NZ + (hk + b.z0);
}

/* Write frame `slot` of one component (t-major, then shot, then box cells). */
static void save_frame(const Geom* g, HBox b, void* dst, int slot, const float* E, float* exact, int kind)
{
    const long long bc = box_cells(b), n = (long long)g->nshot * bc;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < n; ++w) {
        float v = E[box_field_index(g, b, w / bc, w % bc)];
        hist_put(dst, (long long)slot * n + w, v, kind);
        if (exact) exact[w] = v;
    }
}

static int comp_updates(const Geom* g, int comp, long long i, long long j, long long k)
{
    return comp == 0 ? upd_ex(g, i, j, k) : (comp == 1 ? upd_ey(g, i, j, k) : upd_ez(g, i, j, k));
}

/* R^n = (E^(n+1) - a E^n) / cb with a = ca where the component updates, else 1. */
static void save_rhs(const Geom* g, HBox b, void* dst, int slot, const float* E, const void* eh,
    const float* exact, const float* ca, const float* cb, int kind, int comp)
{
    const long long bc = box_cells(b), n = (long long)g->nshot * bc;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < n; ++w) {
        long long fi = box_field_index(g, b, w / bc, w % bc);
        long long c = fi % g->cells;
        long long i = c / g->sx, j = (c % g->sx) / g->NZ, k = c % g->NZ;
        long long hi = (long long)slot * n + w;
        float old = exact ? exact[w] : hist_get(eh, hi, kind);
        float a = comp_updates(g, comp, i, j, k) ? ca[c] : 1.0f;
        float r = cb[c] != 0.0f ? (E[fi] - a * old) / cb[c] : 0.0f;
        hist_put(dst, hi, r, kind);
    }
}

/* ------------------------------------------------------------------------ */
/* ABI-6 forward.                                                            */
/* ------------------------------------------------------------------------ */

static void setup_geom(Geom* g, int NX, int NY, int NZ, int nshot, float dx, float dy, float dz, const int* p)
{
    g->NX = NX; g->NY = NY; g->NZ = NZ;
    g->sy = NZ;
    g->sx = (long long)NY * NZ;
    g->cells = (long long)NX * NY * NZ;
    g->nshot = nshot;
    g->dx = dx; g->dy = dy; g->dz = dz;
    g->R = radius_of(g_order);
    for (int f = 0; f < 6; ++f) g->p[f] = p[f];
}

static void set_faces(Face* F, const int* p, const float* const* R, float* const* psi)
{
    for (int f = 0; f < 6; ++f) {
        F[f].p = p[f];
        F[f].R = R[f];
        F[f].psi1 = psi[2 * f];
        F[f].psi2 = psi[2 * f + 1];
    }
}

ORACLE_API void forward(
    const float* eps_r_pad, const float* sigma_pad, const float* mu_r_pad,
    void* E_saved, void* R_saved,
    float* Ex, float* Ey, float* Ez, float* Hx, float* Hy, float* Hz,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs,
    float* x0e1, float* x0e2, float* x0h1, float* x0h2, float* xme1, float* xme2, float* xmh1, float* xmh2,
    float* y0e1, float* y0e2, float* y0h1, float* y0h2, float* yme1, float* yme2, float* ymh1, float* ymh2,
    float* z0e1, float* z0e2, float* z0h1, float* z0h2, float* zme1, float* zme2, float* zmh1, float* zmh2,
    int p0, int p1, int p2, int p3, int p4, int p5,
    const float* x0E, const float* xmE, const float* y0E, const float* ymE, const float* z0E, const float* zmE,
    const float* x0H, const float* xmH, const float* y0H, const float* ymH, const float* z0H, const float* zmH,
    float dt, int nt, int nshot, int nrx, float dx, float dy, float dz,
    const int* rx_loc, float* rx_out, int rx_comp,
    int NX, int NY, int NZ, int nsrc, const int* src_loc, const float* src_wave, int src_comp,
    int S, int mode, int storage_type, int save_model_history, int use_async_offload)
{
    (void)use_async_offload;
    const int p[6] = {p0, p1, p2, p3, p4, p5};
    const float* eR[6] = {x0E, xmE, y0E, ymE, z0E, zmE};
    const float* hR[6] = {x0H, xmH, y0H, ymH, z0H, zmH};
    float* ePsi[12] = {x0e1, x0e2, xme1, xme2, y0e1, y0e2, yme1, yme2, z0e1, z0e2, zme1, zme2};
    float* hPsi[12] = {x0h1, x0h2, xmh1, xmh2, y0h1, y0h2, ymh1, ymh2, z0h1, z0h2, zmh1, zmh2};
    Geom g;
    State st;
    setup_geom(&g, NX, NY, NZ, nshot, dx, dy, dz, p);
    st.Ex = Ex; st.Ey = Ey; st.Ez = Ez; st.Hx = Hx; st.Hy = Hy; st.Hz = Hz;
    st.ce_hist = ce_hist; st.ce_curl = ce_curl; st.ce_rhs = ce_rhs;
    st.ch_hist = ch_hist; st.ch_curl = ch_curl; st.ch_rhs = ch_rhs;
    set_faces(st.eF, p, eR, ePsi);
    set_faces(st.hF, p, hR, hPsi);

    const int history = (storage_type & ST_DISABLED) == 0;
    const int kind = storage_type & ST_KIND_MASK;
    const int e_only = history && save_model_history && (storage_type & ST_RHS_FROM_E);
    const int keep_r = save_model_history && !e_only;
    const int physical = (storage_type & ST_PHYSICAL) != 0;
    const int has_pml = p0 || p1 || p2 || p3 || p4 || p5;
    const HBox box = make_box(&g, physical);
    const int ncomp = mode == 3 ? 3 : 1;
    const long long frame = (long long)nshot * box_cells(box);
    const int nt_saved = (nt + S - 1) / S;
    const long long comp_stride = (long long)nt_saved * frame;
    float* exact = NULL;

    deepgpr_clear_last_error();
    if (history && save_model_history && has_pml && physical) {
        set_error("oracle forward: material gradients with PML need the extended history");
        return;
    }
    if (e_only && S != 1) {
        set_error("oracle forward: E-only history needs sampling interval 1");
        return;
    }
    if (history && keep_r && kind != ST_F32) {
        exact = (float*)malloc((size_t)ncomp * (size_t)frame * sizeof(float));
        if (!exact) {
            set_error("oracle forward: out of memory for the exact E^n copy");
            return;
        }
    }
    build_coefficients(&g, eps_r_pad, sigma_pad, mu_r_pad, ce_hist, ce_curl, ce_rhs, ch_hist, ch_curl, ch_rhs, dt);

    float* comps[3] = {Ex, Ey, Ez};
    for (int it = 0; it < nt; ++it) {
        const int save = history && it % S == 0;
        if (save) {
            for (int c = 0; c < ncomp; ++c) {
                int fc = mode == 3 ? c : 2;
                save_frame(&g, box, (void*)hist_at(E_saved, c * comp_stride, kind), it / S, comps[fc],
                    exact ? exact + c * frame : NULL, kind);
            }
        }
        h_half_step(&g, &st);
        e_half_step(&g, &st);
        inject(&g, &st, it, nt, nsrc, src_loc, src_wave, src_comp);
        if (save && keep_r) {
            for (int c = 0; c < ncomp; ++c) {
                int fc = mode == 3 ? c : 2;
                save_rhs(&g, box, (void*)hist_at(R_saved, c * comp_stride, kind), it / S, comps[fc],
                    hist_at(E_saved, c * comp_stride, kind), exact ? exact + c * frame : NULL,
                    ce_hist, ce_rhs, kind, fc);
            }
        }
        sample(&g, &st, it, nt, nrx, rx_loc, rx_out, rx_comp);
    }
    (void)has_pml;
    if (e_only) {
        for (int c = 0; c < ncomp; ++c) {
            int fc = mode == 3 ? c : 2;
            save_frame(&g, box, (void*)hist_at(R_saved, c * frame, kind), 0, comps[fc], NULL, kind);
        }
    }
    free(exact);
}

/* ------------------------------------------------------------------------ */
/* Adjoint.                                                                  */
/* ------------------------------------------------------------------------ */

/* Six transposed-curl channels (deepgpr_cpu.c:529-532):
 *   A_X, A_Y -> target lambda_z component (E step: lambda_hz; H step: lambda_ez)
 *   B_X, B_Z -> target lambda_y component
 *   C_Y, C_Z -> target lambda_x component                                     */
enum { CH_AX = 0, CH_AY, CH_BX, CH_BZ, CH_CY, CH_CZ, NCH };

/* CPML part of one adjoint weight; advances the psi cotangent in place
 * (deepgpr_cpu.c:518-527). */
static float pml_weight(float lam, float inv_h, float up, float sign, Prof pr, float* lpsi)
{
    float ph = *lpsi;
    float w = (sign * up * pr.ra1 * lam - pr.rf * ph) * inv_h;
    *lpsi = sign * up * pr.rb * lam + pr.re * ph;
    return w;
}

typedef struct {
    const Geom* g;
    const float* lam;   /* lambda component whose base weight feeds the channel */
    const float* coef;  /* curl coefficient array (ce_curl or ch_curl) */
    const float* pml;   /* CPML part of the channel (full field layout) */
    int comp_kind;      /* which update predicate applies to the source cell */
    int spacing_axis;   /* 0: coef, 1: coef*dx/dy, 2: coef*dx/dz */
    float sign;         /* sign of the base term */
    int e_step;         /* 1: source points are E cells, 0: H cells */
} Channel;

static float scaled_coef(const Geom* g, float c1, int axis)
{
    if (axis == 1) return g->dy == g->dx ? c1 : c1 * g->dx / g->dy;
    if (axis == 2) return g->dz == g->dx ? c1 : c1 * g->dx / g->dz;
    return c1;
}

static int pred(const Geom* g, int which, long long i, long long j, long long k)
{
    switch (which) {
    case 0: return upd_ex(g, i, j, k);
    case 1: return upd_ey(g, i, j, k);
    case 2: return upd_ez(g, i, j, k);
    case 3: return upd_hx(g, i, j, k);
    case 4: return upd_hy(g, i, j, k);
    default: return upd_hz(g, i, j, k);
    }
}

/* Full channel weight at source point `id` = CPML part + base part, summed in
 * the reference's order (CPML faces first, then the interior term). */
static float channel_weight(const void* vctx, long long id)
{
    const Channel* ch = (const Channel*)vctx;
    const Geom* g = ch->g;
    const long long c = id % g->cells;
    const long long i = c / g->sx, j = (c % g->sx) / g->NZ, k = c % g->NZ;
    float w = ch->pml[id];
    if (pred(g, ch->comp_kind, i, j, k)) {
        float co = scaled_coef(g, ch->coef[c], ch->spacing_axis);
        w += (ch->sign * co) * ch->lam[id];
    }
    return w;
}

/* CPML part of the E-step channels; advances the E psi cotangents.
 * Face order and signs follow deepgpr_cpu.c:1155-1234.                      */
static void e_pml_weights(const Geom* g, State* st, const float* lex, const float* ley, const float* lez, float* chan)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    float* W[NCH];
    for (int c = 0; c < NCH; ++c) W[c] = chan + (long long)c * total;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long s = w / g->cells, idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        float acc[NCH] = {0, 0, 0, 0, 0, 0};
        const float up = st->ce_rhs[idx];
        for (int f = 0; f < 6; ++f) {
            Face* F = &st->eF[f];
            const int axis = f / 2;
            const long long cc = axis == 0 ? i : (axis == 1 ? j : k);
            const long long n = axis == 0 ? NX : (axis == 1 ? NY : NZ);
            const long long q = (f % 2 == 0) ? q_low_e(F->p, cc) : q_high(F->p, cc, n);
            if (q < 0 || cc == 0) continue;
            const Prof pr = prof_at(F, q);
            if (axis == 0) {
                if (j < NY - 1) {
                    Box3 b = {F->p + 1, NY - 1, NZ};
                    acc[CH_AX] += pml_weight(ley[w], 1.0f / g->dx, up, -1.0f, pr, &F->psi1[at3(b, s, q, j, k)]);
                }
                if (k < NZ - 1) {
                    Box3 b = {F->p + 1, NY, NZ - 1};
                    acc[CH_BX] += pml_weight(lez[w], 1.0f / g->dx, up, 1.0f, pr, &F->psi2[at3(b, s, q, j, k)]);
                }
            } else if (axis == 1) {
                if (i < NX - 1) {
                    Box3 b = {NX - 1, F->p + 1, NZ};
                    acc[CH_AY] += pml_weight(lex[w], 1.0f / g->dy, up, 1.0f, pr, &F->psi1[at3(b, s, i, q, k)]);
                }
                if (k < NZ - 1) {
                    Box3 b = {NX, F->p + 1, NZ - 1};
                    acc[CH_CY] += pml_weight(lez[w], 1.0f / g->dy, up, -1.0f, pr, &F->psi2[at3(b, s, i, q, k)]);
                }
            } else {
                if (i < NX - 1) {
                    Box3 b = {NX - 1, NY, F->p + 1};
                    acc[CH_BZ] += pml_weight(lex[w], 1.0f / g->dz, up, -1.0f, pr, &F->psi1[at3(b, s, i, j, q)]);
                }
                if (j < NY - 1) {
                    Box3 b = {NX, NY - 1, F->p + 1};
                    acc[CH_CZ] += pml_weight(ley[w], 1.0f / g->dz, up, 1.0f, pr, &F->psi2[at3(b, s, i, j, q)]);
                }
            }
        }
        for (int c = 0; c < NCH; ++c) W[c][w] = acc[c];
    }
}

/* CPML part of the H-step channels; advances the H psi cotangents
 * (deepgpr_cpu.c:1318-1397).                                                */
static void h_pml_weights(const Geom* g, State* st, const float* lhx, const float* lhy, const float* lhz, float* chan)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    float* W[NCH];
    for (int c = 0; c < NCH; ++c) W[c] = chan + (long long)c * total;
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long s = w / g->cells, idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        float acc[NCH] = {0, 0, 0, 0, 0, 0};
        const float up = st->ch_rhs[idx];
        for (int f = 0; f < 6; ++f) {
            Face* F = &st->hF[f];
            const int axis = f / 2;
            const long long cc = axis == 0 ? i : (axis == 1 ? j : k);
            const long long n = axis == 0 ? NX : (axis == 1 ? NY : NZ);
            const long long q = (f % 2 == 0) ? q_low_h(F->p, cc) : q_high(F->p, cc, n);
            if (q < 0) continue;
            const Prof pr = prof_at(F, q);
            if (axis == 0) {
                if (k < NZ - 1) {
                    Box3 b = {F->p, NY, NZ - 1};
                    acc[CH_AX] += pml_weight(lhy[w], 1.0f / g->dx, up, 1.0f, pr, &F->psi1[at3(b, s, q, j, k)]);
                }
                if (j < NY - 1) {
                    Box3 b = {F->p, NY - 1, NZ};
                    acc[CH_BX] += pml_weight(lhz[w], 1.0f / g->dx, up, -1.0f, pr, &F->psi2[at3(b, s, q, j, k)]);
                }
            } else if (axis == 1) {
                if (k < NZ - 1) {
                    Box3 b = {NX, F->p, NZ - 1};
                    acc[CH_AY] += pml_weight(lhx[w], 1.0f / g->dy, up, -1.0f, pr, &F->psi1[at3(b, s, i, q, k)]);
                }
                if (i < NX - 1) {
                    Box3 b = {NX - 1, F->p, NZ};
                    acc[CH_CY] += pml_weight(lhz[w], 1.0f / g->dy, up, 1.0f, pr, &F->psi2[at3(b, s, i, q, k)]);
                }
            } else {
                if (j < NY - 1) {
                    Box3 b = {NX, NY - 1, F->p};
                    acc[CH_BZ] += pml_weight(lhx[w], 1.0f / g->dz, up, 1.0f, pr, &F->psi1[at3(b, s, i, j, q)]);
                }
                if (i < NX - 1) {
                    Box3 b = {NX - 1, NY, F->p};
                    acc[CH_CZ] += pml_weight(lhy[w], 1.0f / g->dz, up, -1.0f, pr, &F->psi2[at3(b, s, i, j, q)]);
                }
            }
        }
        for (int c = 0; c < NCH; ++c) W[c][w] = acc[c];
    }
}

/* Transposed E step (deepgpr_cpu.c:1112-1271): lambda_H += curl^T of the E
 * channels.  lambda_E itself is rescaled later, inside the H step gather.    */
static void e_adjoint(const Geom* g, State* st, float* lex, float* ley, float* lez,
    float* lhx, float* lhy, float* lhz, float* chan)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    e_pml_weights(g, st, lex, ley, lez, chan);
    /* channel -> (lambda feeding it, E predicate, spacing scale, sign) */
    Channel C[NCH] = {
        {g, ley, st->ce_curl, chan + CH_AX * total, 1, 0, -1.0f, 1},
        {g, lex, st->ce_curl, chan + CH_AY * total, 0, 1, 1.0f, 1},
        {g, lez, st->ce_curl, chan + CH_BX * total, 2, 0, 1.0f, 1},
        {g, lex, st->ce_curl, chan + CH_BZ * total, 0, 2, -1.0f, 1},
        {g, lez, st->ce_curl, chan + CH_CY * total, 2, 1, -1.0f, 1},
        {g, ley, st->ce_curl, chan + CH_CZ * total, 1, 2, 1.0f, 1},
    };
    long long w;
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        lhz[w] += t_back(channel_weight, &C[CH_AX], w, g->sx, i, NX, g->R);
        lhz[w] += t_back(channel_weight, &C[CH_AY], w, NZ, j, NY, g->R);
        lhy[w] += t_back(channel_weight, &C[CH_BX], w, g->sx, i, NX, g->R);
        lhy[w] += t_back(channel_weight, &C[CH_BZ], w, 1, k, NZ, g->R);
        lhx[w] += t_back(channel_weight, &C[CH_CY], w, NZ, j, NY, g->R);
        lhx[w] += t_back(channel_weight, &C[CH_CZ], w, 1, k, NZ, g->R);
    }
}

/* Transposed H step (deepgpr_cpu.c:1281-1438); also applies the deferred
 * lambda_E <- ce_hist * lambda_E of the E step.  ch_hist is 1 on every
 * updated H cell, so lambda_H keeps its value.                              */
static void h_adjoint(const Geom* g, State* st, float* lex, float* ley, float* lez,
    float* lhx, float* lhy, float* lhz, float* chan, float* scaled)
{
    const long long total = (long long)g->nshot * g->cells;
    const int NX = g->NX, NY = g->NY, NZ = g->NZ;
    h_pml_weights(g, st, lhx, lhy, lhz, chan);
    Channel C[NCH] = {
        {g, lhy, st->ch_curl, chan + CH_AX * total, 4, 0, 1.0f, 0},
        {g, lhx, st->ch_curl, chan + CH_AY * total, 3, 1, -1.0f, 0},
        {g, lhz, st->ch_curl, chan + CH_BX * total, 5, 0, -1.0f, 0},
        {g, lhx, st->ch_curl, chan + CH_BZ * total, 3, 2, 1.0f, 0},
        {g, lhz, st->ch_curl, chan + CH_CY * total, 5, 1, 1.0f, 0},
        {g, lhy, st->ch_curl, chan + CH_CZ * total, 4, 2, -1.0f, 0},
    };
    long long w;
    /* The rescaled lambda_E goes to a side buffer first: the gather of a
     * neighbour must not see it (it reads only lambda_H, so in-place would be
     * fine too, but keeping the passes separate mirrors the GPU kernels). */
#pragma omp parallel for schedule(static)
    for (w = 0; w < total; ++w) {
        const long long idx = w % g->cells;
        const long long i = idx / g->sx, j = (idx % g->sx) / NZ, k = idx % NZ;
        float ex = lex[w], ey = ley[w], ez = lez[w];
        if (upd_ex(g, i, j, k)) ex = st->ce_hist[idx] * ex;
        if (upd_ey(g, i, j, k)) ey = st->ce_hist[idx] * ey;
        if (upd_ez(g, i, j, k)) ez = st->ce_hist[idx] * ez;
        ez += t_fwd(channel_weight, &C[CH_AX], w, g->sx, i, NX, g->R);
        ez += t_fwd(channel_weight, &C[CH_AY], w, NZ, j, NY, g->R);
        ey += t_fwd(channel_weight, &C[CH_BX], w, g->sx, i, NX, g->R);
        ey += t_fwd(channel_weight, &C[CH_BZ], w, 1, k, NZ, g->R);
        ex += t_fwd(channel_weight, &C[CH_CY], w, NZ, j, NY, g->R);
        ex += t_fwd(channel_weight, &C[CH_CZ], w, 1, k, NZ, g->R);
        scaled[w] = ex;
        scaled[total + w] = ey;
        scaled[2 * total + w] = ez;
    }
    memcpy(lex, scaled, (size_t)total * sizeof(float));
    memcpy(ley, scaled + total, (size_t)total * sizeof(float));
    memcpy(lez, scaled + 2 * total, (size_t)total * sizeof(float));
}

/* Imaging condition for one saved step (deepgpr_cpu.c:1659-1745). */
static void imaging(const Geom* g, HBox b, const float* lex, const float* ley, const float* lez,
    const void* e_frame, long long e_cstride, const void* second, long long s_cstride,
    const float* ca, const float* cb, const float* sig, float* g_eps, float* g_sig,
    float dt, int want_eps, int want_sig, int weight, int mode, int kind, int e_only)
{
    const long long bc = box_cells(b);
    const long long sy = g->NY - 1, sz = g->NZ - 1;
    const int ncomp = mode == 3 ? 3 : 1;
    long long h;
#pragma omp parallel for schedule(static)
    for (h = 0; h < bc; ++h) {
        long long hi = h / ((long long)b.ny * b.nz), rem = h % ((long long)b.ny * b.nz);
        long long ix = hi + b.x0, iy = rem / b.nz + b.y0, iz = rem % b.nz + b.z0;
        long long c = ix * g->sx + iy * g->NZ + iz;
        float acc_e = 0.0f, acc_s = 0.0f;
        for (int s = 0; s < g->nshot; ++s) {
            long long fi = (long long)s * g->cells + c;
            long long base = (long long)s * bc + h;
            const float lam3[3] = {lex[fi], ley[fi], lez[fi]};
            for (int q = 0; q < ncomp; ++q) {
                int comp = mode == 3 ? q : 2;
                int upd = comp_updates(g, comp, ix, iy, iz);
                float eo = hist_get(e_frame, q * e_cstride + base, kind);
                float sec = hist_get(second, q * s_cstride + base, kind);
                float lam = lam3[comp];
                float a = ca[c], bb = cb[c];
                float rhs = sec;
                if (e_only) {
                    float aeff = upd ? a : 1.0f;
                    rhs = bb != 0.0f ? (sec - aeff * eo) / bb : 0.0f;
                }
                if (eo == 0.0f && rhs == 0.0f) lam = 0.0f;
                float gca = upd ? lam * eo * (float)weight : 0.0f;
                float gcb = lam * rhs * (float)weight;
                if (sig[c] <= kPecSigma) {
                    if (want_eps == 1) {
                        float d_ca = kEps0 * (1.0f - a) * bb / dt;
                        float d_cb = -kEps0 * bb * bb / dt;
                        acc_e += gca * d_ca + gcb * d_cb;
                    }
                    if (want_sig == 1) {
                        float d_ca = -0.5f * (1.0f + a) * bb;
                        float d_cb = -0.5f * bb * bb;
                        acc_s += gca * d_ca + gcb * d_cb;
                    }
                }
            }
        }
        long long gi = ix * sy * sz + iy * sz + iz;
        if (want_eps == 1) g_eps[gi] += acc_e;
        if (want_sig == 1) g_sig[gi] += acc_s;
    }
}

ORACLE_API void backward(
    const float* eps_r_pad, const float* sigma_pad, const float* mu_r_pad,
    const void* E_saved, const void* R_saved,
    float* lex, float* ley, float* lez, float* lhx, float* lhy, float* lhz,
    float* ce_hist, float* ce_curl, float* ce_rhs, float* ch_hist, float* ch_curl, float* ch_rhs,
    float* x0e1, float* x0e2, float* x0h1, float* x0h2, float* xme1, float* xme2, float* xmh1, float* xmh2,
    float* y0e1, float* y0e2, float* y0h1, float* y0h2, float* yme1, float* yme2, float* ymh1, float* ymh2,
    float* z0e1, float* z0e2, float* z0h1, float* z0h2, float* zme1, float* zme2, float* zmh1, float* zmh2,
    int p0, int p1, int p2, int p3, int p4, int p5,
    const float* x0E, const float* xmE, const float* y0E, const float* ymE, const float* z0E, const float* zmE,
    const float* x0H, const float* xmH, const float* y0H, const float* ymH, const float* z0H, const float* zmH,
    float dt, int nt, int nshot, int nrx, float dx, float dy, float dz,
    int NX, int NY, int NZ,
    int ndata, const int* rx_loc, const float* data_grad, int rx_comp,
    int nsrc, const int* src_loc, int src_comp, float* grad_source, int want_src,
    float* grad_eps, float* grad_sig, int want_eps, int want_sig,
    int S, int mode, int storage_type, int use_async_offload)
{
    (void)nrx;
    (void)use_async_offload;
    const int p[6] = {p0, p1, p2, p3, p4, p5};
    const float* eR[6] = {x0E, xmE, y0E, ymE, z0E, zmE};
    const float* hR[6] = {x0H, xmH, y0H, ymH, z0H, zmH};
    float* ePsi[12] = {x0e1, x0e2, xme1, xme2, y0e1, y0e2, yme1, yme2, z0e1, z0e2, zme1, zme2};
    float* hPsi[12] = {x0h1, x0h2, xmh1, xmh2, y0h1, y0h2, ymh1, ymh2, z0h1, z0h2, zmh1, zmh2};
    Geom g;
    State st;
    setup_geom(&g, NX, NY, NZ, nshot, dx, dy, dz, p);
    st.Ex = lex; st.Ey = ley; st.Ez = lez; st.Hx = lhx; st.Hy = lhy; st.Hz = lhz;
    st.ce_hist = ce_hist; st.ce_curl = ce_curl; st.ce_rhs = ce_rhs;
    st.ch_hist = ch_hist; st.ch_curl = ch_curl; st.ch_rhs = ch_rhs;
    set_faces(st.eF, p, eR, ePsi);
    set_faces(st.hF, p, hR, hPsi);

    const int kind = storage_type & ST_KIND_MASK;
    const int want_model = want_eps || want_sig;
    const int e_only = want_model && (storage_type & ST_RHS_FROM_E);
    const int physical = (storage_type & ST_PHYSICAL) != 0;
    const int has_pml = p0 || p1 || p2 || p3 || p4 || p5;
    const HBox box = make_box(&g, physical);
    const long long frame = (long long)nshot * box_cells(box);
    const int nt_saved = (nt + S - 1) / S;
    const long long comp_stride = (long long)nt_saved * frame;
    const long long total = (long long)nshot * g.cells;

    deepgpr_clear_last_error();
    if (want_model && has_pml && physical) {
        set_error("oracle backward: material gradients with PML need the extended history");
        return;
    }
    if (e_only && S != 1) {
        set_error("oracle backward: E-only history needs sampling interval 1");
        return;
    }
    float* chan = (float*)malloc((size_t)NCH * (size_t)total * sizeof(float));
    float* scaled = (float*)malloc((size_t)3 * (size_t)total * sizeof(float));
    if (!chan || !scaled) {
        free(chan);
        free(scaled);
        set_error("oracle backward: out of memory for adjoint scratch");
        return;
    }
    build_coefficients(&g, eps_r_pad, sigma_pad, mu_r_pad, ce_hist, ce_curl, ce_rhs, ch_hist, ch_curl, ch_rhs, dt);

    float* lam_rx = rx_comp == 0 ? lex : (rx_comp == 1 ? ley : lez);
    const float* lam_src = src_comp == 0 ? lex : (src_comp == 1 ? ley : lez);
    const float dl = src_comp == 0 ? dx : (src_comp == 1 ? dy : dz);
    const float geo = dl / (dx * dy * dz);

    for (int it = nt - 1; it >= 0; --it) {
        if (rx_comp >= 0 && rx_comp <= 2) {
            for (int s = 0; s < nshot; ++s)
                for (int r = 0; r < ndata; ++r)
                    lam_rx[(long long)s * g.cells + cell_of(&g, rx_loc + ((long long)s * ndata + r) * 3)] +=
                        data_grad[((long long)s * nt + it) * ndata + r];
        }
        if (want_src == 1) {
            for (int m = 0; m < nsrc; ++m)
                for (int s = 0; s < nshot; ++s) {
                    long long c = cell_of(&g, src_loc + ((long long)s * nsrc + m) * 3);
                    grad_source[(long long)m * nt + it] += -ce_rhs[c] * geo * lam_src[(long long)s * g.cells + c];
                }
        }
        if (want_model && it % S == 0) {
            int slot = it / S, weight = S;
            const void* ef = hist_at(E_saved, (long long)slot * frame, kind);
            const void* sec;
            long long sstride = comp_stride;
            if (!e_only) sec = hist_at(R_saved, (long long)slot * frame, kind);
            else if (slot + 1 < nt_saved) sec = hist_at(E_saved, (long long)(slot + 1) * frame, kind);
            else {
                sec = R_saved;
                sstride = frame;
            }
            if (it + weight > nt) weight = nt - it;
            imaging(&g, box, lex, ley, lez, ef, comp_stride, sec, sstride, ce_hist, ce_rhs, sigma_pad,
                grad_eps, grad_sig, dt, want_eps, want_sig, weight, mode, kind, e_only);
        }
        e_adjoint(&g, &st, lex, ley, lez, lhx, lhy, lhz, chan);
        h_adjoint(&g, &st, lex, ley, lez, lhx, lhy, lhz, chan, scaled);
    }
    free(chan);
    free(scaled);
}
