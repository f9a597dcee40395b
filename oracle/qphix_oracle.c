/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- plain-C CPU restatement of the
 * milc-qphix staggered solver path (see qphix_oracle.h for the layout).
 * Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load this library, and only as the checker.
 *
 * Every function cites the reference statement it restates.  The per-site
 * stencil body is absent from the reference (it is #included from the
 * unvendored milc-qphix-codegen, ks_dslash_complete_specialization.cpp:377);
 * it is restated from the MILC asqtad formula:
 *   out(x) = sum_mu F_mu(x) psi(x+mu) - B_mu(x)^dag psi(x-mu)
 *          + sum_mu L_mu(x) psi(x+3mu) - LB_mu(x)^dag psi(x-3mu)
 * with F/L the forward links and B/LB the caller's backward links.
 */
#define _POSIX_C_SOURCE 200809L
#include "qphix_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

enum { ORC_EVEN = 2, ORC_ODD = 1, ORC_EVENODD = 3 };

typedef struct {
    int nx, ny, nz, nt, nxh;
    long V, Vh;
} lat_t;

static lat_t mk_lat(const int L[4])
{
    lat_t g;
    g.nx = L[0]; g.ny = L[1]; g.nz = L[2]; g.nt = L[3];
    g.nxh = g.nx / 2;
    g.V = (long)g.nx * g.ny * g.nz * g.nt;
    g.Vh = g.V / 2;
    return g;
}

static double wall_now(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1.e-6 * tv.tv_usec;
}

/* ------------------------------------------------------------------ */
/* Neighbour tables: init_ks_dslash_imp, qphix_misc.cpp:46-230,       */
/* at VECLEN=1 (Vxh=Nxh, Vy=Ny, ...), XY_PAD=1 (ks_config.h:28),        */
/* XYZ_PAD=0, every direction node-local (non-MPI setup_comms,        */
/* ks_boundary.cpp:76-80).                                            */
/* ------------------------------------------------------------------ */
long orc_neigh_table(const int L[4], unsigned *table, unsigned char *bound)
{
    const int Vxh = L[0] / 2, Vy = L[1], Vz = L[2], Vt = L[3];
    const long Pxy = (long)Vxh * Vy + 1;
    const long Pxyz = Pxy * Vz;
    const long half = Pxyz * Vt;
    for (int cb = 0; cb < 2; ++cb) {
        unsigned *NT = table + (size_t)cb * half * 16;
        unsigned char *BT = bound + (size_t)cb * half * 4;
        for (int t = 0; t < Vt; ++t)
        for (int z = 0; z < Vz; ++z)
        for (int y = 0; y < Vy; ++y)
        for (int x = 0; x < Vxh; ++x) {
            const int xodd = (y + z + t + cb) & 1;
            const long ind = t * Pxyz + z * Pxy + (long)y * Vxh + x;
            unsigned *n = NT + 16 * ind;
            unsigned char *b = BT + 4 * ind;
            b[0] = 0xFF; b[1] = 0xFF; b[2] = 0; b[3] = 0;
            /* one hop, k = 2*dir + (forward) */
            n[0] = (unsigned)(ind + xodd - 1); if (x + xodd - 1 < 0)   { n[0] += Vxh; b[2] ^= 1; }
            n[1] = (unsigned)(ind + xodd);     if (x + xodd >= Vxh)    { n[1] -= Vxh; b[2] ^= 2; }
            n[2] = (unsigned)(ind - Vxh);      if (y == 0)             { n[2] += Vy * Vxh; b[2] ^= 4; }
            n[3] = (unsigned)(ind + Vxh);      if (y == Vy - 1)        { n[3] -= Vy * Vxh; b[2] ^= 8; }
            n[4] = (unsigned)(ind - Pxy);      if (z == 0)             { n[4] += Vz * Pxy; b[2] ^= 16; }
            n[5] = (unsigned)(ind + Pxy);      if (z == Vz - 1)        { n[5] -= Vz * Pxy; b[2] ^= 32; }
            n[6] = (unsigned)(ind - Pxyz);     if (t == 0)             { n[6] += Vt * Pxyz; b[2] ^= 64; }
            n[7] = (unsigned)(ind + Pxyz);     if (t == Vt - 1)        { n[7] -= Vt * Pxyz; b[2] ^= 128; }
            /* three hops; a second wrap is applied for extents < 3 */
            n[8] = (unsigned)(ind + xodd - 2);
            if (x + xodd - 2 < 0) { n[8] += Vxh; if (x + xodd - 2 + Vxh < 0) n[8] += Vxh; else b[3] ^= 1; }
            n[9] = (unsigned)(ind + xodd + 1);
            if (x + xodd + 1 >= Vxh) { n[9] -= Vxh; if (x + xodd + 1 - Vxh >= Vxh) n[9] -= Vxh; else b[3] ^= 2; }
            n[10] = (unsigned)(ind - 3 * Vxh);
            if (y - 3 < 0) { n[10] += Vy * Vxh; if (y - 3 + Vy < 0) n[10] += Vy * Vxh; else b[3] ^= 4; }
            n[11] = (unsigned)(ind + 3 * Vxh);
            if (y + 3 >= Vy) { n[11] -= Vy * Vxh; if (y + 3 - Vy >= Vy) n[11] -= Vy * Vxh; else b[3] ^= 8; }
            n[12] = (unsigned)(ind - 3 * Pxy);
            if (z - 3 < 0) { n[12] += Vz * Pxy; if (z - 3 + Vz < 0) n[12] += Vz * Pxy; else b[3] ^= 16; }
            n[13] = (unsigned)(ind + 3 * Pxy);
            if (z + 3 >= Vz) { n[13] -= Vz * Pxy; if (z + 3 - Vz >= Vz) n[13] -= Vz * Pxy; else b[3] ^= 32; }
            n[14] = (unsigned)(ind - 3 * Pxyz);
            if (t - 3 < 0) { n[14] += Vt * Pxyz; if (t - 3 + Vt < 0) n[14] += Vt * Pxyz; else b[3] ^= 64; }
            n[15] = (unsigned)(ind + 3 * Pxyz);
            if (t + 3 >= Vt) { n[15] -= Vt * Pxyz; if (t + 3 - Vt >= Vt) n[15] -= Vt * Pxyz; else b[3] ^= 128; }
        }
    }
    return half;
}

/* ------------------------------------------------------------------ */
/* Precision-generic part.  T is the reference's fptype.              */
/* ------------------------------------------------------------------ */

static inline long blk_index(const lat_t *g, int x, int y, int z, int t)
{
    x = (x % g->nx + g->nx) % g->nx;
    y = (y % g->ny + g->ny) % g->ny;
    z = (z % g->nz + g->nz) % g->nz;
    t = (t % g->nt + g->nt) % g->nt;
    return (((long)t * g->nz + z) * g->ny + y) * g->nxh + x / 2;
}

#define ORC_DEFINE(T, SFX)                                                              \
                                                                                        \
/* acc += U v  or  acc -= U^dag v  (3x3 complex, interleaved re/im) */                  \
static inline void mv_##SFX(T *acc, const T *u, const T *v, int adj)                    \
{                                                                                       \
    for (int r = 0; r < 3; ++r) {                                                       \
        T re = 0, im = 0;                                                               \
        for (int c = 0; c < 3; ++c) {                                                   \
            T ur, ui;                                                                   \
            if (!adj) { ur = u[6 * r + 2 * c]; ui = u[6 * r + 2 * c + 1]; }             \
            else      { ur = u[6 * c + 2 * r]; ui = -u[6 * c + 2 * r + 1]; }            \
            re += ur * v[2 * c] - ui * v[2 * c + 1];                                    \
            im += ur * v[2 * c + 1] + ui * v[2 * c];                                    \
        }                                                                               \
        if (!adj) { acc[2 * r] += re; acc[2 * r + 1] += im; }                           \
        else      { acc[2 * r] -= re; acc[2 * r + 1] -= im; }                           \
    }                                                                                   \
}                                                                                       \
                                                                                        \
/* qphix_ks_dslash (ks_long_dslash.cpp:564-668): out[cb] = D in[1-cb]; the link      */ \
/* block of output site j is the raw site cb*Vh + j (qphix_f3.cpp:995-1018).         */ \
void orc_dslash_##SFX(const int L[4], const T *fat, const T *lng, const T *fatback,     \
                      const T *lngback, T *out, const T *in, int cb)                    \
{                                                                                       \
    const lat_t g = mk_lat(L);                                                          \
    _Pragma("omp parallel for schedule(static)")                                        \
    for (long j = 0; j < g.Vh; ++j) {                                                   \
        const int xh = (int)(j % g.nxh);                                                \
        long r = j / g.nxh;                                                             \
        const int y = (int)(r % g.ny); r /= g.ny;                                       \
        const int z = (int)(r % g.nz);                                                  \
        const int t = (int)(r / g.nz);                                                  \
        const int x = 2 * xh + ((y + z + t + cb) & 1);                                  \
        const long site = cb * g.Vh + j;                                                \
        T acc[6] = {0, 0, 0, 0, 0, 0};                                                  \
        for (int mu = 0; mu < 4; ++mu) {                                                \
            int d[4] = {0, 0, 0, 0};                                                    \
            d[mu] = 1;                                                                  \
            const long fp = blk_index(&g, x + d[0], y + d[1], z + d[2], t + d[3]);      \
            const long fm = blk_index(&g, x - d[0], y - d[1], z - d[2], t - d[3]);      \
            const long lp = blk_index(&g, x + 3 * d[0], y + 3 * d[1], z + 3 * d[2], t + 3 * d[3]); \
            const long lm = blk_index(&g, x - 3 * d[0], y - 3 * d[1], z - 3 * d[2], t - 3 * d[3]); \
            const long lo = 72 * site + 18 * mu;                                        \
            mv_##SFX(acc, fat + lo, in + 6 * fp, 0);                                    \
            mv_##SFX(acc, fatback + lo, in + 6 * fm, 1);                                \
            mv_##SFX(acc, lng + lo, in + 6 * lp, 0);                                    \
            mv_##SFX(acc, lngback + lo, in + 6 * lm, 1);                                \
        }                                                                               \
        for (int k = 0; k < 6; ++k) out[6 * j + k] = acc[k];                            \
    }                                                                                   \
}                                                                                       \
                                                                                        \
/* QPHIX_*_asqtad_dslash, qphix_f3.cpp:1233-1245 */                                     \
void orc_asqtad_dslash_##SFX(const int L[4], const T *fat, const T *lng,                \
                             const T *fatback, const T *lngback, T *out,                \
                             const T *in, int parity)                                   \
{                                                                                       \
    const lat_t g = mk_lat(L);                                                          \
    const long n = g.Vh * 6;                                                            \
    if (parity == ORC_EVEN)                                                             \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, out, in + n, 0);                \
    else                                                                                \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, out + n, in, 1);                \
}                                                                                       \
                                                                                        \
/* calc_source_norm, ks_d_congrad_fn.cpp:62-71 (fptype accumulator) */                 \
static double norm_##SFX(const T *s, long n)                                            \
{                                                                                       \
    T acc = 0;                                                                          \
    for (long i = 0; i < n; ++i) acc += s[i] * s[i];                                    \
    return (double)acc;                                                                 \
}                                                                                       \
                                                                                        \
/* relative_residue, ks_blas_utils_c.cpp:110-149 */                                     \
static T relres_##SFX(const lat_t *g, const T *p, const T *q)                           \
{                                                                                       \
    double residue = 0.0;                                                               \
    for (long s = 0; s < g->Vh; ++s) {                                                  \
        double num = 0, den = 0;                                                        \
        for (int k = 0; k < 6; ++k) {                                                   \
            num += (double)(p[6 * s + k] * p[6 * s + k]);                               \
            den += (double)(q[6 * s + k] * q[6 * s + k]);                               \
        }                                                                               \
        if (num == 0) continue;                                                         \
        residue += (den == 0) ? 1.0 : (num / den);                                      \
    }                                                                                   \
    return (T)sqrt(2 * residue / (double)g->V);                                         \
}                                                                                       \
                                                                                        \
/* QPHIX_fptype_asqtad_invert, ks_d_congrad_fn.cpp:221-619 */                           \
int orc_invert_##SFX(const int L[4], const T *fat, const T *lng, const T *fatback,      \
                     const T *lngback, orc_info_t *info, const orc_invert_arg_t *inv,   \
                     orc_resid_arg_t *res, T mass, T *out, const T *in)                 \
{                                                                                       \
    const lat_t g = mk_lat(L);                                                          \
    const long n = g.Vh * 6;                                                            \
    const T *t_src;                                                                     \
    T *t_dest;                                                                          \
    if (inv->parity != ORC_ODD) { t_src = in; t_dest = out; }                           \
    else                        { t_src = in + n; t_dest = out + n; }                   \
    int iteration;                                                                      \
    T a, b;                                                                             \
    double rsq = 0, relrsq = 0, oldrsq, pkp, source_norm;                               \
    int nrestart;                                                                       \
    const int niter = inv->max;                                                         \
    const int max_restarts = inv->nrestart;                                             \
    const T rsqmin = (T)res->resid;                                                     \
    const T relrsqmin = (T)res->relresid;                                               \
    const int max_cg = max_restarts * niter;                                            \
    const T msq_x4 = (T)(4.0 * mass * mass);                                            \
    int parity = inv->parity & 1;                                                       \
    int otherparity = 1 - parity;                                                       \
    int parity0 = inv->parity;                                                          \
    T *ttt = calloc(n, sizeof(T)), *ttt_temp = calloc(n, sizeof(T));                    \
    T *cg_p = calloc(n, sizeof(T)), *resid = calloc(n, sizeof(T));                      \
    info->final_sec = wall_now();                                                       \
    info->final_flop = 0.;                                                              \
    int total_iters = 0;                                                                \
    iteration = 0;                                                                      \
start:                                                                                  \
    source_norm = norm_##SFX(t_src, n);                                                 \
    nrestart = 0;                                                                       \
    total_iters += iteration;                                                           \
    iteration = 0;                                                                      \
    res->size_r = 0;                                                                    \
    res->size_relr = 0;                                                                 \
    if (source_norm == 0.0) { /* trivial source, :326-350 */                            \
        for (long i = 0; i < n; ++i) t_dest[i] = 0;                                     \
        info->final_sec = wall_now() - info->final_sec;                                 \
        res->final_rel = 0;                                                             \
        res->final_rsq = 0;                                                             \
        res->final_iter = total_iters;                                                  \
        res->final_restart = nrestart;                                                  \
        free(ttt); free(ttt_temp); free(cg_p); free(resid);                             \
        return iteration;                                                               \
    }                                                                                   \
    for (;;) {                                                                          \
        if ((iteration % niter == 0) ||                                                 \
            ((rsqmin <= 0 || rsqmin > res->size_r) &&                                   \
             (relrsqmin <= 0 || relrsqmin > res->size_relr))) {                         \
            /* restart: true residual, :365-448 */                                      \
            rsq = 0.0;                                                                  \
            orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt_temp, t_dest, otherparity); \
            orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt, ttt_temp, parity);     \
            {                                                                           \
                T acc = 0; /* calc_rsq, :82-99 */                                       \
                for (long i = 0; i < n; ++i) {                                          \
                    ttt[i] = ttt[i] + (-msq_x4) * t_dest[i];                            \
                    resid[i] = t_src[i] + ttt[i];                                       \
                    cg_p[i] = resid[i];                                                 \
                    acc += resid[i] * resid[i];                                         \
                }                                                                       \
                rsq = (double)acc;                                                      \
            }                                                                           \
            if (relrsqmin > 0) relrsq = relres_##SFX(&g, resid, t_dest);                \
            res->final_rsq = (T)rsq / source_norm;                                      \
            res->final_rel = (T)relrsq;                                                 \
            iteration++;                                                                \
            if (iteration >= max_cg || nrestart >= max_restarts ||                      \
                ((rsqmin <= 0 || rsqmin > res->final_rsq) &&                            \
                 (relrsqmin <= 0 || relrsqmin > res->final_rel))) {                     \
                if (parity0 == ORC_EVENODD) { /* :437-444 */                            \
                    otherparity = parity0 & 1;                                          \
                    parity = 1 - otherparity;                                           \
                    parity0 = ORC_EVEN;                                                 \
                    t_src = in + n;                                                     \
                    t_dest = out + n;                                                   \
                    goto start;                                                         \
                } else                                                                  \
                    break;                                                              \
            }                                                                           \
            if (iteration != 0) nrestart++;                                             \
        }                                                                               \
        oldrsq = rsq;                                                                   \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt_temp, cg_p, otherparity);   \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt, ttt_temp, parity);         \
        {                                                                               \
            T acc = 0; /* calc_pkp, :159-171 */                                         \
            for (long i = 0; i < n; ++i) {                                              \
                ttt[i] = ttt[i] + (-msq_x4) * cg_p[i];                                  \
                acc += cg_p[i] * ttt[i];                                                \
            }                                                                           \
            pkp = (double)acc;                                                          \
        }                                                                               \
        iteration++;                                                                    \
        a = (T)(-rsq / pkp);                                                            \
        rsq = 0.0;                                                                      \
        {                                                                               \
            T acc = 0; /* calc_rsq2, :131-147 */                                        \
            for (long i = 0; i < n; ++i) {                                              \
                t_dest[i] = t_dest[i] + a * cg_p[i];                                    \
                resid[i] = resid[i] + a * ttt[i];                                       \
                acc += resid[i] * resid[i];                                             \
            }                                                                           \
            rsq = (double)acc;                                                          \
        }                                                                               \
        if (relrsqmin > 0) relrsq = relres_##SFX(&g, resid, t_dest);                    \
        res->size_r = (T)rsq / source_norm;                                             \
        res->size_relr = (T)relrsq;                                                     \
        res->final_rsq = res->size_r;                                                   \
        b = (T)((T)rsq / oldrsq);                                                       \
        for (long i = 0; i < n; ++i) cg_p[i] = resid[i] + b * cg_p[i]; /* axpy :178 */  \
    }                                                                                   \
    info->final_sec = wall_now() - info->final_sec;                                     \
    total_iters += iteration;                                                           \
    res->final_iter = total_iters;                                                      \
    res->final_restart = nrestart;                                                      \
    free(ttt); free(ttt_temp); free(cg_p); free(resid);                                 \
    info->final_flop = 1187. * total_iters * (double)g.V;                               \
    return iteration;                                                                   \
}                                                                                       \
                                                                                        \
/* QPHIX_fptype_asqtad_invert_multi, ks_multicg_offset.cpp:205-689 */                   \
int orc_invert_multi_##SFX(const int L[4], const T *fat, const T *lng,                  \
                           const T *fatback, const T *lngback, orc_info_t *info,        \
                           const orc_invert_arg_t *inv, orc_resid_arg_t *res[],         \
                           const T *mass, int num_offsets, T *out[], const T *in)       \
{                                                                                       \
    if (num_offsets <= 0) return 0; /* :218-225 */                                      \
    const lat_t g = mk_lat(L);                                                          \
    const long n = g.Vh * 6;                                                            \
    int parity0 = inv->parity;                                                          \
    const T *t_src = (parity0 != ORC_ODD) ? in : in + n;                                \
    T **t_dest = malloc(sizeof(T *) * num_offsets);                                     \
    for (int j = 0; j < num_offsets; ++j)                                               \
        t_dest[j] = (parity0 != ORC_ODD) ? out[j] : out[j] + n;                         \
    int iteration, total_iters;                                                         \
    double rsq = 0., oldrsq, pkp, source_norm;                                          \
    int nrestart = 0;                                                                   \
    int j, j_low;                                                                       \
    const int niter = inv->max;                                                         \
    const int max_restarts = inv->nrestart;                                             \
    const T rsqmin = (T)res[0]->resid;                                                  \
    const int max_cg = max_restarts * niter;                                            \
    int parity = parity0 & 1;                                                           \
    int otherparity = 1 - parity;                                                       \
    T *ttt = calloc(n, sizeof(T)), *ttt_temp = calloc(n, sizeof(T));                    \
    T *resid = calloc(n, sizeof(T));                                                    \
    T **pm = malloc(sizeof(T *) * num_offsets);                                         \
    for (j = 0; j < num_offsets; ++j) pm[j] = calloc(n, sizeof(T));                     \
    T *shifts = malloc(num_offsets * sizeof(T));                                        \
    T *zeta_i = malloc(num_offsets * sizeof(T)), *zeta_im1 = malloc(num_offsets * sizeof(T)); \
    T *zeta_ip1 = malloc(num_offsets * sizeof(T)), *beta_i = malloc(num_offsets * sizeof(T)); \
    T *beta_im1 = malloc(num_offsets * sizeof(T)), *alpha = malloc(num_offsets * sizeof(T)); \
    /* the reference leaves `finished` uninitialised (:329); zero is what a fresh   */ \
    /* allocation holds and the only value under which its shrink logic is defined */  \
    int *finished = calloc(num_offsets, sizeof(int));                                   \
    double offset_low = 1.0e+20;                                                        \
    j_low = -1;                                                                         \
    for (j = 0; j < num_offsets; j++) { /* :332-342 */                                  \
        shifts[j] = (T)(mass[j] * mass[j] * 4.0);                                       \
        if (shifts[j] < offset_low) { offset_low = shifts[j]; j_low = j; }              \
    }                                                                                   \
    for (j = 0; j < num_offsets; j++)                                                   \
        if (j != j_low) shifts[j] -= shifts[j_low];                                     \
    iteration = 0;                                                                      \
    total_iters = 0;                                                                    \
    info->final_sec = wall_now();                                                       \
    info->final_flop = 0.;                                                              \
    int rc;                                                                             \
start:;                                                                                 \
    int num_offsets_now = num_offsets;                                                  \
    source_norm = norm_##SFX(t_src, n);                                                 \
    for (j = 0; j < num_offsets; ++j) memset(t_dest[j], 0, n * sizeof(T));              \
    for (j = 0; j < num_offsets; ++j) memcpy(pm[j], t_src, n * sizeof(T));              \
    memcpy(resid, t_src, n * sizeof(T));                                                \
    rsq = source_norm;                                                                  \
    if (source_norm == 0.) { /* :377-419 */                                             \
        for (j = 0; j < num_offsets; j++) {                                             \
            res[j]->final_rsq = 0.;                                                     \
            res[j]->size_r = 0.;                                                        \
            res[j]->size_relr = 0.;                                                     \
            res[j]->final_iter = iteration;                                             \
            res[j]->final_restart = nrestart;                                           \
        }                                                                               \
        rc = iteration;                                                                 \
        goto done;                                                                      \
    }                                                                                   \
    double rsqstop = rsqmin * source_norm;                                              \
    for (j = 0; j < num_offsets; j++) {                                                 \
        zeta_im1[j] = zeta_i[j] = 1.0;                                                  \
        beta_im1[j] = -1.0;                                                             \
        alpha[j] = 0.0;                                                                 \
    }                                                                                   \
    do {                                                                                \
        oldrsq = rsq;                                                                   \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt_temp, pm[j_low], otherparity); \
        orc_dslash_##SFX(L, fat, lng, fatback, lngback, ttt, ttt_temp, parity);         \
        {                                                                               \
            const T m4 = (T)(-1.0 * offset_low); /* calc_pkp :107-122 */                \
            T acc = 0;                                                                  \
            for (long i = 0; i < n; ++i) {                                              \
                ttt[i] = ttt[i] + m4 * pm[j_low][i];                                    \
                acc += pm[j_low][i] * ttt[i];                                           \
            }                                                                           \
            pkp = (double)acc;                                                          \
        }                                                                               \
        iteration++;                                                                    \
        total_iters++;                                                                  \
        beta_i[j_low] = (T)(-rsq / pkp); /* :475-496 */                                 \
        zeta_ip1[j_low] = 1.0;                                                          \
        for (j = 0; j < num_offsets_now; j++) if (j != j_low) {                         \
            zeta_ip1[j] = zeta_i[j] * zeta_im1[j] * beta_im1[j_low];                    \
            T c1 = beta_i[j_low] * alpha[j_low] * (zeta_im1[j] - zeta_i[j]);            \
            T c2 = (T)((T)(zeta_im1[j] * beta_im1[j_low]) *                             \
                       (1.0 + (T)(shifts[j] * beta_i[j_low])));                         \
            if ((T)(c1 + c2) != 0.0)                                                    \
                zeta_ip1[j] /= (T)(c1 + c2);                                            \
            else { zeta_ip1[j] = 0.0; finished[j] = 1; }                                \
            if (zeta_i[j] != 0.0)                                                       \
                beta_i[j] = beta_i[j_low] * zeta_ip1[j] / zeta_i[j];                    \
            else { zeta_ip1[j] = 0.0; beta_i[j] = 0.0; finished[j] = 1; }               \
            if (finished[j] == 1 && j == num_offsets_now - 1 && j > j_low)              \
                num_offsets_now--;                                                      \
        }                                                                               \
        {                                                                               \
            T acc = 0; /* calc_rsq2 :124-140 */                                         \
            const T bl = beta_i[j_low];                                                 \
            for (long i = 0; i < n; ++i) {                                              \
                resid[i] = resid[i] + bl * ttt[i];                                      \
                acc += resid[i] * resid[i];                                             \
            }                                                                           \
            rsq = (double)acc;                                                          \
        }                                                                               \
        if (rsq <= rsqstop) {                                                           \
            for (j = 0; j < num_offsets_now; ++j) /* update_dest :142-159 */            \
                for (long i = 0; i < n; ++i)                                            \
                    t_dest[j][i] = t_dest[j][i] + beta_i[j] * pm[j][i];                 \
            if (parity0 == ORC_EVENODD) { /* :534-543 */                                \
                otherparity = parity0 & 1;                                              \
                parity = 1 - otherparity;                                               \
                parity0 = ORC_EVEN;                                                     \
                iteration = 0;                                                          \
                t_src = in + n;                                                         \
                for (j = 0; j < num_offsets; ++j) t_dest[j] = out[j] + n;               \
                goto start;                                                             \
            }                                                                           \
            for (j = 0; j < num_offsets; j++) {                                         \
                res[j]->final_rsq = (T)rsq / source_norm;                               \
                res[j]->size_r = res[j]->final_rsq;                                     \
                res[j]->size_relr = res[j]->final_rel;                                  \
                res[j]->final_iter = iteration;                                         \
                res[j]->final_restart = nrestart;                                       \
            }                                                                           \
            rc = iteration;                                                             \
            goto done;                                                                  \
        }                                                                               \
        alpha[j_low] = (T)(rsq / oldrsq); /* :587-598 */                                \
        for (j = 0; j < num_offsets_now; j++) if (j != j_low) {                         \
            if (zeta_i[j] * beta_i[j_low] != 0.0)                                       \
                alpha[j] = alpha[j_low] * zeta_ip1[j] * beta_i[j] /                     \
                           (zeta_i[j] * beta_i[j_low]);                                 \
            else { alpha[j] = 0.0; finished[j] = 1; }                                   \
        }                                                                               \
        for (j = 0; j < num_offsets_now; ++j) { /* update_pm :161-184 */                \
            const T bj = beta_i[j], zj = zeta_ip1[j], aj = alpha[j];                    \
            T *d = t_dest[j], *p = pm[j];                                               \
            for (long i = 0; i < n; ++i) {                                              \
                d[i] = d[i] + bj * p[i];                                                \
                T tt = (T)((double)resid[i] * (double)zj);                              \
                p[i] = tt + aj * p[i];                                                  \
            }                                                                           \
        }                                                                               \
        for (j = 0; j < num_offsets_now; j++) {                                         \
            beta_im1[j] = beta_i[j];                                                    \
            zeta_im1[j] = zeta_i[j];                                                    \
            zeta_i[j] = zeta_ip1[j];                                                    \
        }                                                                               \
    } while (iteration < max_cg);                                                       \
    for (j = 0; j < num_offsets; j++) { /* not converged, :626-653 */                   \
        res[j]->final_rsq = (T)rsq / source_norm;                                       \
        res[j]->size_r = res[j]->final_rsq;                                             \
        res[j]->size_relr = res[j]->final_rel;                                          \
        res[j]->final_iter = iteration;                                                 \
        res[j]->final_restart = nrestart;                                               \
    }                                                                                   \
    if (parity0 == ORC_EVENODD) {                                                       \
        otherparity = parity0 & 1;                                                      \
        parity = 1 - otherparity;                                                       \
        parity0 = ORC_EVEN;                                                             \
        t_src = in + n;                                                                 \
        for (j = 0; j < num_offsets; ++j) t_dest[j] = out[j] + n;                       \
        iteration = 0;                                                                  \
        goto start;                                                                     \
    }                                                                                   \
    rc = iteration;                                                                     \
done:                                                                                   \
    info->final_sec = wall_now() - info->final_sec;                                     \
    info->final_flop = (1205. + 15. * num_offsets) * total_iters * (double)g.V;         \
    info->status = 0;                                                                   \
    for (j = 0; j < num_offsets; j++) free(pm[j]);                                      \
    free(pm); free(t_dest); free(ttt); free(ttt_temp); free(resid);                     \
    free(zeta_i); free(zeta_ip1); free(zeta_im1); free(beta_i); free(beta_im1);         \
    free(alpha); free(shifts); free(finished);                                          \
    return rc;                                                                          \
}

ORC_DEFINE(double, d)
ORC_DEFINE(float, f)

/* reconstruct_gauge_third_row, qphix_f3.cpp:1072-1084, applied to every
 * site's 4 forward links: row2 = conj(row0 x row1), negated where the MILC
 * phase of that direction is -1 (x: t odd, y: t+x odd, z: t+x+y odd). */
void orc_reconstruct_third_row_d(const int L[4], double *lng)
{
    const lat_t g = mk_lat(L);
    for (long s = 0; s < g.V; ++s) {
        const int cb = s >= g.Vh;
        const long j = s - cb * g.Vh;
        const int xh = (int)(j % g.nxh);
        long r = j / g.nxh;
        const int y = (int)(r % g.ny); r /= g.ny;
        const int z = (int)(r % g.nz);
        const int t = (int)(r / g.nz);
        const int x = 2 * xh + ((y + z + t + cb) & 1);
        double *gl = lng + 72 * s;
        for (int d = 0; d < 4; ++d) {
            double *m = gl + 18 * d;
            for (int c = 0; c < 3; ++c) {
                const double *a = m + 2 * ((c + 1) % 3), *bb = m + 6 + 2 * ((c + 2) % 3);
                const double *a2 = m + 2 * ((c + 2) % 3), *b2 = m + 6 + 2 * ((c + 1) % 3);
                double re = a[0] * bb[0] - a[1] * bb[1] - (a2[0] * b2[0] - a2[1] * b2[1]);
                double im = -(a[0] * bb[1] + a[1] * bb[0]) + (a2[0] * b2[1] + a2[1] * b2[0]);
                if ((d == 0 && (t & 1)) || (d == 1 && ((t + x) & 1)) || (d == 2 && ((t + x + y) & 1))) {
                    re = -re; im = -im;
                }
                m[12 + 2 * c] = re;
                m[12 + 2 * c + 1] = im;
            }
        }
    }
}
