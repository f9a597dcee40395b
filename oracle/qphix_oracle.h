/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- a plain-C CPU restatement of the
 * milc-qphix staggered solver path, used by the tests, the smoke check and
 * the benchmark's CPU-baseline leg as the checker.  Never linked into, or
 * called by, the product library.
 *
 * Data live in MILC's raw even-first layout (the arrays MILC passes to
 * QPHIX_*_create_*_from_raw):
 *   colour vector  v[6*i + 2*c + ri]                 i in [0, V)
 *   links          u[72*i + 18*dir + 6*row + 2*col + ri]
 *   site index     i = par*V/2 + ((t*Nz+z)*Ny+y)*Nxh + x/2
 * A "parity block" is the V/2-site half of a vector; block index j of parity
 * cb has coordinates x = 2*(j%Nxh) + ((y+z+t+cb)&1), exactly like the
 * reference's internal KS arrays at VECLEN=1 (ks_long_dslash.cpp:614-617)
 * without the XY padding.
 *
 * The solver entry points reproduce the reference control flow statement by
 * statement (see the citations in qphix_oracle.c), including its handling
 * of QPHIX_EVENODD and its fptype-precision reductions.
 */
#ifndef QPHIX_ORACLE_H
#define QPHIX_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* same layouts as QPHIX_info_t / QPHIX_invert_arg_t / QPHIX_resid_arg_t
 * (qphix_int.h:44-85) so one set of ctypes structures serves every library */
typedef struct {
    double final_sec;
    double final_flop;
    int status;
    int count1, count2;
} orc_info_t;

typedef struct {
    int parity;
    int max;
    int restart;
    int nrestart;
    int evenodd;
} orc_invert_arg_t;

typedef struct {
    double resid;
    double final_rsq;
    double relresid;
    double final_rel;
    double size_r;
    double size_relr;
    int final_iter;
    int final_restart;
} orc_resid_arg_t;

/* NeighTable/BoundTable of init_ks_dslash_imp (qphix_misc.cpp:46-230) at
 * VECLEN=1 with XY_PAD=1: entries for padded index
 * ind = t*Pxyz + z*Pxy + y*Nxh + xh, Pxy = Nxh*Ny + 1, Pxyz = Pxy*Nz.
 * table has 2*Pxyz*Nt*16 entries (cb-major), bound 2*Pxyz*Nt*4 bytes.
 * Returns the number of padded sites per parity (Pxyz*Nt). */
long orc_neigh_table(const int L[4], unsigned *table, unsigned char *bound);

/* out_blk[parity cb] = D * in_blk[parity 1-cb]  (qphix_ks_dslash, ks_long_dslash.cpp:564) */
void orc_dslash_d(const int L[4], const double *fat, const double *lng, const double *fatback,
                  const double *lngback, double *out_blk, const double *in_blk, int cb);
void orc_dslash_f(const int L[4], const float *fat, const float *lng, const float *fatback,
                  const float *lngback, float *out_blk, const float *in_blk, int cb);

/* QPHIX_D3/F3_asqtad_dslash semantics on raw vectors (qphix_f3.cpp:1233-1245):
 * parity QPHIX_EVEN(2) writes the even block of out from the odd block of in. */
void orc_asqtad_dslash_d(const int L[4], const double *fat, const double *lng,
                         const double *fatback, const double *lngback, double *out,
                         const double *in, int parity);
void orc_asqtad_dslash_f(const int L[4], const float *fat, const float *lng,
                         const float *fatback, const float *lngback, float *out,
                         const float *in, int parity);

/* QPHIX_*_asqtad_invert (ks_d_congrad_fn.cpp:221-619) on raw vectors */
int orc_invert_d(const int L[4], const double *fat, const double *lng, const double *fatback,
                 const double *lngback, orc_info_t *info, const orc_invert_arg_t *inv,
                 orc_resid_arg_t *res, double mass, double *out, const double *in);
int orc_invert_f(const int L[4], const float *fat, const float *lng, const float *fatback,
                 const float *lngback, orc_info_t *info, const orc_invert_arg_t *inv,
                 orc_resid_arg_t *res, float mass, float *out, const float *in);

/* QPHIX_*_asqtad_invert_multi (ks_multicg_offset.cpp:205-689) on raw vectors */
int orc_invert_multi_d(const int L[4], const double *fat, const double *lng,
                       const double *fatback, const double *lngback, orc_info_t *info,
                       const orc_invert_arg_t *inv, orc_resid_arg_t *res[],
                       const double *mass, int n, double *out[], const double *in);
int orc_invert_multi_f(const int L[4], const float *fat, const float *lng,
                       const float *fatback, const float *lngback, orc_info_t *info,
                       const orc_invert_arg_t *inv, orc_resid_arg_t *res[],
                       const float *mass, int n, float *out[], const float *in);

/* 12-real compression of a raw long-link field and the reconstruction of
 * reconstruct_gauge_third_row (qphix_f3.cpp:1072-1084), applied per site to
 * the 4 forward links, with the staggered-phase sign rule of :1079. */
void orc_reconstruct_third_row_d(const int L[4], double *lng);

#ifdef __cplusplus
}
#endif
#endif
