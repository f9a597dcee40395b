/*
 * qphix_f3.h -- single-precision QPhiX C API served by libqphix_b200.so.
 *
 * Drop-in for the reference header qphix_f3.h: same opaque handle types,
 * same prototypes, same generic-name mapping.  Each prototype cites the
 * reference declaration it replaces (qphix_f3.h:line) and the reference
 * definition whose behaviour it reproduces.  Handles own GPU memory;
 * raw arrays stay caller-owned host memory in MILC's even-first layout.
 * Every call is synchronous on return, like the reference.
 */
#ifndef _QPHIX_F3
#define _QPHIX_F3

#ifdef __cplusplus
extern "C" {
#endif

typedef struct QPHIX_F3_ColorVector_struct        QPHIX_F3_ColorVector;
typedef struct QPHIX_F3_FermionLinksAsqtad_struct QPHIX_F3_FermionLinksAsqtad;
typedef struct QPHIX_F3_GaugeField_struct         QPHIX_F3_GaugeField;
typedef struct QPHIX_F3_Force_struct              QPHIX_F3_Force;

/* qphix_f3.h:18; behaviour of QPHIX_F3_create_V_from_raw, qphix_f3.cpp:63-159.
 * Copies the selected parity blocks of `src` (6 reals/site) to the GPU. */
QPHIX_F3_ColorVector *QPHIX_F3_create_V_from_raw(QPHIX_F_Real *src, QPHIX_evenodd_t evenodd);

/* qphix_f3.h:21; qphix_f3.cpp:474-543.  Copies the blocks the handle holds
 * back to `dest` (the `evenodd` argument is ignored, as in the reference). */
void QPHIX_F3_extract_V_to_raw(QPHIX_F_Real *dest, QPHIX_F3_ColorVector *src, QPHIX_evenodd_t evenodd);

/* qphix_f3.h:32-50.  Gauge-force objects are outside this library's
 * solver path: these entry points exist so a full MILC link resolves;
 * create_* return NULL, the force sets info->status = QPHIX_FAIL. */
QPHIX_F3_Force *QPHIX_F3_create_F_from_raw(QPHIX_F_Real *fwdrawmom, QPHIX_evenodd_t evenodd);
void QPHIX_F3_extract_F_to_raw(QPHIX_F_Real *rawdest, QPHIX_F3_Force *src, QPHIX_evenodd_t evenodd);
void QPHIX_F3_destroy_F(QPHIX_F3_Force *field);
QPHIX_F3_GaugeField *QPHIX_F3_create_G_from_raw(QPHIX_F_Real *fwdrawgauge, QPHIX_evenodd_t evenodd);
void QPHIX_F3_extract_G_to_raw(QPHIX_F_Real *rawdest, QPHIX_F3_GaugeField *src, QPHIX_evenodd_t evenodd);
void QPHIX_F3_destroy_G(QPHIX_F3_GaugeField *field);
void QPHIX_F3_symanzik_1loop_gauge_force(QPHIX_info_t *info, QPHIX_F3_GaugeField *gauge,
                                          QPHIX_F3_Force *force, QPHIX_gauge_coeffs_t *coeffs,
                                          QPHIX_F_Real eps);

/* qphix_f3.h:55; qphix_f3.cpp:954-1070.  fat/lng: forward links at each site
 * (72 reals/site), fatback/lngback: the caller's backward links (the forward
 * link of x-mu, resp. x-3mu, shifted to x without adjoint).  The stencil
 * subtracts adj(backward link) * psi(x-mu) (resp. x-3mu). */
QPHIX_F3_FermionLinksAsqtad *QPHIX_F3_asqtad_create_L_from_raw(QPHIX_F_Real *fat, QPHIX_F_Real *lng,
                                                                 QPHIX_F_Real *fatback, QPHIX_F_Real *lngback,
                                                                 QPHIX_evenodd_t evenodd);

/* qphix_f3.h:58; qphix_f3.cpp:1086-1192.  Writes the forward links back. */
void QPHIX_F3_asqtad_extract_L_to_raw(QPHIX_F_Real *fat, QPHIX_F_Real *lng,
                                        QPHIX_F3_FermionLinksAsqtad *src, QPHIX_evenodd_t evenodd);

/* qphix_f3.h:72,75; qphix_f3.cpp:1194-1214 */
void QPHIX_F3_destroy_V(QPHIX_F3_ColorVector *V);
void QPHIX_F3_asqtad_destroy_L(QPHIX_F3_FermionLinksAsqtad *L);

/* qphix_f3.h:78-81; qphix_f3.cpp:1233-1245.  out[parity] = D in[opposite]. */
void QPHIX_F3_asqtad_dslash(QPHIX_F3_FermionLinksAsqtad *asqtad, QPHIX_F3_ColorVector *out,
                              QPHIX_F3_ColorVector *in, QPHIX_evenodd_t parity);

/* qphix_f3.h:84-90; ks_d_congrad_fn.cpp:221-619.  CG on
 * (4m^2 - D_eo D_oe) out = in; returns the iteration count of the last pass. */
int QPHIX_F3_asqtad_invert(QPHIX_info_t *info, QPHIX_F3_FermionLinksAsqtad *asqtad,
                            QPHIX_invert_arg_t *inv_arg, QPHIX_resid_arg_t *res_arg,
                            QPHIX_F_Real mass, QPHIX_F3_ColorVector *out, QPHIX_F3_ColorVector *in);

/* qphix_f3.h:93-100; ks_multicg_offset.cpp:205-689.  Multi-mass CG:
 * out[j] solves (4 mass[j]^2 - D_eo D_oe) out[j] = in. */
int QPHIX_F3_asqtad_invert_multi(QPHIX_info_t *info, QPHIX_F3_FermionLinksAsqtad *asqtad,
                                  QPHIX_invert_arg_t *inv_arg, QPHIX_resid_arg_t *res_arg[],
                                  QPHIX_F_Real *mass, int num_offsets,
                                  QPHIX_F3_ColorVector *out[], QPHIX_F3_ColorVector *in);

#if QPHIX_Precision == 'F'
#include <qphix_f3_generic.h>
#endif

#ifdef __cplusplus
}
#endif

#endif /* _QPHIX_F3 */
