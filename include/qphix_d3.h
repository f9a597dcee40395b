/*
 * qphix_d3.h -- double-precision QPhiX C API served by libqphix_b200.so.
 *
 * Drop-in for the reference header qphix_d3.h: same opaque handle types,
 * same prototypes, same generic-name mapping.  Each prototype cites the
 * reference declaration it replaces (qphix_d3.h:line) and the reference
 * definition whose behaviour it reproduces.  Handles own GPU memory;
 * raw arrays stay caller-owned host memory in MILC's even-first layout.
 * Every call is synchronous on return, like the reference.
 */
#ifndef _QPHIX_D3
#define _QPHIX_D3

#ifdef __cplusplus
extern "C" {
#endif

typedef struct QPHIX_D3_ColorVector_struct        QPHIX_D3_ColorVector;
typedef struct QPHIX_D3_FermionLinksAsqtad_struct QPHIX_D3_FermionLinksAsqtad;
typedef struct QPHIX_D3_GaugeField_struct         QPHIX_D3_GaugeField;
typedef struct QPHIX_D3_Force_struct              QPHIX_D3_Force;

/* qphix_d3.h:18; behaviour of QPHIX_D3_create_V_from_raw, qphix_d3.cpp:79-175.
 * Copies the selected parity blocks of `src` (6 reals/site) to the GPU. */
QPHIX_D3_ColorVector *QPHIX_D3_create_V_from_raw(QPHIX_D_Real *src, QPHIX_evenodd_t evenodd);

/* qphix_d3.h:21; qphix_d3.cpp:490-560.  Copies the blocks the handle holds
 * back to `dest` (the `evenodd` argument is ignored, as in the reference). */
void QPHIX_D3_extract_V_to_raw(QPHIX_D_Real *dest, QPHIX_D3_ColorVector *src, QPHIX_evenodd_t evenodd);

/* qphix_d3.h:38-58.  Gauge-force objects are outside this library's
 * solver path: these entry points exist so a full MILC link resolves;
 * create_* return NULL, the force sets info->status = QPHIX_FAIL. */
QPHIX_D3_Force *QPHIX_D3_create_F_from_raw(QPHIX_D_Real *fwdrawmom, QPHIX_evenodd_t evenodd);
void QPHIX_D3_extract_F_to_raw(QPHIX_D_Real *rawdest, QPHIX_D3_Force *src, QPHIX_evenodd_t evenodd);
void QPHIX_D3_destroy_F(QPHIX_D3_Force *field);
QPHIX_D3_GaugeField *QPHIX_D3_create_G_from_raw(QPHIX_D_Real *fwdrawgauge, QPHIX_evenodd_t evenodd);
void QPHIX_D3_extract_G_to_raw(QPHIX_D_Real *rawdest, QPHIX_D3_GaugeField *src, QPHIX_evenodd_t evenodd);
void QPHIX_D3_destroy_G(QPHIX_D3_GaugeField *field);
void QPHIX_D3_symanzik_1loop_gauge_force(QPHIX_info_t *info, QPHIX_D3_GaugeField *gauge,
                                          QPHIX_D3_Force *force, QPHIX_gauge_coeffs_t *coeffs,
                                          QPHIX_D_Real eps);

/* qphix_d3.h:32; qphix_d3.cpp:970-1086.  fat/lng: forward links at each site
 * (72 reals/site), fatback/lngback: the caller's backward links (the forward
 * link of x-mu, resp. x-3mu, shifted to x without adjoint).  The stencil
 * subtracts adj(backward link) * psi(x-mu) (resp. x-3mu). */
QPHIX_D3_FermionLinksAsqtad *QPHIX_D3_asqtad_create_L_from_raw(QPHIX_D_Real *fat, QPHIX_D_Real *lng,
                                                                 QPHIX_D_Real *fatback, QPHIX_D_Real *lngback,
                                                                 QPHIX_evenodd_t evenodd);

/* qphix_d3.h:35; qphix_d3.cpp:1101-1207.  Writes the forward links back. */
void QPHIX_D3_asqtad_extract_L_to_raw(QPHIX_D_Real *fat, QPHIX_D_Real *lng,
                                        QPHIX_D3_FermionLinksAsqtad *src, QPHIX_evenodd_t evenodd);

/* qphix_d3.h:72,75; qphix_d3.cpp:1208-1230 */
void QPHIX_D3_destroy_V(QPHIX_D3_ColorVector *V);
void QPHIX_D3_asqtad_destroy_L(QPHIX_D3_FermionLinksAsqtad *L);

/* qphix_d3.h:78-81; qphix_d3.cpp:1247-1262.  out[parity] = D in[opposite]. */
void QPHIX_D3_asqtad_dslash(QPHIX_D3_FermionLinksAsqtad *asqtad, QPHIX_D3_ColorVector *out,
                              QPHIX_D3_ColorVector *in, QPHIX_evenodd_t parity);

/* qphix_d3.h:84-90; ks_d_congrad_fn.cpp:221-619.  CG on
 * (4m^2 - D_eo D_oe) out = in; returns the iteration count of the last pass. */
int QPHIX_D3_asqtad_invert(QPHIX_info_t *info, QPHIX_D3_FermionLinksAsqtad *asqtad,
                            QPHIX_invert_arg_t *inv_arg, QPHIX_resid_arg_t *res_arg,
                            QPHIX_D_Real mass, QPHIX_D3_ColorVector *out, QPHIX_D3_ColorVector *in);

/* qphix_d3.h:93-100; ks_multicg_offset.cpp:205-689.  Multi-mass CG:
 * out[j] solves (4 mass[j]^2 - D_eo D_oe) out[j] = in. */
int QPHIX_D3_asqtad_invert_multi(QPHIX_info_t *info, QPHIX_D3_FermionLinksAsqtad *asqtad,
                                  QPHIX_invert_arg_t *inv_arg, QPHIX_resid_arg_t *res_arg[],
                                  QPHIX_D_Real *mass, int num_offsets,
                                  QPHIX_D3_ColorVector *out[], QPHIX_D3_ColorVector *in);

#if QPHIX_Precision == 'D'
#include <qphix_d3_generic.h>
#endif

#ifdef __cplusplus
}
#endif

#endif /* _QPHIX_D3 */
