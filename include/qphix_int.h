/*
 * qphix_int.h -- precision-independent types of the QPhiX C API, as served
 * by the B200 library libqphix_b200.so.
 *
 * Drop-in for the reference header qphix_int.h: every enum value, struct
 * member (names, types, order) and macro below matches it, so MILC code
 * compiled against the reference header links against this library
 * unchanged.  Citations are file:line in the reference (JeffersonLab/milc-qphix).
 */
#ifndef _QPHIX_INT_H
#define _QPHIX_INT_H

#ifdef __cplusplus
extern "C" {
#endif

#include <sys/types.h>

/* return status of every entry point; replaces qphix_int.h:13-17 */
typedef enum {
  QPHIX_SUCCESS = 0,
  QPHIX_FAIL = 1,
  QPHIX_MEM_ERROR /* device or host allocation failed */
} QPHIX_status_t;

/* site subsets; replaces qphix_int.h:19-23 */
typedef enum {
  QPHIX_EVEN = 0x02,
  QPHIX_ODD = 0x01,
  QPHIX_EVENODD = 0x03
} QPHIX_evenodd_t;

typedef float QPHIX_F_Real;   /* qphix_int.h:25 */
typedef double QPHIX_D_Real;  /* qphix_int.h:26 */

#define QPHIX_EXTENDED_LAYOUT

/* lattice layout handed to QPHIX_init; replaces qphix_int.h:30-41.
 * This library runs one lattice per GPU: machsize must be all ones,
 * machdim == latdim == 4, and node_number must be callable. */
typedef struct {
  int (*node_number)(const int coords[]);
  size_t (*node_index)(const int coords[]);
  int latdim;
  int *latsize;
  int machdim;
  int *machsize;
  int this_node;
  size_t sites_on_node;
  size_t even_sites_on_node;
  void *mpi_comm;
} QPHIX_layout_t;
#define QPHIX_LAYOUT_ZERO ((QPHIX_layout_t){NULL,NULL,0,NULL,0,NULL,0,0,0,NULL})

/* per-call diagnostics; replaces qphix_int.h:43-49 */
typedef struct {
  double final_sec;        /* (out) wall seconds of the call */
  double final_flop;       /* (out) flops by the reference's own count */
  QPHIX_status_t status;   /* (out) error status */
  int count1, count2;      /* (out) generic counters */
} QPHIX_info_t;
#define QPHIX_INFO_ZERO ((QPHIX_info_t){0,0,QPHIX_SUCCESS,0,0})

/* gauge-force coefficients; replaces qphix_int.h:51-58 */
typedef struct {
   double plaquette;
   double rectangle;
   double parallelogram;
   double adjoint_plaquette;
} QPHIX_gauge_coeffs_t;
#define QPHIX_GAUGE_COEFFS_ZERO ((QPHIX_gauge_coeffs_t){0.,0.,0.,0.})

/* solver controls shared by all masses; replaces qphix_int.h:61-68.
 * As in the reference solvers (ks_d_congrad_fn.cpp:274-278), `max` is the
 * restart interval and the iteration cap is max*nrestart. */
typedef struct {
  QPHIX_evenodd_t parity;
  int max;
  int restart;
  int nrestart;
  QPHIX_evenodd_t evenodd;
} QPHIX_invert_arg_t;
/* the reference initialiser (qphix_int.h:69), four values for five members */
#define QPHIX_INVERT_ARG_DEFAULT ((QPHIX_invert_arg_t){2000,1000,5,QPHIX_EVENODD})

/* per-mass tolerances and results; replaces qphix_int.h:72-85.
 * resid and relresid are SQUARED tolerances. */
typedef struct {
  double resid;
  double final_rsq;
  double relresid;
  double final_rel;
  double size_r;
  double size_relr;
  int final_iter;
  int final_restart;
} QPHIX_resid_arg_t;
#define QPHIX_RESID_ARG_DEFAULT ((QPHIX_resid_arg_t){1e-6,0,0,0,0,0})

/* initialise / release both precisions; replaces qphix_int.h:91-96 */
QPHIX_status_t QPHIX_init_F(QPHIX_layout_t *layout);
QPHIX_status_t QPHIX_init_D(QPHIX_layout_t *layout);
QPHIX_status_t QPHIX_init(QPHIX_layout_t *layout);
QPHIX_status_t QPHIX_finalize();
QPHIX_status_t QPHIX_finalize_F();
QPHIX_status_t QPHIX_finalize_D();

#ifdef __cplusplus
}
#endif

/* qphix_int.h:99-100 */
#define QPHIX_OPP_PAR(p) ((p)==QPHIX_EVENODD ? (p) : (p)^11)
#define QPHIX_OPP_DIR(d) ((d)&1 ? (d)-1 : (d)+1)
#endif /* _QPHIX_INT_H */
