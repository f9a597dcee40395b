/*
 * qphix_b200.h -- additions of libqphix_b200.so beyond the reference QPhiX
 * C API.  None of these has a counterpart in the reference (which is CPU
 * only); they control how the GPU runs the reference entry points and
 * expose measurements.  All are optional: a MILC build that only includes
 * qphix.h gets the reference behaviour (pure-precision solves).
 */
#ifndef _QPHIX_B200_H
#define _QPHIX_B200_H

#include <qphix_int.h>
#include <qphix_f3.h>
#include <qphix_d3.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Inner (sloppy) precision of QPHIX_D3_asqtad_invert / _invert_multi.
 * DOUBLE:     FP64 throughout with the reference control flow (default).
 * SINGLE:     FP32 inner CG with FP64 reliable updates; FP64 solution, FP64
 *             reductions; converges on the FP64 true residual.
 * HALF:       16-bit inner CG: vectors as 16-bit fixed point with a per-site
 *             norm, 16-bit fixed-point links, FP32 arithmetic and an FP32
 *             partial solution; FP64 reliable updates.
 * HALF_LINKS: FP32 vectors with 16-bit fixed-point links (half the link
 *             bytes of SINGLE); FP64 reliable updates.
 * A 16-bit inner solve that stops reducing the true residual continues
 * with FP32 links and vectors.  QPHIX_GPU_PRECISION=double|single|half|
 * half-links sets the initial value at QPHIX_init. */
typedef enum {
  QPHIX_B200_PREC_HALF = 0,
  QPHIX_B200_PREC_SINGLE = 1,
  QPHIX_B200_PREC_DOUBLE = 2,
  QPHIX_B200_PREC_HALF_LINKS = 3
} QPHIX_B200_precision_t;

QPHIX_status_t QPHIX_B200_set_inner_precision(QPHIX_B200_precision_t p);
QPHIX_B200_precision_t QPHIX_B200_get_inner_precision(void);

/* Reliable-update threshold of the mixed-precision solvers: the FP64 true
 * residual is recomputed when the sloppy residual norm has dropped by this
 * factor since the last update (default 0.2).  The per-shift refinements
 * that end a mixed multi-shift with FP32 links use a quarter of it. */
QPHIX_status_t QPHIX_B200_set_reliable_delta(double delta);

/* Compressed Naik links for the FP32 inner solves of QPHIX_D3_asqtad_invert /
 * _invert_multi (0 = off, the default).  Like the reference's COMPRESSED_12
 * storage of the long links (qphix_f3.cpp:1008-1016), the third row of every
 * Naik link is dropped and rebuilt in the Dslash, here as
 * lambda * conj(row0 x row1), with lambda measured from the FP64 links when
 * the FP32 copy is made:
 *   12-real: lambda = sign * s, one magnitude s for the field and a sign per
 *            link (Naik links SU(3) times one real factor: asqtad);
 *   13-real: one complex lambda per link (U(3) times a real factor per link:
 *            HISQ Naik links built from unitarised links).
 * A field of neither form keeps its 18-real links; QPHIX_B200_get_last_stats
 * reports which was used.  FP64 links and all FP64 arithmetic are
 * unaffected.  Saves 16 % (12-real) or 11 % (13-real) of the FP32 Dslash's
 * bytes.  QPHIX_GPU_LINK_COMPRESSION=1 in the environment sets it at
 * QPHIX_init. */
QPHIX_status_t QPHIX_B200_set_link_compression(int on);

/* Diagnostics of the most recent invert / invert_multi / batch_invert call. */
typedef struct {
  double solve_ms;        /* device time of the call (CUDA events) */
  int iterations;         /* Krylov iterations (all precisions) */
  int reliable_updates;   /* FP64 true-residual recomputations */
  int dslash_launches;    /* plain Dslash launches that did work (timing on) */
  double dslash_ms;       /* their summed device time */
  int mdagm_launches;     /* fused Dslash + M^dag M epilogue launches (timing on) */
  double mdagm_ms;        /* their summed device time */
  double true_rsq;        /* final |b - M x|^2 / |b|^2 (largest over masses) */
  int escalated;          /* 1 if a 16-bit inner solve stalled and continued in FP32 */
  int links_compressed;   /* Naik links of the FP32 inner solve: 0 18-real, 1 12-real, 2 13-real */
  int batch_rhs_per_thread; /* batched solves: systems per thread (4, 2 or 1) the FP32 Dslash tuner chose;
                              QPHIX_B200_BATCH_G=4|2|1 in the environment forces it */
} QPHIX_B200_stats_t;

QPHIX_status_t QPHIX_B200_get_last_stats(QPHIX_B200_stats_t *stats);

/* Per-launch CUDA-event timing of the Dslash kernels inside solves
 * (0 = off, the default). */
QPHIX_status_t QPHIX_B200_set_kernel_timing(int on);

/* Device timer on the library's CUDA stream: start, then stop returns the
 * elapsed milliseconds between the two points of the stream. */
QPHIX_status_t QPHIX_B200_timer_start(void);
QPHIX_status_t QPHIX_B200_timer_stop(double *ms);

/* `reps` back-to-back Dslash launches out[parity] = D in[opposite]
 * timed with CUDA events; *ms_per_call = mean device time of one launch. */
QPHIX_status_t QPHIX_B200_F3_dslash_timed(void *links, void *out, void *in,
                                          QPHIX_evenodd_t parity, int reps,
                                          double *ms_per_call);
QPHIX_status_t QPHIX_B200_D3_dslash_timed(void *links, void *out, void *in,
                                          QPHIX_evenodd_t parity, int reps,
                                          double *ms_per_call);

/* Dslash kernel variant chosen by the library's autotuner for precision p
 * (HALF_LINKS: FP32 vectors with 16-bit links; QPHIX_B200_TUNE_F32_R12 /
 * _R13: FP32 vectors with 12-real / 13-real Naik links):
 * 0 register streaming over a resident grid, 1 register streaming with one
 * thread per site, 2 TMA bulk-copy pipeline.  The first Dslash of each
 * precision and lattice times all three on scratch vectors and keeps the
 * fastest; us[3] receives those timings (microseconds per launch).  Returns
 * -1 before the first Dslash in that precision.  QPHIX_B200_DSLASH=plain|
 * full|tma in the environment forces a variant.  QPHIX_B200_mdagm_variant
 * reports the same for the fused Dslash + M^dag M kernel of the solvers,
 * which is tuned on its own.  With QPHIX_B200_TUNECACHE=<file> in the
 * environment the choices are kept in that file (one line per lattice
 * volume, precision and link storage, tagged with the GPU model) and later
 * processes read them instead of timing again. */
#define QPHIX_B200_TUNE_F32_R12 4
#define QPHIX_B200_TUNE_F32_R13 5
int QPHIX_B200_dslash_variant(int p, double us[3]);
int QPHIX_B200_mdagm_variant(int p, double us[3]);
/* The same for kernel 0 (Dslash) or 1 (fused M^dag M), with the timings of
 * all variants: us[0..n-1] for variants 0..n-1, where variant 3 is the
 * TMA neighbour-tile kernel (the nine (z, t) input planes of each output
 * plane staged in shared memory by cp.async.bulk; FP32 and FP64 vectors,
 * planes of up to 227 KB in all; 0 where a variant does not apply).
 * Returns the chosen variant or -1. */
int QPHIX_B200_tuning(int kernel, int p, double *us, int n);

/* Forces the Dslash variant of every precision (0, 1, 2 as above, 3 the
 * neighbour-tile kernel of QPHIX_B200_tuning; a variant that does not apply
 * to a precision or lattice runs as 1) or, with -1 (the default), lets the
 * autotuner choose.  Same effect as QPHIX_B200_DSLASH=plain|full|tma|tile,
 * which sets the value at load. */
QPHIX_status_t QPHIX_B200_set_dslash_variant(int variant);

/* Poll limit of the bounded mbarrier waits of the TMA-pipeline Dslash
 * (variant 2).  A wait that reaches the limit stops the kernel, which lets
 * the copies it issued land, records the failure in a device error word and
 * returns; the call then reports QPHIX_FAIL and QPHIX_B200_last_error says
 * so.  polls < 0 restores the default (2^22 polls, far longer than any copy
 * takes); 0 gives up at the first wait, which exercises the failure path. */
QPHIX_status_t QPHIX_B200_set_wait_limit(long polls);

/* ---- Operators of the inner solves (no counterpart in the reference) ------
 * The mixed-precision solvers apply the Dslash with lower-precision copies
 * of the links and vectors.  These entry points apply exactly those
 * kernels to FP64 handles, so the inner operators can be compared with
 * the FP64 one element by element:
 *   in[1-parity] is rounded to the storage's vector format, the operator
 *   runs on the storage's link copy, and the result is widened to FP64.
 * QPHIX_B200_STORE_F32_R12 / _R13 need Naik links of that form (see
 * QPHIX_B200_set_link_compression); QPHIX_FAIL otherwise. */
typedef enum {
  QPHIX_B200_STORE_F32 = 0,         /* FP32 vectors, 18-real FP32 links */
  QPHIX_B200_STORE_F32_R12 = 1,     /* FP32 vectors, 12-real Naik links */
  QPHIX_B200_STORE_F32_R13 = 2,     /* FP32 vectors, 13-real Naik links */
  QPHIX_B200_STORE_HALF_LINKS = 3,  /* FP32 vectors, 16-bit fixed-point links */
  QPHIX_B200_STORE_HALF = 4         /* 16-bit vectors (per-site norm) and links */
} QPHIX_B200_storage_t;

/* out[parity] = D in[1-parity] with the inner kernel of `storage`
 * (QPHIX_D3_asqtad_dslash's operator, qphix_f3.cpp:1233-1245). */
QPHIX_status_t QPHIX_B200_D3_asqtad_dslash_inner(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                 QPHIX_D3_ColorVector *in, QPHIX_evenodd_t parity,
                                                 QPHIX_B200_storage_t storage);
/* out[parity] = D D in[parity] - 4 mass^2 in[parity] through the inner
 * solve's two kernels (the plain Dslash, then the fused Dslash with the
 * M^dag M epilogue), *in_dot_out = in . out reduced on the device: the
 * vector and the scalar calc_pkp forms in the reference CG
 * (ks_d_congrad_fn.cpp:159-171). */
QPHIX_status_t QPHIX_B200_D3_asqtad_mdagm_inner(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                QPHIX_D3_ColorVector *in, QPHIX_D_Real mass,
                                                QPHIX_evenodd_t parity, QPHIX_B200_storage_t storage,
                                                double *in_dot_out);

/* Allocation-free application of the CG operator (no counterpart in the
 * reference).  For callers that cannot allocate GPU memory at the point of
 * use -- a memory budget reserved up front, another framework's allocator
 * in charge, or no room for the synchronisation an allocation may cost.
 *   out[parity] = D D in[parity] - 4 mass^2 in[parity]   (= -(4m^2 - D D) in,
 *   the vector the reference CG forms in calc_pkp), *in_dot_out = in . out
 * Its scratch (the intermediate D in, reduction partials) is a fixed array
 * inside the library: at most 262144 sites per parity (larger lattices get
 * QPHIX_FAIL), about 12.6 MB held on every GPU that loads the library until
 * the process exits.  All calls share that array, so calls that overlap on
 * the GPU race.  The first call on each device looks the array up; make it
 * before any stream capture.  The call allocates nothing. */
QPHIX_status_t QPHIX_B200_D3_asqtad_mdagm_noalloc(QPHIX_D3_FermionLinksAsqtad *L, QPHIX_D3_ColorVector *out,
                                                 QPHIX_D3_ColorVector *in, QPHIX_D_Real mass,
                                                 QPHIX_evenodd_t parity, double *in_dot_out);

/* ---- Batched solves (no counterpart in the reference) ----------------------
 * The reference solves one system per QPHIX_D3_asqtad_invert call
 * (ks_d_congrad_fn.cpp:221) on the lattice fixed by QPHIX_init.  A batch
 * holds the gauge fields of nlat <= 16 lattices, each of any size QPHIX_init
 * accepts and independent of the QPHIX_init lattice (which must exist), and
 * solves many systems on them in one device run.
 *
 * QPHIX_B200_D3_batch_create_L: lattice l has extents latsize[4l..4l+3]
 * = {Nx,Ny,Nz,Nt} and raw MILC links fat[l], lng[l], fatback[l],
 * lngback[l] (the layout of QPHIX_D3_asqtad_create_L_from_raw, both
 * parities).  Returns NULL on failure (QPHIX_B200_last_error). */
typedef struct QPHIX_B200_Batch_struct QPHIX_B200_Batch;
QPHIX_B200_Batch *QPHIX_B200_D3_batch_create_L(int nlat, const int *latsize, double *const *fat,
                                               double *const *lng, double *const *fatback,
                                               double *const *lngback);
void QPHIX_B200_D3_batch_destroy_L(QPHIX_B200_Batch *B);

/* Solves (4 mass[k]^2 - D_eo D_oe) x_k = in_k for k = 0..nsys-1 (nsys <= 64)
 * on the sites of parity inv_arg->parity (QPHIX_EVEN or QPHIX_ODD), system
 * k on lattice lat[k].  in[k] and out[k] are raw MILC colour vectors of that
 * lattice (6 reals per site, even sites first); out[k] holds the initial
 * guess and receives the solution on the solve parity.  Inner CG in FP32
 * with FP64 reliable updates (QPHIX_B200_set_reliable_delta); each system
 * stops when its FP64 true residual satisfies |r|^2 <= res_arg[k]->resid
 * |b|^2.  Systems on one lattice share every link load.  At most
 * inv_arg->max * inv_arg->nrestart iterations.  res_arg[k] receives
 * final_rsq (relative, squared), final_iter and final_restart (reliable
 * updates); returns the largest iteration count. */
int QPHIX_B200_D3_batch_invert(QPHIX_info_t *info, QPHIX_B200_Batch *B, QPHIX_invert_arg_t *inv_arg,
                               QPHIX_resid_arg_t **res_arg, int nsys, const int *lat,
                               const double *mass, double *const *out, double *const *in);

/* Applies the batched solver's Dslash kernels to nsys systems in one launch
 * (the operators QPHIX_B200_D3_batch_invert runs), system k on lattice
 * lat[k] of the batch, raw MILC vectors in and out (6 reals per site, even
 * sites first, both parities in the arrays):
 *   op 0: out_k[parity] = D in_k[1-parity]
 *   op 1: out_k[parity] = 4 mass[k]^2 in_k[parity] - D D in_k[parity]
 *         (the inner CG's M p; FP32 only)
 * prec QPHIX_B200_PREC_SINGLE runs the FP32 inner kernels on the batch's
 * FP32 links with `rhs_per_thread` = 4, 2 or 1 systems per thread (0: 4);
 * QPHIX_B200_PREC_DOUBLE the FP64 reliable-update kernel.  The parity of
 * out_k that the operator does not write is left as it was. */
QPHIX_status_t QPHIX_B200_D3_batch_dslash(QPHIX_B200_Batch *B, int nsys, const int *lat, const double *mass,
                                          QPHIX_evenodd_t parity, int op, QPHIX_B200_precision_t prec,
                                          int rhs_per_thread, double *const *out, double *const *in);

/* ---- Fermion force (no counterpart in the reference) -----------------------
 * Gradient of S = sum_k coef[k] phi_k^dag (4 m_k^2 - D_pq D_qp)^{-1} phi_k
 * with respect to the fat and Naik links, given the solutions
 * x[k] = (4 m_k^2 - D_pq D_qp)^{-1} phi_k on parity p = `parity` (EVEN or
 * ODD; e.g. from QPHIX_*_asqtad_invert or the shifts of _invert_multi).
 * The backward links are taken to be the caller's shifted forward links
 * (fatback(x) = fat(x - mu), lngback(x) = lng(x - 3 mu)), so the gradient
 * covers both uses of each link.  grad_fat and grad_lng have the layout of
 * the raw fat and lng arrays (72 reals per site, both parities): entry
 * (site, mu, a, b, re/im) = dS / d(Re or Im of U_mu(site)_ab).  D x is
 * recomputed on the device; the call allocates two raw-layout buffers.
 * Afterwards QPHIX_B200_get_last_stats reports in solve_ms the device time
 * of the force kernels (D x and the outer products, not the copies). */
QPHIX_status_t QPHIX_B200_D3_asqtad_force(QPHIX_D3_FermionLinksAsqtad *L, int n, const double *coef,
                                          QPHIX_D3_ColorVector **x, QPHIX_evenodd_t parity,
                                          double *grad_fat, double *grad_lng);
QPHIX_status_t QPHIX_B200_F3_asqtad_force(QPHIX_F3_FermionLinksAsqtad *L, int n, const float *coef,
                                          QPHIX_F3_ColorVector **x, QPHIX_evenodd_t parity,
                                          float *grad_fat, float *grad_lng);

/* ---- Domain decomposition over several GPUs (no counterpart in this form
 * in the reference) ---------------------------------------------------------
 * The reference runs one MPI rank per node, exchanges the depth-3 faces of
 * the Dslash input before each application (ks_boundary.cpp:185-825) and
 * sums every dot product over the ranks (g_doublesum,
 * ks_blas_utils_c.cpp:101-107).  Here one process drives one GPU and the
 * lattice is cut into slabs along t only: faces go over NVLink with NCCL
 * send/recv into each GPU's own ghost buffer while the interior of the
 * Dslash runs, and the FP64 sums are ncclAllReduce calls.  NCCL is loaded
 * at run time (libnccl.so.2); a single-GPU build needs none.
 * Set-up: rank 0 calls QPHIX_B200_comm_unique_id and hands the 128 bytes to
 * every rank (MPI_Bcast, a shared file, ...); every rank calls
 * QPHIX_B200_comm_init(id, nranks, rank) with QPHIX_GPU_DEVICE naming its
 * GPU, then QPHIX_init with the global latsize, machsize {1, 1, 1, nranks}
 * and this_node = rank.  Nt / nranks must satisfy the QPHIX_init lattice
 * checks (a multiple of 4).  The raw arrays of create/extract are then the
 * rank's own sites in MILC's node-local even-first order, and
 * fatback / lngback are the backward links of those sites (MILC gathers
 * them).  The Dslash, CG and multi-shift CG (FP64 and mixed) run
 * decomposed; the fermion force and the allocation-free operator refuse
 * more than one rank.  QPHIX_B200_comm_finalize after QPHIX_finalize. */
QPHIX_status_t QPHIX_B200_comm_unique_id(void *id128);
QPHIX_status_t QPHIX_B200_comm_init(const void *id128, int nranks, int rank);
QPHIX_status_t QPHIX_B200_comm_finalize(void);

/* One GPU through the decomposed path: with on = 1 every Dslash packs its
 * first and last three t-slices into the ghost buffer and reads its t
 * neighbours beyond the slab from there -- the rank is its own t neighbour,
 * each send buffer being the matching receive buffer, like the
 * reference's ASSUME_MULTINODE (ks_boundary.cpp:196-200, 250-256) -- and
 * every reduction goes through the split (sum over ranks, then finish)
 * path.  Results equal the periodic single-GPU path to rounding.  For
 * testing the decomposition on one GPU. */
QPHIX_status_t QPHIX_B200_set_loopback_halo(int on);

/* Host-side neighbour arithmetic used by the Dslash kernels (no GPU
 * needed): block index, in the opposite parity, of neighbour k of site
 * `site` of parity cb on lattice L[4] = {Nx,Ny,Nz,Nt}.  k follows the
 * reference NeighTable order (qphix_misc.cpp:88-221). */
long QPHIX_B200_neighbor_index(const int L[4], int cb, long site, int k);

/* Message of the last failed call (empty string if none). */
const char *QPHIX_B200_last_error(void);

/* Library version, e.g. 100 for 1.0.0. */
int QPHIX_B200_version(void);

#ifdef __cplusplus
}
#endif
#endif /* _QPHIX_B200_H */
