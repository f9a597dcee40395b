/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * Restated per-site kernel that lets the reference's own host code
 * (layout remap, neighbour tables, site loop, CG, multi-shift, BLAS) be
 * compiled and run here.  The reference takes the body of
 * ks_long_dslash_vec_noinline() from the generated milc-qphix-codegen
 * repository (ks_dslash_complete_specialization.cpp:377 #includes
 * ./ARCH/ks_long_dslash_body_<fp>_<fp>_v<VECLEN>_s<18|12>), which is not
 * vendored, not a submodule and has no pinned version.  This file restates
 * that body for VECLEN=1 from the MILC asqtad/HISQ stencil:
 *
 *   out(x) = sum_mu [ F_mu(x) psi(x+mu)   - B_mu(x)^dag psi(x-mu)  ]
 *          + sum_mu [ L_mu(x) psi(x+3mu)  - LB_mu(x)^dag psi(x-3mu) ]
 *
 * where, per ks_long_dslash.cpp:638-650 and qphix_f3.cpp:998-1018, slot
 * [2*dir+1] of the per-site link block holds the forward link F_dir(x)
 * (MILC `fat`/`lng`) and slot [2*dir] holds the caller-supplied backward
 * link (MILC `fatback`/`lngback`).  MILC's QPhiX glue fills the backward
 * slots with the forward link of the neighbour x-mu (x-3mu for Naik)
 * shifted WITHOUT taking the adjoint, so the kernel applies the adjoint and
 * the minus sign.  Neighbour pointers neighs[k]/neighs3[k] follow the
 * NeighTable order (x-,x+,y-,y+,z-,z+,t-,t+), qphix_misc.cpp:88-221.
 * The output is overwritten, and a direction whose `accumulate` bit is
 * clear is skipped (its contribution arrives through the halo unpack,
 * ks_boundary.cpp:738-825; on one node every bit is set).
 *
 * Also provided: stubs for the two gauge-force kernels whose bodies live in
 * the same absent repository (gauge_force_imp_complete_specialization.cpp
 * :25,74).  The gauge force is outside the solver path; calling it through
 * this oracle library is an error.
 */
#include <cstdio>
#include <cstdlib>
#include "ks_config.h"
#include "ks_globals.h"
#include "ks_dslash_complete_specialization.h"
#include "gauge_force_imp_complete_specialization.h"

namespace {

/* acc += s * U * v   (s = +1) or acc -= U^dag * v   (adj = true) */
template <typename T, typename M>
inline void su3_apply(T acc[3][2], const M &u, const T v[3][2], bool adj)
{
    for (int r = 0; r < 3; ++r) {
        T re = 0, im = 0;
        for (int c = 0; c < 3; ++c) {
            T ur, ui;
            if (!adj) { ur = u[r][c][0][0]; ui = u[r][c][1][0]; }
            else      { ur = u[c][r][0][0]; ui = -u[c][r][1][0]; }
            re += ur * v[c][0] - ui * v[c][1];
            im += ur * v[c][1] + ui * v[c][0];
        }
        if (!adj) { acc[r][0] += re; acc[r][1] += im; }
        else      { acc[r][0] -= re; acc[r][1] -= im; }
    }
}

template <typename T>
inline void load_ks(T v[3][2], const KS *p)
{
    for (int c = 0; c < 3; ++c) { v[c][0] = (*p)[c][0][0]; v[c][1] = (*p)[c][1][0]; }
}

} // namespace

__attribute__((noinline)) void
ks_long_dslash_vec_noinline(int nthreads, KS *oBase, const Gauge18 *gBase,
                            const Gauge *gllBase, KS *neighs[8], KS *neighs3[8],
                            char accumulate, char accumulate3, char isBoundary,
                            char isBoundary3, const int ind_next, const int x,
                            const int y, const int t)
{
    (void)nthreads; (void)isBoundary; (void)isBoundary3; (void)ind_next;
    (void)x; (void)y; (void)t;
#if VECLEN != 1
#error "the restated oracle kernel is written for VECLEN=1"
#endif
#ifdef COMPRESSED_12
#error "the restated oracle kernel is built with 18-real long links only"
#endif
    fptype acc[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    fptype v[3][2];
    for (int d = 0; d < 4; ++d) {
        const int kf = 2 * d + 1, kb = 2 * d;
        if (accumulate & (1 << kf)) { load_ks(v, neighs[kf]); su3_apply(acc, (*gBase)[kf], v, false); }
        if (accumulate & (1 << kb)) { load_ks(v, neighs[kb]); su3_apply(acc, (*gBase)[kb], v, true); }
        if (accumulate3 & (1 << kf)) { load_ks(v, neighs3[kf]); su3_apply(acc, (*gllBase)[kf], v, false); }
        if (accumulate3 & (1 << kb)) { load_ks(v, neighs3[kb]); su3_apply(acc, (*gllBase)[kb], v, true); }
    }
    for (int c = 0; c < 3; ++c) { (*oBase)[c][0][0] = acc[c][0]; (*oBase)[c][1][0] = acc[c][1]; }
}

__attribute__((noinline)) void
gforce_imp_body_vec_noinline(double, Hermit *[8], Gauge *[8], const char, Gauge *, Gauge *,
                             Gauge *, Gauge *, double, double, double, const long, const long,
                             const long, const long)
{
    std::fprintf(stderr, "oracle: gauge force kernel is not part of the solver-path oracle\n");
    std::abort();
}

__attribute__((noinline)) void
update_mg_body_vec_noinline(double, Gauge *, Hermit *, HermitHelperYZT *, const char, const long,
                            const long, const long, const long)
{
    std::fprintf(stderr, "oracle: gauge force kernel is not part of the solver-path oracle\n");
    std::abort();
}
