// Lattice geometry and neighbour arithmetic shared by host and device.
//
// The reference precomputes a 16-entry neighbour table per site and parity
// (init_ks_dslash_imp, qphix_misc.cpp:46-230) and the Dslash site loop reads
// it for every output site (ks_long_dslash.cpp:619-622).  On the GPU the
// same indices are computed in registers from the site index, with periodic
// wrap, so no table is streamed from HBM.  The entry order k is the
// reference's: k = 2*dir + (1 for forward, 0 for backward) for the one-hop
// neighbours, 8 + 2*dir + ... for the three-hop (Naik) neighbours, dir =
// x, y, z, t.  The same function serves the host-side export used by the
// bit-exact index tests.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define QB_HD __host__ __device__ __forceinline__
#else
#define QB_HD inline
#endif

namespace qb {

// One parity block: Vh sites with block index
//   j = ((t*Nz + z)*Ny + y)*Nxh + xh,   x = 2*xh + ((y+z+t+cb)&1)
// which is MILC's raw even-first order inside a parity (qphix_f3.cpp:95-100)
// and the reference's internal order without its XY padding
// (ks_long_dslash.cpp:617, Pxy = Vxh*Vy + XY_PAD, ks_config.h:28).
struct Geom {
    int nx, ny, nz, nt;
    int nxh;
    int vh;      // sites per parity block
    int sy;      // block-index stride of y  (= nxh)
    int sz;      // stride of z              (= nxh*ny)
    int st;      // stride of t              (= nxh*ny*nz)
};

inline Geom make_geom(int nx, int ny, int nz, int nt)
{
    Geom g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.nt = nt;
    g.nxh = nx / 2;
    g.sy = g.nxh;
    g.sz = g.nxh * ny;
    g.st = g.nxh * ny * nz;
    g.vh = g.st * nt;
    return g;
}

QB_HD int wrap(int v, int n)
{
    // v is at most two extents outside [0, n) for every extent allowed
    if (v < 0) v += n;
    if (v < 0) v += n;
    if (v >= n) v -= n;
    if (v >= n) v -= n;
    return v;
}

struct SiteCoords {
    int xh, y, z, t, xodd;
};

QB_HD SiteCoords decode(const Geom &g, int cb, int j)
{
    SiteCoords s;
    s.xh = j % g.nxh;
    int r = j / g.nxh;
    s.y = r % g.ny;
    r /= g.ny;
    s.z = r % g.nz;
    s.t = r / g.nz;
    s.xodd = (s.y + s.z + s.t + cb) & 1;
    return s;
}

// Block index (in the opposite parity) of neighbour k of output site s.
QB_HD int neighbor(const Geom &g, const SiteCoords &s, int k)
{
    const int hop = (k < 8) ? 1 : 3;
    const int dir = (k & 7) >> 1;
    const int fwd = k & 1;
    int xh = s.xh, y = s.y, z = s.z, t = s.t;
    switch (dir) {
    case 0:
        // x +/- hop in checkerboard units: xh + xodd - 1 / xh + xodd (one hop),
        // xh + xodd - 2 / xh + xodd + 1 (three hops)
        xh = wrap(s.xh + s.xodd + (fwd ? (hop == 1 ? 0 : 1) : (hop == 1 ? -1 : -2)), g.nxh);
        break;
    case 1: y = wrap(s.y + (fwd ? hop : -hop), g.ny); break;
    case 2: z = wrap(s.z + (fwd ? hop : -hop), g.nz); break;
    default: t = wrap(s.t + (fwd ? hop : -hop), g.nt); break;
    }
    return t * g.st + z * g.sz + y * g.sy + xh;
}

}  // namespace qb
