"""Host-side helpers of the domain-decomposed path: t slabs of MILC raw
arrays and the face/ghost layout of the halo exchange.

The library cuts the lattice into ``P`` slabs along t (QPHIX_init with
machsize {1, 1, 1, P}); rank ``r`` holds t in [r*Lt, (r+1)*Lt), Lt = Nt/P.
Its raw arrays are its own sites in MILC's node-local even-first order
i = ((t'*Nz + z)*Ny + y)*Nxh + xh with the local t' = t - r*Lt.  Lt is a
multiple of 4, so a site's parity (x+y+z+t) is the same in local and
global coordinates and the slab of a global parity block is one
contiguous range of it -- slicing, not a gather.

Before each Dslash the library packs the first and last three t-slices of
the input parity (k_halo_pack): per colour component c, the 3*st sites
(st = Nxh*Ny*Nz sites of one parity per t-slice) of slices 0..2 go to the
previous rank, which keeps them as its forward ghost (t = Lt..Lt+2), and
those of slices Lt-3..Lt-1 go to the next rank as its backward ghost
(t = -3..-1).  `pack_faces` and `extend` restate that layout so the
exchange plumbing can be checked on the host.
"""
from __future__ import annotations

import numpy as np


def slab_dims(dims, nranks):
    nx, ny, nz, nt = (int(d) for d in dims)
    if nt % nranks:
        raise ValueError("Nt must be a multiple of the number of ranks")
    return (nx, ny, nz, nt // nranks)


def _sites_per_slice(dims):
    nx, ny, nz, _ = dims
    return (nx // 2) * ny * nz


def scatter(dims, raw, nranks, rank, per_site):
    """Rank ``rank``'s part of a global raw array (``per_site`` reals per
    site: 6 for colour vectors, 72 for links), in its local order."""
    dims = tuple(int(d) for d in dims)
    V = int(np.prod(dims))
    st = _sites_per_slice(dims)
    lt = slab_dims(dims, nranks)[3]
    raw = np.asarray(raw).reshape(2, V // 2, per_site)
    lo, hi = rank * lt * st, (rank + 1) * lt * st
    return np.ascontiguousarray(raw[:, lo:hi, :]).reshape(-1)


def gather(dims, parts, per_site):
    """Inverse of ``scatter``: the global raw array from every rank's part."""
    dims = tuple(int(d) for d in dims)
    V = int(np.prod(dims))
    P = len(parts)
    blocks = [np.asarray(p).reshape(2, V // 2 // P, per_site) for p in parts]
    return np.concatenate(blocks, axis=1).reshape(-1)


def pack_faces(local_dims, raw, parity):
    """(send_back, send_fwd) of one parity block of a local raw colour
    vector, component-major as the library packs them: array [3][3*st] of
    complex numbers for slices 0..2 and Lt-3..Lt-1."""
    local_dims = tuple(int(d) for d in local_dims)
    Vl = int(np.prod(local_dims))
    st = _sites_per_slice(local_dims)
    lt = local_dims[3]
    cb = 0 if parity == "even" else 1
    v = np.asarray(raw).reshape(2, Vl // 2, 3, 2)[cb]
    z = v[..., 0] + 1j * v[..., 1]                 # [site][c]
    back = np.ascontiguousarray(z[: 3 * st].T)      # [c][3*st]
    fwd = np.ascontiguousarray(z[(lt - 3) * st: lt * st].T)
    return back, fwd


def extend(local_dims, raw, parity, ghost_back, ghost_fwd):
    """The parity block with its ghosts, t = -3 .. Lt+2, as complex [site][c]
    in local order (what the Dslash of the boundary sites reads)."""
    local_dims = tuple(int(d) for d in local_dims)
    Vl = int(np.prod(local_dims))
    cb = 0 if parity == "even" else 1
    v = np.asarray(raw).reshape(2, Vl // 2, 3, 2)[cb]
    z = v[..., 0] + 1j * v[..., 1]
    return np.concatenate([np.asarray(ghost_back).T, z, np.asarray(ghost_fwd).T], axis=0)


def periodic_window(dims, raw, nranks, rank, parity):
    """The same window (t = r*Lt - 3 .. (r+1)*Lt + 2, periodic) cut directly
    out of the global array: what the exchange must reproduce."""
    dims = tuple(int(d) for d in dims)
    V = int(np.prod(dims))
    st = _sites_per_slice(dims)
    nt = dims[3]
    lt = slab_dims(dims, nranks)[3]
    cb = 0 if parity == "even" else 1
    v = np.asarray(raw).reshape(2, V // 2, 3, 2)[cb]
    z = (v[..., 0] + 1j * v[..., 1]).reshape(nt, st, 3)
    ts = [(rank * lt + t) % nt for t in range(-3, lt + 3)]
    return z[ts].reshape(-1, 3)
