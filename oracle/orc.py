"""ORACLE / TEST INFRASTRUCTURE ONLY -- ctypes front end of the plain-C
oracle (qphix_oracle.c, built as _build/liboracle.so).

Functions take and return numpy arrays in MILC's raw layout (see
qphix_oracle.h) and mirror the QPhiX entry points: ``asqtad_dslash``,
``invert``, ``invert_multi``, plus ``neigh_table`` (the reference's
NeighTable restated).  Used by the tests, __graft_entry__.smoke() and the
benchmark's CPU-baseline leg, only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libqphix_ref.so")

PARITY = {"even": 2, "odd": 1, "evenodd": 3}


class Info(C.Structure):
    _fields_ = [("final_sec", C.c_double), ("final_flop", C.c_double),
                ("status", C.c_int), ("count1", C.c_int), ("count2", C.c_int)]


class InvertArg(C.Structure):
    _fields_ = [("parity", C.c_int), ("max", C.c_int), ("restart", C.c_int),
                ("nrestart", C.c_int), ("evenodd", C.c_int)]


class ResidArg(C.Structure):
    _fields_ = [("resid", C.c_double), ("final_rsq", C.c_double),
                ("relresid", C.c_double), ("final_rel", C.c_double),
                ("size_r", C.c_double), ("size_relr", C.c_double),
                ("final_iter", C.c_int), ("final_restart", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            env = dict(os.environ)
            env.pop("CC", None)
            env.pop("CXX", None)
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, env=env,
                           stdout=subprocess.DEVNULL)
        _lib = C.CDLL(LIB)
    return _lib


def _types(prec):
    return (C.c_double, np.float64) if prec == "D" else (C.c_float, np.float32)


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _links(links, nt, ct):
    arrs = [np.ascontiguousarray(links[k], dtype=nt) for k in ("fat", "lng", "fatback", "lngback")]
    return arrs, [_ptr(a, ct) for a in arrs]


def asqtad_dslash(dims, links, vin, parity, prec="D"):
    """QPHIX_*_asqtad_dslash on raw vectors; returns a full raw vector with
    only the output parity block filled."""
    ct, nt = _types(prec)
    Ld = (C.c_int * 4)(*dims)
    arrs, ptrs = _links(links, nt, ct)
    s = np.ascontiguousarray(vin, dtype=nt)
    o = np.zeros_like(s)
    getattr(lib(), "orc_asqtad_dslash_" + prec.lower())(Ld, *ptrs, _ptr(o, ct), _ptr(s, ct), PARITY[parity])
    return o


def invert(dims, links, vin, mass, parity="even", prec="D", max_iter=1000, nrestart=5,
           resid=1e-20, relresid=0.0, x0=None):
    """QPHIX_*_asqtad_invert on raw vectors: (iterations, x, resid_arg)."""
    ct, nt = _types(prec)
    Ld = (C.c_int * 4)(*dims)
    arrs, ptrs = _links(links, nt, ct)
    s = np.ascontiguousarray(vin, dtype=nt)
    o = np.zeros_like(s) if x0 is None else np.array(x0, dtype=nt)
    info = Info()
    inv = InvertArg(PARITY[parity], max_iter, max_iter, nrestart, 3)
    res = ResidArg(resid, 0, relresid, 0, 0, 0, 0, 0)
    fn = getattr(lib(), "orc_invert_" + prec.lower())
    fn.restype = C.c_int
    fn.argtypes = ([C.POINTER(C.c_int)] + [C.POINTER(ct)] * 4 +
                   [C.POINTER(Info), C.POINTER(InvertArg), C.POINTER(ResidArg), ct,
                    C.POINTER(ct), C.POINTER(ct)])
    it = fn(Ld, *ptrs, C.byref(info), C.byref(inv), C.byref(res), mass, _ptr(o, ct), _ptr(s, ct))
    return it, o, res


def invert_multi(dims, links, vin, masses, parity="even", prec="D", max_iter=1000, nrestart=5,
                 resid=1e-20):
    """QPHIX_*_asqtad_invert_multi on raw vectors: (iterations, [x_j], [resid_arg_j], info)."""
    ct, nt = _types(prec)
    Ld = (C.c_int * 4)(*dims)
    arrs, ptrs = _links(links, nt, ct)
    s = np.ascontiguousarray(vin, dtype=nt)
    n = len(masses)
    outs = [np.zeros_like(s) for _ in range(n)]
    info = Info()
    inv = InvertArg(PARITY[parity], max_iter, max_iter, nrestart, 3)
    res = [ResidArg(resid, 0, 0, 0, 0, 0, 0, 0) for _ in range(n)]
    rp = (C.POINTER(ResidArg) * n)(*[C.pointer(r) for r in res])
    op = (C.POINTER(ct) * n)(*[_ptr(o, ct) for o in outs])
    m = np.ascontiguousarray(masses, dtype=nt)
    fn = getattr(lib(), "orc_invert_multi_" + prec.lower())
    fn.restype = C.c_int
    it = fn(Ld, *ptrs, C.byref(info), C.byref(inv), rp, _ptr(m, ct), n, op, _ptr(s, ct))
    return it, outs, res, info


def neigh_table(dims):
    """Restated NeighTable/BoundTable of the reference (VECLEN=1, padded index)."""
    nx, ny, nz, nt = dims
    pxyz = ((nx // 2) * ny + 1) * nz
    half = pxyz * nt
    table = np.zeros(2 * half * 16, dtype=np.uint32)
    bound = np.zeros(2 * half * 4, dtype=np.uint8)
    Ld = (C.c_int * 4)(*dims)
    f = lib().orc_neigh_table
    f.restype = C.c_long
    f(Ld, table.ctypes.data_as(C.POINTER(C.c_uint)), bound.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return table.reshape(2, half, 16), bound.reshape(2, half, 4)


def padded_index(dims, j):
    """Reference internal index (ks_long_dslash.cpp:617, XY_PAD=1) of block index j."""
    nx, ny, nz, nt = dims
    nxh = nx // 2
    pxy = nxh * ny + 1
    pxyz = pxy * nz
    j = np.asarray(j)
    xh = j % nxh
    r = j // nxh
    y = r % ny
    r = r // ny
    z = r % nz
    t = r // nz
    return t * pxyz + z * pxy + y * nxh + xh


def true_residual(dims, links, x, b, mass, parity, prec="D"):
    """|b - (4m^2 - D D) x|^2 / |b|^2 on one parity (FP64 unless prec='F')."""
    other = "odd" if parity == "even" else "even"
    t = asqtad_dslash(dims, links, x, other, prec)
    t = asqtad_dslash(dims, links, t, parity, prec)
    V = int(np.prod(dims))
    sl = slice(0, V * 3) if parity == "even" else slice(V * 3, V * 6)
    r = b[sl] - (4 * mass * mass * x[sl] - t[sl])
    return float(np.dot(r, r) / np.dot(b[sl], b[sl]))
