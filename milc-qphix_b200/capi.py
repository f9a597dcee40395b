"""ctypes mirror of the QPhiX C API (qphix_int.h, qphix_f3.h, qphix_d3.h).

One class, ``QphixLib``, drives any shared library that exports the
reference's ``QPHIX_*`` symbols: the product library ``libqphix_b200.so``
and, in the tests, the reference host code built as ``oracle/_ref``.  The
structures below restate ``QPHIX_layout_t``, ``QPHIX_info_t``,
``QPHIX_invert_arg_t`` and ``QPHIX_resid_arg_t`` (qphix_int.h:30-85) field by
field; the call sequence is MILC's (init -> create_L -> create_V ->
invert/dslash -> extract_V -> destroy).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

QPHIX_SUCCESS, QPHIX_FAIL, QPHIX_MEM_ERROR = 0, 1, 2
QPHIX_EVEN, QPHIX_ODD, QPHIX_EVENODD = 0x02, 0x01, 0x03
PARITY = {"even": QPHIX_EVEN, "odd": QPHIX_ODD, "evenodd": QPHIX_EVENODD}

NODE_NUMBER_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_int))
NODE_INDEX_FN = C.CFUNCTYPE(C.c_size_t, C.POINTER(C.c_int))


class Layout(C.Structure):
    _fields_ = [
        ("node_number", NODE_NUMBER_FN),
        ("node_index", NODE_INDEX_FN),
        ("latdim", C.c_int),
        ("latsize", C.POINTER(C.c_int)),
        ("machdim", C.c_int),
        ("machsize", C.POINTER(C.c_int)),
        ("this_node", C.c_int),
        ("sites_on_node", C.c_size_t),
        ("even_sites_on_node", C.c_size_t),
        ("mpi_comm", C.c_void_p),
    ]


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


def _node_number(coords):
    return 0


def _node_index(coords):
    return 0


_NODE_NUMBER = NODE_NUMBER_FN(_node_number)
_NODE_INDEX = NODE_INDEX_FN(_node_index)


def make_layout(dims, machsize=(1, 1, 1, 1), this_node=0):
    """Layout for the lattice ``dims`` = [Nx, Ny, Nz, Nt] cut into
    ``machsize`` nodes; this process is node ``this_node``."""
    lat = (C.c_int * 4)(*dims)
    mach = (C.c_int * 4)(*machsize)
    V = int(np.prod(dims)) // int(np.prod(machsize))
    lay = Layout(_NODE_NUMBER, _NODE_INDEX, 4, lat, 4, mach, int(this_node), V, V // 2, None)
    lay._keep = (lat, mach)
    return lay


class GaugeCoeffs(C.Structure):
    _fields_ = [("plaquette", C.c_double), ("rectangle", C.c_double),
                ("parallelogram", C.c_double), ("adjoint_plaquette", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("solve_ms", C.c_double), ("iterations", C.c_int),
                ("reliable_updates", C.c_int), ("dslash_launches", C.c_int),
                ("dslash_ms", C.c_double), ("mdagm_launches", C.c_int),
                ("mdagm_ms", C.c_double), ("true_rsq", C.c_double), ("escalated", C.c_int),
                ("links_compressed", C.c_int), ("batch_rhs_per_thread", C.c_int)]


PRECISION = {"half": 0, "single": 1, "double": 2, "half-links": 3}
# QPHIX_B200_dslash_variant precision codes: PRECISION plus FP32 vectors with
# 12-real / 13-real Naik links
TUNE_CODE = dict(PRECISION, **{"single-r12": 4, "single-r13": 5})
# QPHIX_B200_storage_t: vector and link format of an inner-solve operator
STORAGE = {"single": 0, "single-r12": 1, "single-r13": 2, "half-links": 3, "half": 4}


class QphixLib:
    """Calls into one QPHIX_* library; ``prec`` is 'F' (float) or 'D' (double)."""

    def __init__(self, path, mode=C.RTLD_LOCAL):
        self.path = str(path)
        self.lib = C.CDLL(self.path, mode=mode)
        L = self.lib
        L.QPHIX_init.restype = C.c_int
        L.QPHIX_init.argtypes = [C.POINTER(Layout)]
        L.QPHIX_finalize.restype = C.c_int
        for P, real in (("F", C.c_float), ("D", C.c_double)):
            rp = C.POINTER(real)
            f = getattr(L, f"QPHIX_{P}3_create_V_from_raw")
            f.restype, f.argtypes = C.c_void_p, [rp, C.c_int]
            f = getattr(L, f"QPHIX_{P}3_extract_V_to_raw")
            f.restype, f.argtypes = None, [rp, C.c_void_p, C.c_int]
            f = getattr(L, f"QPHIX_{P}3_destroy_V")
            f.restype, f.argtypes = None, [C.c_void_p]
            f = getattr(L, f"QPHIX_{P}3_asqtad_create_L_from_raw")
            f.restype, f.argtypes = C.c_void_p, [rp, rp, rp, rp, C.c_int]
            f = getattr(L, f"QPHIX_{P}3_asqtad_extract_L_to_raw")
            f.restype, f.argtypes = None, [rp, rp, C.c_void_p, C.c_int]
            f = getattr(L, f"QPHIX_{P}3_asqtad_destroy_L")
            f.restype, f.argtypes = None, [C.c_void_p]
            f = getattr(L, f"QPHIX_{P}3_asqtad_dslash")
            f.restype, f.argtypes = None, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
            f = getattr(L, f"QPHIX_{P}3_asqtad_invert")
            f.restype = C.c_int
            f.argtypes = [C.POINTER(Info), C.c_void_p, C.POINTER(InvertArg),
                          C.POINTER(ResidArg), real, C.c_void_p, C.c_void_p]
            f = getattr(L, f"QPHIX_{P}3_asqtad_invert_multi")
            f.restype = C.c_int
            f.argtypes = [C.POINTER(Info), C.c_void_p, C.POINTER(InvertArg),
                          C.POINTER(C.POINTER(ResidArg)), rp, C.c_int,
                          C.POINTER(C.c_void_p), C.c_void_p]
            for obj in ("G", "F"):
                f = getattr(L, f"QPHIX_{P}3_create_{obj}_from_raw")
                f.restype, f.argtypes = C.c_void_p, [rp, C.c_int]
                f = getattr(L, f"QPHIX_{P}3_extract_{obj}_to_raw")
                f.restype, f.argtypes = None, [rp, C.c_void_p, C.c_int]
                f = getattr(L, f"QPHIX_{P}3_destroy_{obj}")
                f.restype, f.argtypes = None, [C.c_void_p]
            f = getattr(L, f"QPHIX_{P}3_symanzik_1loop_gauge_force")
            f.restype = None
            f.argtypes = [C.POINTER(Info), C.c_void_p, C.c_void_p, C.POINTER(GaugeCoeffs), real]

        # QPHIX_B200_* additions (absent from the reference library)
        self.has_b200 = hasattr(L, "QPHIX_B200_version")
        if self.has_b200:
            L.QPHIX_B200_last_error.restype = C.c_char_p
            L.QPHIX_B200_set_inner_precision.argtypes = [C.c_int]
            L.QPHIX_B200_set_reliable_delta.argtypes = [C.c_double]
            L.QPHIX_B200_get_last_stats.argtypes = [C.POINTER(Stats)]
            L.QPHIX_B200_set_kernel_timing.argtypes = [C.c_int]
            L.QPHIX_B200_timer_stop.argtypes = [C.POINTER(C.c_double)]
            for P in ("F", "D"):
                f = getattr(L, f"QPHIX_B200_{P}3_dslash_timed")
                f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                              C.POINTER(C.c_double)]
            L.QPHIX_B200_D3_asqtad_mdagm_noalloc.restype = C.c_int
            L.QPHIX_B200_D3_asqtad_mdagm_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                                             C.c_int, C.POINTER(C.c_double)]
            L.QPHIX_B200_dslash_variant.restype = C.c_int
            L.QPHIX_B200_dslash_variant.argtypes = [C.c_int, C.POINTER(C.c_double)]
            L.QPHIX_B200_mdagm_variant.restype = C.c_int
            L.QPHIX_B200_mdagm_variant.argtypes = [C.c_int, C.POINTER(C.c_double)]
            L.QPHIX_B200_set_dslash_variant.argtypes = [C.c_int]
            L.QPHIX_B200_tuning.restype = C.c_int
            L.QPHIX_B200_tuning.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int]
            L.QPHIX_B200_comm_unique_id.argtypes = [C.c_void_p]
            L.QPHIX_B200_comm_init.argtypes = [C.c_void_p, C.c_int, C.c_int]
            L.QPHIX_B200_set_loopback_halo.argtypes = [C.c_int]
            L.QPHIX_B200_set_wait_limit.argtypes = [C.c_long]
            L.QPHIX_B200_D3_asqtad_dslash_inner.restype = C.c_int
            L.QPHIX_B200_D3_asqtad_dslash_inner.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
            L.QPHIX_B200_D3_asqtad_mdagm_inner.restype = C.c_int
            L.QPHIX_B200_D3_asqtad_mdagm_inner.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                                           C.c_int, C.c_int, C.POINTER(C.c_double)]
            L.QPHIX_B200_D3_batch_dslash.restype = C.c_int
            L.QPHIX_B200_D3_batch_dslash.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                                     C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
                                                     C.POINTER(C.POINTER(C.c_double)),
                                                     C.POINTER(C.POINTER(C.c_double))]
            dpp = C.POINTER(C.POINTER(C.c_double))
            L.QPHIX_B200_D3_batch_create_L.restype = C.c_void_p
            L.QPHIX_B200_D3_batch_create_L.argtypes = [C.c_int, C.POINTER(C.c_int), dpp, dpp, dpp, dpp]
            L.QPHIX_B200_D3_batch_destroy_L.restype = None
            L.QPHIX_B200_D3_batch_destroy_L.argtypes = [C.c_void_p]
            L.QPHIX_B200_D3_batch_invert.restype = C.c_int
            L.QPHIX_B200_D3_batch_invert.argtypes = [C.POINTER(Info), C.c_void_p, C.POINTER(InvertArg),
                                                     C.POINTER(C.POINTER(ResidArg)), C.c_int,
                                                     C.POINTER(C.c_int), C.POINTER(C.c_double), dpp, dpp]
            for P, real in (("F", C.c_float), ("D", C.c_double)):
                f = getattr(L, f"QPHIX_B200_{P}3_asqtad_force")
                f.restype = C.c_int
                f.argtypes = [C.c_void_p, C.c_int, C.POINTER(real), C.POINTER(C.c_void_p), C.c_int,
                              C.POINTER(real), C.POINTER(real)]
            L.QPHIX_B200_neighbor_index.restype = C.c_long
            L.QPHIX_B200_neighbor_index.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_long, C.c_int]

    # -- QPHIX_B200_* ------------------------------------------------------
    @staticmethod
    def _dptrs(arrays):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in arrays]
        ptrs = (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        return ptrs, arrs

    def batch_create_L(self, lattices):
        """``lattices``: list of (dims, links), links a dict of raw FP64
        ``fat, lng, fatback, lngback``.  Returns the batch handle (or None)."""
        n = len(lattices)
        sizes = (C.c_int * (4 * n))(*[int(v) for dims, _ in lattices for v in dims])
        keep, ptrs = [], []
        for key in ("fat", "lng", "fatback", "lngback"):
            p, a = self._dptrs([links[key] for _, links in lattices])
            ptrs.append(p)
            keep.append(a)
        return self.lib.QPHIX_B200_D3_batch_create_L(n, sizes, *ptrs)

    def batch_destroy_L(self, B):
        self.lib.QPHIX_B200_D3_batch_destroy_L(B)

    def batch_invert(self, B, systems, parity="even", max_iter=1000, nrestart=5, resid=1e-20, outs=None):
        """``systems``: list of (lattice index, mass, source raw vector[,
        initial guess]).  ``outs`` (optional): the raw arrays that receive
        the solutions.  Returns (iterations, info, [ResidArg], [solutions])."""
        n = len(systems)
        info = Info()
        inv = InvertArg(PARITY[parity], max_iter, max_iter, nrestart, QPHIX_EVENODD)
        res = [ResidArg(resid, 0, 0, 0, 0, 0, 0, 0) for _ in range(n)]
        res_ptrs = (C.POINTER(ResidArg) * n)(*[C.pointer(r) for r in res])
        lat = (C.c_int * n)(*[int(s[0]) for s in systems])
        mass = (C.c_double * n)(*[float(s[1]) for s in systems])
        srcs = [np.ascontiguousarray(s[2], dtype=np.float64) for s in systems]
        if outs is None:
            outs = [np.array(s[3], dtype=np.float64) if len(s) > 3 else np.zeros_like(srcs[k])
                    for k, s in enumerate(systems)]
        pin, _ = self._dptrs(srcs)
        pout = (C.POINTER(C.c_double) * n)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
        it = self.lib.QPHIX_B200_D3_batch_invert(C.byref(info), B, C.byref(inv), res_ptrs, n, lat, mass, pout, pin)
        return it, info, res, outs

    def force(self, prec, L, xs, coef, parity="even"):
        """Gradient of sum_k coef[k] phi_k^dag M^-1 phi_k with respect to the
        raw fat and Naik links, from the solutions ``xs`` (handles).  Returns
        (grad_fat, grad_lng) in the raw link layout."""
        ct, nt = self._real(prec)
        n = len(xs)
        V = int(np.prod(self.dims))
        gf = np.zeros(V * 72, dtype=nt)
        gl = np.zeros(V * 72, dtype=nt)
        c = np.ascontiguousarray(coef, dtype=nt)
        arr = (C.c_void_p * n)(*xs)
        rc = getattr(self.lib, f"QPHIX_B200_{prec}3_asqtad_force")(
            L, n, c.ctypes.data_as(C.POINTER(ct)), arr, PARITY[parity],
            gf.ctypes.data_as(C.POINTER(ct)), gl.ctypes.data_as(C.POINTER(ct)))
        if rc != 0:
            raise RuntimeError("asqtad_force failed: " + self.last_error())
        return gf, gl

    def last_error(self):
        if not self.has_b200:
            return ""
        return self.lib.QPHIX_B200_last_error().decode()

    def set_inner_precision(self, name):
        return self.lib.QPHIX_B200_set_inner_precision(PRECISION[name])

    def set_link_compression(self, on):
        return self.lib.QPHIX_B200_set_link_compression(1 if on else 0)

    def set_reliable_delta(self, delta):
        return self.lib.QPHIX_B200_set_reliable_delta(delta)

    def last_stats(self):
        s = Stats()
        self.lib.QPHIX_B200_get_last_stats(C.byref(s))
        return s

    def set_kernel_timing(self, on):
        return self.lib.QPHIX_B200_set_kernel_timing(1 if on else 0)

    def timer_start(self):
        return self.lib.QPHIX_B200_timer_start()

    def timer_stop(self):
        ms = C.c_double()
        self.lib.QPHIX_B200_timer_stop(C.byref(ms))
        return ms.value

    def dslash_timed(self, prec, L, out, inp, parity, reps):
        ms = C.c_double()
        rc = getattr(self.lib, f"QPHIX_B200_{prec}3_dslash_timed")(L, out, inp, PARITY[parity], reps,
                                                                   C.byref(ms))
        if rc != 0:
            raise RuntimeError("dslash_timed failed: " + self.last_error())
        return ms.value

    def mdagm_noalloc(self, L, out, inp, mass, parity):
        """QPHIX_B200_D3_asqtad_mdagm_noalloc: (status, in . out)."""
        dot = C.c_double()
        rc = self.lib.QPHIX_B200_D3_asqtad_mdagm_noalloc(L, out, inp, mass, PARITY[parity], C.byref(dot))
        return rc, dot.value

    def dslash_variant(self, prec_name, kernel="dslash"):
        """(variant, [us per variant]) the autotuner chose for the Dslash
        (kernel='dslash') or the fused M^dag M kernel (kernel='mdagm');
        prec_name: a PRECISION name, 'single-r12' or 'single-r13'."""
        us = (C.c_double * 3)()
        f = self.lib.QPHIX_B200_dslash_variant if kernel == "dslash" else self.lib.QPHIX_B200_mdagm_variant
        v = f(TUNE_CODE[prec_name], us)
        return v, list(us)

    def comm_unique_id(self):
        """128-byte NCCL unique id (rank 0 makes it, every rank gets a copy)."""
        buf = C.create_string_buffer(128)
        rc = self.lib.QPHIX_B200_comm_unique_id(buf)
        if rc != 0:
            raise RuntimeError("comm_unique_id failed: " + self.last_error())
        return bytes(buf.raw)

    def comm_init(self, uid, nranks, rank):
        buf = C.create_string_buffer(bytes(uid), 128)
        return self.lib.QPHIX_B200_comm_init(buf, int(nranks), int(rank))

    def comm_finalize(self):
        return self.lib.QPHIX_B200_comm_finalize()

    def set_loopback_halo(self, on):
        """Run one GPU through the decomposed (halo) path."""
        return self.lib.QPHIX_B200_set_loopback_halo(1 if on else 0)

    def tuning(self, prec_name, kernel="dslash"):
        """(variant, [us of variants 0..3]) of the autotuner."""
        us = (C.c_double * 4)()
        v = self.lib.QPHIX_B200_tuning(0 if kernel == "dslash" else 1, TUNE_CODE[prec_name], us, 4)
        return v, list(us)

    def set_dslash_variant(self, variant):
        """Force Dslash variant 0, 1 or 2 everywhere; -1 returns to the autotuner."""
        return self.lib.QPHIX_B200_set_dslash_variant(int(variant))

    def set_wait_limit(self, polls):
        """Poll limit of the TMA pipeline's bounded waits (< 0: the default)."""
        return self.lib.QPHIX_B200_set_wait_limit(int(polls))

    def dslash_inner(self, L, out, inp, parity, storage):
        """QPHIX_B200_D3_asqtad_dslash_inner: the inner solve's Dslash for
        ``storage`` (a STORAGE name) on FP64 handles; returns the status."""
        return self.lib.QPHIX_B200_D3_asqtad_dslash_inner(L, out, inp, PARITY[parity], STORAGE[storage])

    def mdagm_inner(self, L, out, inp, mass, parity, storage):
        """QPHIX_B200_D3_asqtad_mdagm_inner: (status, in . out)."""
        dot = C.c_double()
        rc = self.lib.QPHIX_B200_D3_asqtad_mdagm_inner(L, out, inp, mass, PARITY[parity], STORAGE[storage],
                                                      C.byref(dot))
        return rc, dot.value

    def batch_dslash(self, B, systems, parity="even", op=0, prec="single", rhs_per_thread=0):
        """QPHIX_B200_D3_batch_dslash.  ``systems``: list of (lattice index,
        mass, raw input vector).  Returns (status, [raw outputs])."""
        n = len(systems)
        lat = (C.c_int * n)(*[int(s[0]) for s in systems])
        mass = (C.c_double * n)(*[float(s[1]) for s in systems])
        pin, keep = self._dptrs([s[2] for s in systems])
        outs = [np.zeros_like(k) for k in keep]
        pout = (C.POINTER(C.c_double) * n)(*[o.ctypes.data_as(C.POINTER(C.c_double)) for o in outs])
        rc = self.lib.QPHIX_B200_D3_batch_dslash(B, n, lat, mass, PARITY[parity], int(op), PRECISION[prec],
                                                 int(rhs_per_thread), pout, pin)
        return rc, outs

    def neighbor_index(self, dims, cb, site, k):
        Ld = (C.c_int * 4)(*dims)
        return self.lib.QPHIX_B200_neighbor_index(Ld, cb, site, k)

    # -- helpers -----------------------------------------------------------
    @staticmethod
    def _real(prec):
        return (C.c_float, np.float32) if prec == "F" else (C.c_double, np.float64)

    def _fn(self, prec, name):
        return getattr(self.lib, f"QPHIX_{prec}3_{name}")

    # -- API ---------------------------------------------------------------
    def init(self, dims, machsize=(1, 1, 1, 1), this_node=0):
        """QPHIX_init for the global lattice ``dims``; with several nodes
        ``self.dims`` is this node's slab (the size of its raw arrays)."""
        self._layout = make_layout(dims, machsize, this_node)
        self.dims = tuple(int(d) // int(m) for d, m in zip(dims, machsize))
        return self.lib.QPHIX_init(C.byref(self._layout))

    def finalize(self):
        return self.lib.QPHIX_finalize()

    def create_V(self, prec, raw, evenodd="evenodd"):
        ct, nt = self._real(prec)
        a = np.ascontiguousarray(raw, dtype=nt)
        return self._fn(prec, "create_V_from_raw")(a.ctypes.data_as(C.POINTER(ct)), PARITY[evenodd])

    def extract_V(self, prec, handle, evenodd="evenodd", out=None):
        ct, nt = self._real(prec)
        V = int(np.prod(self.dims))
        if out is None:
            out = np.zeros(V * 6, dtype=nt)
        self._fn(prec, "extract_V_to_raw")(out.ctypes.data_as(C.POINTER(ct)), handle, PARITY[evenodd])
        return out

    def destroy_V(self, prec, handle):
        self._fn(prec, "destroy_V")(handle)

    def create_L(self, prec, links, evenodd="evenodd"):
        ct, nt = self._real(prec)
        arrs = [np.ascontiguousarray(links[k], dtype=nt) for k in ("fat", "lng", "fatback", "lngback")]
        ptrs = [a.ctypes.data_as(C.POINTER(ct)) for a in arrs]
        return self._fn(prec, "asqtad_create_L_from_raw")(*ptrs, PARITY[evenodd])

    def extract_L(self, prec, handle, evenodd="evenodd"):
        ct, nt = self._real(prec)
        V = int(np.prod(self.dims))
        fat = np.zeros(V * 72, dtype=nt)
        lng = np.zeros(V * 72, dtype=nt)
        self._fn(prec, "asqtad_extract_L_to_raw")(fat.ctypes.data_as(C.POINTER(ct)),
                                                   lng.ctypes.data_as(C.POINTER(ct)),
                                                   handle, PARITY[evenodd])
        return fat, lng

    def destroy_L(self, prec, handle):
        self._fn(prec, "asqtad_destroy_L")(handle)

    def create_G(self, prec, raw, evenodd="evenodd"):
        ct, nt = self._real(prec)
        a = np.ascontiguousarray(raw, dtype=nt)
        return self._fn(prec, "create_G_from_raw")(a.ctypes.data_as(C.POINTER(ct)), PARITY[evenodd])

    def create_F(self, prec, raw, evenodd="evenodd"):
        ct, nt = self._real(prec)
        a = np.ascontiguousarray(raw, dtype=nt)
        return self._fn(prec, "create_F_from_raw")(a.ctypes.data_as(C.POINTER(ct)), PARITY[evenodd])

    def _extract72(self, prec, name, handle, evenodd):
        ct, nt = self._real(prec)
        out = np.zeros(int(np.prod(self.dims)) * 72, dtype=nt)
        self._fn(prec, name)(out.ctypes.data_as(C.POINTER(ct)), handle, PARITY[evenodd])
        return out

    def extract_G(self, prec, handle, evenodd="evenodd"):
        return self._extract72(prec, "extract_G_to_raw", handle, evenodd)

    def extract_F(self, prec, handle, evenodd="evenodd"):
        return self._extract72(prec, "extract_F_to_raw", handle, evenodd)

    def destroy_G(self, prec, handle):
        self._fn(prec, "destroy_G")(handle)

    def destroy_F(self, prec, handle):
        self._fn(prec, "destroy_F")(handle)

    def gauge_force(self, prec, G, F, coeffs, eps):
        """QPHIX_*_symanzik_1loop_gauge_force; coeffs: dict of plaquette,
        rectangle, parallelogram.  Returns the info struct."""
        info = Info()
        co = GaugeCoeffs(coeffs.get("plaquette", 0.0), coeffs.get("rectangle", 0.0),
                         coeffs.get("parallelogram", 0.0), coeffs.get("adjoint_plaquette", 0.0))
        self._fn(prec, "symanzik_1loop_gauge_force")(C.byref(info), G, F, C.byref(co), eps)
        return info

    def dslash(self, prec, L, out, inp, parity):
        self._fn(prec, "asqtad_dslash")(L, out, inp, PARITY[parity])

    def invert(self, prec, L, out, inp, mass, parity="even", max_iter=1000, restart=1000,
               nrestart=5, resid=1e-20, relresid=0.0):
        info = Info()
        inv = InvertArg(PARITY[parity], max_iter, restart, nrestart, QPHIX_EVENODD)
        res = ResidArg(resid, 0, relresid, 0, 0, 0, 0, 0)
        it = self._fn(prec, "asqtad_invert")(C.byref(info), L, C.byref(inv), C.byref(res),
                                             mass, out, inp)
        return it, info, res

    def invert_multi(self, prec, L, outs, inp, masses, parity="even", max_iter=1000,
                     restart=1000, nrestart=5, resid=1e-20, relresid=0.0):
        ct, nt = self._real(prec)
        n = len(masses)
        info = Info()
        inv = InvertArg(PARITY[parity], max_iter, restart, nrestart, QPHIX_EVENODD)
        res = [ResidArg(resid, 0, relresid, 0, 0, 0, 0, 0) for _ in range(n)]
        res_ptrs = (C.POINTER(ResidArg) * n)(*[C.pointer(r) for r in res])
        m = np.ascontiguousarray(masses, dtype=nt)
        outs_arr = (C.c_void_p * n)(*outs)
        it = self._fn(prec, "asqtad_invert_multi")(C.byref(info), L, C.byref(inv), res_ptrs,
                                                   m.ctypes.data_as(C.POINTER(ct)), n,
                                                   outs_arr, inp)
        return it, info, res
