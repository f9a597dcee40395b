"""CPU: the product library's C ABI -- loads without a GPU, exports every
symbol include/*.h declares, fails cleanly without a GPU, and its Dslash
neighbour arithmetic equals the reference's NeighTable bit for bit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, capi, orc

INCLUDE = os.path.join(ROOT, "include")


def declared_symbols():
    names = set()
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#define[^\n]*", "", text)
        for m in re.finditer(r"\b(QPHIX_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def exported_symbols(path):
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def test_every_declared_symbol_is_exported(product_lib_path):
    decl = declared_symbols()
    assert len(decl) >= 50
    exp = exported_symbols(product_lib_path)
    missing = sorted(decl - exp)
    assert not missing, missing


def test_exports_only_the_c_abi(product_lib_path):
    exp = exported_symbols(product_lib_path)
    assert all(s.startswith("QPHIX_") for s in exp), sorted(s for s in exp if not s.startswith("QPHIX_"))


def test_reference_api_symbols_all_present(product_lib_path, ref_lib):
    """Every QPHIX_* function the reference library defines has a counterpart."""
    ref_syms = {s for s in exported_symbols(orc.REF_LIB) if s.startswith("QPHIX_")}
    assert ref_syms <= exported_symbols(product_lib_path), sorted(ref_syms - exported_symbols(product_lib_path))


def test_loads_and_reports_errors_without_gpu(product_lib_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = capi.QphixLib(product_lib_path)
    assert lib.lib.QPHIX_B200_version() == 100
    # no GPU: init fails with a status, does not abort
    assert lib.init((4, 4, 4, 4)) != 0
    assert "CUDA" in lib.last_error() or "cuda" in lib.last_error()
    # use before init fails cleanly
    assert lib.create_V("D", np.zeros(256 * 6)) is None
    assert "before QPHIX_init" in lib.last_error()


def test_bad_layouts_rejected(product_lib_path):
    """The lattice checks of QPHIX_init (qphix_misc.cpp:455-469, 494-497)
    return QPHIX_FAIL instead of exiting; they run before any device call."""
    lib = capi.QphixLib(product_lib_path)
    for dims in [(6, 4, 4, 4), (8, 6, 4, 4), (8, 4, 4, 2), (0, 4, 4, 4)]:
        assert lib.init(dims) == 1
        assert "QPHIX_init" in lib.last_error()
    lay = capi.make_layout((8, 8, 8, 8))
    mach = (C.c_int * 4)(2, 1, 1, 1)
    lay.machsize = mach
    assert lib.lib.QPHIX_init(C.byref(lay)) == 1
    assert "machsize" in lib.last_error()


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 4, 8, 4), (12, 8, 4, 4), (8, 8, 8, 8)])
def test_device_neighbour_arithmetic_equals_reference_table(product_lib_path, ref_lib, dims):
    """QPHIX_B200_neighbor_index runs the same __host__ __device__ function
    the Dslash kernels use; mapped to the reference's padded internal index it
    must equal NeighTable (qphix_misc.cpp:88-221) for every site, parity and k."""
    lib = capi.QphixLib(product_lib_path)
    ref_lib.init(dims)
    nt_ptr = C.c_void_p.in_dll(ref_lib.lib, "NeighTableD").value
    pxyz = C.c_int.in_dll(ref_lib.lib, "Pxyzd").value
    vt = C.c_int.in_dll(ref_lib.lib, "Vtd").value
    half = pxyz * vt
    table = np.ctypeslib.as_array((C.c_uint * (2 * half * 16)).from_address(nt_ptr)).reshape(2, half, 16).copy()
    ref_lib.finalize()
    vh = int(np.prod(dims)) // 2
    f = lib.lib.QPHIX_B200_neighbor_index
    Ld = (C.c_int * 4)(*dims)
    padded = orc.padded_index(dims, np.arange(vh))
    for cb in (0, 1):
        mine = np.array([[f(Ld, cb, j, k) for k in range(16)] for j in range(vh)])
        assert (mine >= 0).all()
        assert np.array_equal(orc.padded_index(dims, mine), table[cb, padded].astype(np.int64))


def test_neighbour_index_rejects_out_of_range(product_lib_path):
    lib = capi.QphixLib(product_lib_path)
    f = lib.lib.QPHIX_B200_neighbor_index
    Ld = (C.c_int * 4)(4, 4, 4, 4)
    assert f(Ld, 0, 128, 0) == -1
    assert f(Ld, 0, 0, 16) == -1
    assert f(Ld, 2, 0, 0) == -1


def test_gauge_force_entry_points_fail_cleanly(product_lib_path):
    """Without QPHIX_init (and with NULL arguments) the gauge-force entry
    points return QPHIX_FAIL / NULL instead of exiting."""
    lib = capi.QphixLib(product_lib_path)
    info = capi.Info()
    lib.lib.QPHIX_D3_symanzik_1loop_gauge_force.argtypes = [C.POINTER(capi.Info), C.c_void_p, C.c_void_p,
                                                           C.c_void_p, C.c_double]
    lib.lib.QPHIX_D3_symanzik_1loop_gauge_force(C.byref(info), None, None, None, 0.1)
    assert info.status == 1
    lib.lib.QPHIX_F3_create_G_from_raw.restype = C.c_void_p
    assert lib.lib.QPHIX_F3_create_G_from_raw(None, 3) is None


def test_headers_compile_as_c_and_cxx(tmp_path):
    """A MILC-style translation unit including qphix.h builds against the
    headers in C and C++ for both precisions."""
    import subprocess

    src = tmp_path / "milc_tu.c"
    src.write_text("""
#include <qphix.h>
#include <qphix_b200.h>
int probe(QPHIX_info_t *info, QPHIX_FermionLinksAsqtad *L, QPHIX_ColorVector *x, QPHIX_ColorVector *b) {
#ifndef __cplusplus
  /* the reference initialiser puts 2000 in the enum member `parity`; C accepts it */
  QPHIX_invert_arg_t inv = QPHIX_INVERT_ARG_DEFAULT;
  QPHIX_resid_arg_t res = QPHIX_RESID_ARG_DEFAULT;
#else
  QPHIX_invert_arg_t inv = {QPHIX_EVEN, 1000, 1000, 5, QPHIX_EVENODD};
  QPHIX_resid_arg_t res = {1e-6, 0, 0, 0, 0, 0, 0, 0};
#endif
  inv.parity = QPHIX_EVEN;
  return QPHIX_asqtad_invert(info, L, &inv, &res, 0.01, x, b) + QPHIX_B200_version();
}
""")
    for comp, extra in (("gcc", []), ("g++", ["-x", "c++"])):
        for prec in ("1", "2"):
            subprocess.run([comp, *extra, "-c", f"-DQPHIX_PrecisionInt={prec}", "-I", INCLUDE, str(src),
                            "-o", str(tmp_path / "x.o")], check=True)
