"""Generate the golden fixtures of tests/golden from the reference itself.

Runs the reference's own host code (layout remap, neighbour tables, OpenMP
site loop, CG, multi-shift CG, BLAS) compiled as oracle/_ref/libqphix_ref.so
with the restated per-site kernel, on small deterministic inputs, and stores
its outputs:

  golden.json  iteration/restart counts, flop counts, residuals and
               weighted checksums of every output, neighbour-table digests
  dslash_4x4x4x4.npz  one full Dslash output vector (FP64)

Inputs are regenerated from their seeds (milc-qphix_b200/synthetic.py); a
digest of each input is stored so drift of the generator is detected.

Usage (needs the reference sources to build oracle/_ref):
    python tests/golden/make_golden.py
"""
import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import __graft_entry__ as entry  # noqa: E402

entry.load_package()
from milc_qphix_b200 import capi, synthetic  # noqa: E402
import orc  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()[:16]


def weights(n, seed=77):
    return np.random.Generator(np.random.PCG64(seed)).standard_normal(n)


def wsum(v):
    v = np.asarray(v, dtype=np.float64)
    return float(np.dot(v, weights(v.size)))


def main():
    ref = capi.QphixLib(orc.REF_LIB)
    out = {"source": "reference host code (oracle/_ref) + restated per-site kernel", "cases": {}}

    # 1. Dslash on random links, both precisions, three lattices
    for dims in [(4, 4, 4, 4), (8, 4, 4, 8), (8, 8, 8, 8)]:
        links = synthetic.asqtad_links(dims, seed=11)
        src = synthetic.gaussian_source(dims, seed=22, parity="evenodd")
        ref.init(dims)
        for prec in ("D", "F"):
            L = ref.create_L(prec, links)
            vin = ref.create_V(prec, src)
            vout = ref.create_V(prec, np.zeros_like(src))
            ref.dslash(prec, L, vout, vin, "even")
            ref.dslash(prec, L, vout, vin, "odd")
            res = ref.extract_V(prec, vout).astype(np.float64)
            for h in (vin, vout):
                ref.destroy_V(prec, h)
            ref.destroy_L(prec, L)
            key = f"dslash_{'x'.join(map(str, dims))}_{prec}"
            out["cases"][key] = {"dims": dims, "link_seed": 11, "src_seed": 22,
                                 "links_digest": digest(links["fat"]), "src_digest": digest(src),
                                 "wsum": wsum(res), "absmax": float(np.abs(res).max())}
            if dims == (4, 4, 4, 4) and prec == "D":
                np.savez_compressed(os.path.join(HERE, "dslash_4x4x4x4.npz"), out=res)
        ref.finalize()

    # 2. ubench analytic fields (ubench_helper.h:256-364), checksums (:451-487)
    dims = (8, 4, 4, 8)
    f = synthetic.ubench_fields(dims)
    links = {k: f[k] for k in ("fat", "lng", "fatback", "lngback")}
    ref.init(dims)
    L = ref.create_L("D", links)
    vin = ref.create_V("D", f["spinor"])
    vout = ref.create_V("D", np.zeros_like(f["spinor"]))
    ref.dslash("D", L, vout, vin, "even")
    ref.dslash("D", L, vout, vin, "odd")
    res = ref.extract_V("D", vout)
    out["cases"]["ubench_8x4x4x8_D"] = {"dims": dims, "checksum_even": synthetic.ubench_checksum(dims, res, 0),
                                        "checksum_odd": synthetic.ubench_checksum(dims, res, 1)}
    for h in (vin, vout):
        ref.destroy_V("D", h)
    ref.destroy_L("D", L)
    ref.finalize()

    # 3. CG (ks_d_congrad_fn.cpp) on 8^4, m = 0.05
    dims = (8, 8, 8, 8)
    links = synthetic.asqtad_links(dims, seed=1001)
    src = synthetic.gaussian_source(dims, seed=2002, parity="evenodd")
    ref.init(dims)
    for prec, resid in (("D", 1e-20), ("F", 1e-12)):
        for parity in ("even", "odd", "evenodd"):
            L = ref.create_L(prec, links)
            b = ref.create_V(prec, src, parity)
            x = ref.create_V(prec, np.zeros_like(src), parity)
            it, info, r = ref.invert(prec, L, x, b, 0.05, parity=parity, max_iter=1000, nrestart=5, resid=resid)
            xs = ref.extract_V(prec, x, parity).astype(np.float64)
            for h in (b, x):
                ref.destroy_V(prec, h)
            ref.destroy_L(prec, L)
            out["cases"][f"cg_8x8x8x8_{prec}_{parity}"] = {
                "dims": dims, "mass": 0.05, "resid": resid, "max": 1000, "nrestart": 5,
                "links_digest": digest(links["fat"]), "src_digest": digest(src),
                "return": it, "final_iter": r.final_iter, "final_restart": r.final_restart,
                "final_rsq": r.final_rsq, "final_flop": info.final_flop, "wsum": wsum(xs)}
    # relresid path
    L = ref.create_L("D", links)
    b = ref.create_V("D", src, "even")
    x = ref.create_V("D", np.zeros_like(src), "even")
    it, info, r = ref.invert("D", L, x, b, 0.05, parity="even", max_iter=50, nrestart=8, resid=1e-16, relresid=1e-6)
    xs = ref.extract_V("D", x, "even")
    out["cases"]["cg_8x8x8x8_D_even_relresid"] = {
        "dims": dims, "mass": 0.05, "resid": 1e-16, "relresid": 1e-6, "max": 50, "nrestart": 8,
        "return": it, "final_iter": r.final_iter, "final_restart": r.final_restart,
        "final_rsq": r.final_rsq, "final_rel": r.final_rel, "wsum": wsum(xs)}
    for h in (b, x):
        ref.destroy_V("D", h)
    ref.destroy_L("D", L)

    # 4. multi-shift (ks_multicg_offset.cpp) on 8^4, 5 masses, lightest not first
    sig = np.logspace(-3, 0, 5)
    masses = np.sqrt(0.05 ** 2 + sig / 4)
    masses = np.concatenate([masses[2:], masses[:2]])
    for prec, resid in (("D", 1e-20), ("F", 1e-12)):
        for parity in ("even", "evenodd"):
            L = ref.create_L(prec, links)
            b = ref.create_V(prec, src, parity)
            outs = [ref.create_V(prec, np.zeros_like(src), parity) for _ in masses]
            it, info, r = ref.invert_multi(prec, L, outs, b, masses, parity=parity, max_iter=1000, nrestart=5,
                                           resid=resid)
            xs = [ref.extract_V(prec, o, parity).astype(np.float64) for o in outs]
            for h in outs + [b]:
                ref.destroy_V(prec, h)
            ref.destroy_L(prec, L)
            out["cases"][f"multishift_8x8x8x8_{prec}_{parity}"] = {
                "dims": dims, "masses": masses.tolist(), "resid": resid, "max": 1000, "nrestart": 5,
                "return": it, "final_iter": [q.final_iter for q in r], "final_rsq": r[0].final_rsq,
                "final_flop": info.final_flop, "wsum": [wsum(v) for v in xs]}
    ref.finalize()

    # 5. neighbour tables (init_ks_dslash_imp): digest of the real-site entries
    for dims in [(4, 4, 4, 4), (8, 4, 8, 4), (12, 8, 4, 4)]:
        ref.init(dims)
        nt_ptr = C.c_void_p.in_dll(ref.lib, "NeighTableF").value
        pxyz = C.c_int.in_dll(ref.lib, "Pxyzf").value
        vt = C.c_int.in_dll(ref.lib, "Vtf").value
        half = pxyz * vt
        arr = np.ctypeslib.as_array((C.c_uint * (2 * half * 16)).from_address(nt_ptr)).reshape(2, half, 16).copy()
        ref.finalize()
        real = orc.padded_index(dims, np.arange(int(np.prod(dims)) // 2))
        sel = np.ascontiguousarray(arr[:, real]).astype(np.uint32)
        out["cases"]["neigh_" + "x".join(map(str, dims))] = {
            "dims": dims, "sha256": hashlib.sha256(sel.tobytes()).hexdigest()}

    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
