"""Benchmark: time to |r|/|b| < 1e-10 on one B200 (mixed vs FP64 CG) and the
Dslash's achieved HBM bandwidth.

Workload (one "step" = one solve): even-odd asqtad CG for
(4 m^2 - D_eo D_oe) x = b on a 24^3x48 lattice, mass 0.01, random SU(3)
links exp(i 0.3 H) (fat x0.9, Naik x(-1/24), staggered phases, seeded),
Gaussian source on the even sites, squared relative tolerance 1e-20, with the
FP32 inner solve and FP64 reliable updates (every 0.1 residual drop).  The
FP64 CG and the 16-bit inner variant are timed on the same input.

Arms:
  default           the product library through its C ABI (GPU)
  --impl reference  the reference's own CPU implementation of the path
                    (its host code + the restated per-site kernel,
                    oracle/_ref) on the host cores, on a bounded sample.

Prints one JSON line (rank 0).  Multi-GPU (torchrun): replicas only -- every
rank solves its own copy; the time reported is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import __graft_entry__ as entry  # noqa: E402

entry.load_package()
from milc_qphix_b200 import LIB_PATH, capi, synthetic  # noqa: E402

DIMS = (24, 24, 24, 48)
MASS = 0.01
RESID = 1e-20          # squared: |r|/|b| < 1e-10
MAX_ITER, NRESTART = 20000, 5
LINK_SEED, SRC_SEED = 1001, 2002
DSLASH_BYTES_F32 = 1200  # algorithmic bytes per output site, FP32, 18-real links
DSLASH_BYTES_F64 = 2400
DSLASH_FLOPS = 1146
METRIC = "time to |r|/|b|<1e-10, mixed vs FP64 CG on 1 B200; Dslash HBM GB/s"
WORKLOAD = "asqtad mixed-precision CG 24^3x48 m=0.01 tol 1e-10 (FP32 inner, FP64 reliable updates)"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thr = None

    def start(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                vals = [v.strip() for v in out.split(",")]
                if len(vals) == 6:
                    self.samples.append(vals)
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._thr:
            self._thr.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("gloo", timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def make_inputs(device=None):
    # the eigendecompositions of the generator run on the host (torch CPU)
    links = synthetic.asqtad_links(DIMS, seed=LINK_SEED)
    src = synthetic.gaussian_source(DIMS, seed=SRC_SEED, parity="even")
    return links, src


# ---------------------------------------------------------------- GPU arm --
def run_gpu(args):
    world, rank, local, pg = dist_setup()
    os.environ["QPHIX_GPU_DEVICE"] = str(local)
    import torch

    torch.cuda.set_device(local)
    links, src = make_inputs()
    V = int(np.prod(DIMS))
    Vh = V // 2
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(DIMS) == 0, lib.last_error()
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    assert L and b, lib.last_error()
    zeros = np.zeros_like(src)

    def solve(inner, timed=True):
        lib.set_inner_precision(inner)
        x = lib.create_V("D", zeros, "even")
        lib.timer_start()
        it, info, res = lib.invert("D", L, x, b, MASS, parity="even", max_iter=MAX_ITER, nrestart=NRESTART,
                                   resid=RESID)
        ms = lib.timer_stop()
        st = lib.last_stats()
        assert info.status == 0, lib.last_error()
        return x, ms, res, st

    # reference-equivalent FP64 CG on the same input (also the FP64 solution)
    x64, _, _, _ = solve("double")
    lib.destroy_V("D", x64)
    x64, ms64, res64, st64 = solve("double")
    xsol64 = lib.extract_V("D", x64, "even")[: Vh * 6]
    lib.destroy_V("D", x64)

    for _ in range(args.warmup):
        x, _, _, _ = solve("single")
        lib.destroy_V("D", x)

    clocks = ClockSampler(local)
    barrier(pg)
    clocks.start()
    times, iters, rus, trues = [], [], [], []
    xs_last = None
    for k in range(args.steps):
        x, ms, res, st = solve("single")
        times.append(ms)
        iters.append(st.iterations)
        rus.append(st.reliable_updates)
        trues.append(res.final_rsq)
        if k == args.steps - 1:
            xs_last = lib.extract_V("D", x, "even")[: Vh * 6]
        lib.destroy_V("D", x)
    barrier(pg)
    clk = clocks.stop()
    ms_step = max_over_ranks(pg, float(np.mean(times)))

    # per-kernel CUDA-event durations from one more solve of the same input
    # (events around every launch cost host time, so not inside the timed steps)
    lib.set_kernel_timing(True)
    x, ms_inst, _, st = solve("single")
    lib.destroy_V("D", x)
    lib.set_kernel_timing(False)
    dslash_ms, dslash_n, mdagm_ms, mdagm_n = st.dslash_ms, st.dslash_launches, st.mdagm_ms, st.mdagm_launches

    # 16-bit links with FP32 vectors (one warm-up solve, then one measured)
    xl, _, _, _ = solve("half-links")
    lib.destroy_V("D", xl)
    xl, msl, resl, stl = solve("half-links")
    xsoll = lib.extract_V("D", xl, "even")[: Vh * 6]
    lib.destroy_V("D", xl)

    # 16-bit inner variant (one warm-up solve, then one measured)
    xh, _, _, _ = solve("half")
    lib.destroy_V("D", xh)
    xh, msh, resh, sth = solve("half")
    xsolh = lib.extract_V("D", xh, "even")[: Vh * 6]
    lib.destroy_V("D", xh)

    # end to end through the C ABI with host buffers: create b, x (H2D from
    # pinned host memory), solve, extract x (D2H), all inside the timed region
    pinned_src = torch.from_numpy(src).pin_memory().numpy()
    pinned_zero = torch.zeros(src.shape, dtype=torch.float64).pin_memory().numpy()
    pinned_out = torch.zeros(src.shape, dtype=torch.float64).pin_memory().numpy()
    lib.set_inner_precision("single")
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        barrier(pg)
        t0 = time.perf_counter()
        lib.timer_start()
        bb = lib.create_V("D", pinned_src, "even")
        xx = lib.create_V("D", pinned_zero, "even")
        it, info, res = lib.invert("D", L, xx, bb, MASS, parity="even", max_iter=MAX_ITER, nrestart=NRESTART,
                                   resid=RESID)
        lib.extract_V("D", xx, "even", out=pinned_out)
        ms_dev = lib.timer_stop()
        wall = (time.perf_counter() - t0) * 1e3
        lib.destroy_V("D", bb)
        lib.destroy_V("D", xx)
        e2e.append(max(ms_dev, wall))
    e2e_ms = max_over_ranks(pg, float(np.mean(e2e)))

    # isolated Dslash bandwidth (FP32 and FP64), timed with CUDA events
    vin = lib.create_V("F", np.random.default_rng(1).standard_normal(V * 6))
    vout = lib.create_V("F", np.zeros(V * 6))
    Lf = lib.create_L("F", links)
    ms_f32 = lib.dslash_timed("F", Lf, vout, vin, "even", 50)
    lib.destroy_V("F", vin)
    lib.destroy_V("F", vout)
    lib.destroy_L("F", Lf)
    vin = lib.create_V("D", np.random.default_rng(1).standard_normal(V * 6))
    vout = lib.create_V("D", np.zeros(V * 6))
    ms_f64 = lib.dslash_timed("D", L, vout, vin, "even", 50)
    lib.destroy_V("D", vin)
    lib.destroy_V("D", vout)
    lib.destroy_V("D", b)
    lib.destroy_L("D", L)
    tuning = {name: lib.dslash_variant(name) for name in ("single", "double", "half", "half-links")}
    lib.finalize()

    peak, peak_kind = peaks()
    k1_ms = dslash_ms / max(dslash_n, 1)
    achieved = DSLASH_BYTES_F32 * Vh / (k1_ms * 1e-3) / 1e9
    err_vs_fp64 = float(np.abs(xs_last - xsol64).max() / np.abs(xsol64).max())
    err_half = float(np.abs(xsolh - xsol64).max() / np.abs(xsol64).max())
    err_hl = float(np.abs(xsoll - xsol64).max() / np.abs(xsol64).max())
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = (cpu_baseline_sample(res64.final_iter, links, src)
           if world == 1 and not args.no_cpu_baseline else None)
    line = {
        "metric": METRIC,
        "value": ms_step / 1e3,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 inner / f64 reliable updates",
        "data": "synthetic (seeded random SU(3) links, Gaussian source)",
        "config": {"workload": WORKLOAD, "lattice": "24x24x24x48", "mass": MASS, "resid_sq": RESID,
                   "seeds": {"links": LINK_SEED, "source": SRC_SEED}, "parallelism": f"replicas{world}",
                   "l2": "working set (links 0.76 GB FP32, 1.5 GB FP64) exceeds the 126 MB L2"},
        "solve": {"iterations": int(np.median(iters)), "reliable_updates": int(np.median(rus)),
                  "true_rsq_rel": float(max(trues)), "err_vs_fp64_solution": err_vs_fp64},
        "fp64_cg": {"s": ms64 / 1e3, "iterations": res64.final_iter, "true_rsq_rel": res64.final_rsq,
                    "speedup_mixed_vs_fp64": ms64 / ms_step},
        "half_inner_cg": {"s": msh / 1e3, "iterations": sth.iterations, "reliable_updates": sth.reliable_updates,
                          "true_rsq_rel": resh.final_rsq, "err_vs_fp64_solution": err_half,
                          "escalated_to_fp32": sth.escalated,
                          "storage": "16-bit fixed-point vectors (per-site norm) and links"},
        "half_links_cg": {"s": msl / 1e3, "iterations": stl.iterations, "reliable_updates": stl.reliable_updates,
                          "true_rsq_rel": resl.final_rsq, "err_vs_fp64_solution": err_hl,
                          "escalated_to_fp32": stl.escalated, "storage": "FP32 vectors, 16-bit fixed-point links"},
        "dslash": {"f32_us": ms_f32 * 1e3, "f32_gbs": DSLASH_BYTES_F32 * Vh / (ms_f32 * 1e-3) / 1e9,
                   "f64_us": ms_f64 * 1e3, "f64_gbs": DSLASH_BYTES_F64 * Vh / (ms_f64 * 1e-3) / 1e9,
                   "f32_gflops": DSLASH_FLOPS * Vh / (ms_f32 * 1e-3) / 1e9,
                   "bytes_per_site": {"f32": DSLASH_BYTES_F32, "f64": DSLASH_BYTES_F64},
                   "autotuner": {k: {"variant": ["resident-grid", "full-grid", "tma-pipeline"][v] if v >= 0 else None,
                                     "us": [round(x, 2) for x in us]} for k, (v, us) in tuning.items()}},
        "roofline": {"kernel": "k_dslash<float> (K1) in a solve of the timed workload (CUDA events per launch)",
                     "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     # ncu dram__bytes_read+write of k_dslash<float> at 24^3x32 (264.3 MB,
                     # profiles/k_dslash_f32_24x24x24x32.md) scaled by sites to 24^3x48
                     "traffic": 264.33e6 * Vh / 221184,
                     "launches": int(dslash_n), "avg_launch_us": k1_ms * 1e3},
        "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * Vh * 6 * 8,
                "d2h_bytes_per_step": Vh * 6 * 8},
        "gpu_launches": None,
        "clocks": clk,
        "cpu_baseline": cpu,
    }
    # our kernel launches per step: 4 per iteration + restart/reliable-update kernels
    line["gpu_launches"] = int(np.median(iters)) * 4 + 8 * int(np.median(rus)) + 8
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


# ------------------------------------------------------- reference (CPU) --
def ref_iteration_sample(links, src, n_iter):
    """Time n_iter FP64 CG iterations of the reference's own solver
    (ks_d_congrad_fn.cpp, OpenMP on all host cores) on the full lattice."""
    import orc

    ref = capi.QphixLib(orc.REF_LIB)
    ref.init(DIMS)
    L = ref.create_L("D", links)
    b = ref.create_V("D", src, "even")
    x = ref.create_V("D", np.zeros_like(src), "even")
    t0 = time.perf_counter()
    it, info, res = ref.invert("D", L, x, b, MASS, parity="even", max_iter=n_iter, nrestart=1, resid=RESID)
    dt = time.perf_counter() - t0
    ref.destroy_V("D", b)
    ref.destroy_V("D", x)
    ref.destroy_L("D", L)
    ref.finalize()
    return dt, res.final_iter


def cpu_baseline_sample(full_iters, links=None, src=None, n_iter=12):
    import orc

    if not os.path.exists(orc.REF_LIB):
        return None
    if links is None:
        links, src = make_inputs(None)
    dt, done = ref_iteration_sample(links, src, n_iter)
    per_iter = dt / max(done, 1)
    return {"value": per_iter * full_iters, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
            "sample": f"{done} FP64 CG iterations of the reference solver on the full 24^3x48 lattice "
                      f"({dt:.1f} s), scaled to the {full_iters} iterations the FP64 solve needs"}


def run_reference(args):
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return
    import orc

    if not os.path.exists(orc.REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqphix_ref.so was not built"}))
        return
    links, src = make_inputs(None)
    full_iters = FP64_ITERATIONS
    samples = []
    for k in range(args.warmup + args.steps):
        dt, done = ref_iteration_sample(links, src, args.ref_iters)
        if k >= args.warmup:
            samples.append(dt / max(done, 1) * full_iters)
    v = float(np.mean(samples))
    sample = (f"{args.ref_iters} FP64 CG iterations per step of the reference solver (its host code + restated "
              f"kernel, OpenMP) on the full 24^3x48 lattice, scaled to the {full_iters} iterations of the "
              f"FP64 solve")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random SU(3) links, Gaussian source)",
        "config": {"workload": WORKLOAD, "lattice": "24x24x24x48", "mass": MASS, "resid_sq": RESID},
        "cpu_baseline": {"value": v, "unit": "s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": sample},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# iterations the FP64 CG (reference control flow) needs on this workload; the
# GPU arm measures it on every run and reports it as fp64_cg.iterations
FP64_ITERATIONS = 808


def run_profile_dslash(args):
    """--mode dslash: one FP32 and one FP64 Dslash launch after a warm-up
    (small-lattice capture target for ncu)."""
    dims = tuple(int(v) for v in args.lattice.split("x"))
    links = synthetic.asqtad_links(dims, seed=LINK_SEED)
    V = int(np.prod(dims))
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(dims) == 0, lib.last_error()
    out = {}
    for prec in ("F", "D"):
        L = lib.create_L(prec, links)
        vin = lib.create_V(prec, np.random.default_rng(1).standard_normal(V * 6))
        vout = lib.create_V(prec, np.zeros(V * 6))
        ms = lib.dslash_timed(prec, L, vout, vin, "even", args.reps)
        nbytes = (DSLASH_BYTES_F32 if prec == "F" else DSLASH_BYTES_F64) * (V // 2)
        out[prec] = {"us": ms * 1e3, "gbs": nbytes / (ms * 1e-3) / 1e9,
                     "variant": lib.dslash_variant("single" if prec == "F" else "double")}
        lib.destroy_V(prec, vin)
        lib.destroy_V(prec, vout)
        lib.destroy_L(prec, L)
    lib.finalize()
    print(json.dumps({"mode": "dslash", "lattice": args.lattice, "reps": args.reps, **out}))


def run_profile_mixed(args):
    """--mode mixed: only the timed mixed-precision solves (ncu launch list)."""
    links, src = make_inputs()
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(DIMS) == 0, lib.last_error()
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    lib.set_inner_precision(args.inner)
    res_all = []
    for _ in range(args.warmup + args.steps):
        x = lib.create_V("D", np.zeros_like(src), "even")
        lib.timer_start()
        it, info, res = lib.invert("D", L, x, b, MASS, parity="even", max_iter=MAX_ITER, nrestart=NRESTART,
                                   resid=RESID)
        ms = lib.timer_stop()
        st = lib.last_stats()
        res_all.append({"ms": ms, "iterations": st.iterations, "reliable_updates": st.reliable_updates,
                        "true_rsq_rel": res.final_rsq})
        lib.destroy_V("D", x)
    lib.destroy_V("D", b)
    lib.destroy_L("D", L)
    lib.finalize()
    print(json.dumps({"mode": "mixed", "inner": args.inner, "solves": res_all}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="bench", choices=["bench", "dslash", "mixed"],
                    help="bench: the benchmark line; dslash/mixed: small profiling targets")
    ap.add_argument("--lattice", default="16x16x16x32")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--inner", default="single", choices=["single", "half", "double"])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-iters", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.mode == "dslash":
        run_profile_dslash(args)
        return
    if args.mode == "mixed":
        run_profile_mixed(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
