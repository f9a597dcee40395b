"""Benchmark: time to |r|/|b| < 1e-10 on one B200 (mixed vs FP64 CG) and the
Dslash's achieved HBM bandwidth.

Workload (one "step" = one solve): even-odd asqtad CG for
(4 m^2 - D_eo D_oe) x = b on a 24^3x48 lattice, mass 0.01, random SU(3)
links exp(i 0.3 H) (fat x0.9, Naik x(-1/24), staggered phases, seeded),
Gaussian source on the even sites, squared relative tolerance 1e-20, with the
FP32 inner solve (12-real Naik links, third rows rebuilt in the Dslash) and
FP64 reliable updates (every 0.1 residual drop).  The FP64 CG, the FP32 inner
solve with 18-real links and the 16-bit variants are timed on the same input.

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
RU_DELTA = 0.1         # reliable update at every 0.1 drop of |r| (24^3x48 workload)
DSLASH_BYTES_F32 = 1200  # algorithmic bytes per output site, FP32, 18-real links
DSLASH_BYTES_F64 = 2400
DSLASH_BYTES_R12 = 1012  # FP32 with 12-real Naik links: 8x72 + 8x48 + 4 (sign word) + 48
# DRAM bytes per output site of one K1 launch measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum / Vh): 264.33 MB at 24^3x32
K1_TRAFFIC_PER_SITE_F32 = 264.33e6 / 221184
# 332.36 MB (327.83 read + 4.53 write) at 24^3x48 for the pipelined k_dslash<float, Recon12>
K1_TRAFFIC_PER_SITE_R12 = 332.361728e6 / 331776
DSLASH_FLOPS = 1146
METRIC = "time to |r|/|b|<1e-10, mixed vs FP64 CG on 1 B200; Dslash HBM GB/s"
VARIANTS = ["resident-grid", "full-grid", "tma-link-pipeline", "tma-neighbour-tiles"]
WORKLOAD = ("asqtad mixed-precision CG 24^3x48 m=0.01 tol 1e-10 (FP32 inner with 12-real Naik links, "
            "FP64 reliable updates)")


def bench_config(world, dims=DIMS):
    """The workload's config object, printed identically by both arms."""
    return {"workload": WORKLOAD, "lattice": "x".join(map(str, dims)), "mass": MASS, "resid_sq": RESID,
            "reliable_delta": RU_DELTA, "seeds": {"links": LINK_SEED, "source": SRC_SEED},
            "parallelism": f"replicas{world}",
            "l2": "working set (FP32 links 0.64 GB with 12-real Naik links, 0.76 GB with 18; FP64 1.5 GB) exceeds "
                  "the 126 MB L2"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.

    NVML (read-only queries: SM clock, max SM clock, active clock-event
    reasons) every 20 ms; nvidia-smi every 200 ms when NVML is missing."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    BITS = (0x8, 0x40, 0x20, 0x4)

    def __init__(self, index):
        self.index = index
        self.samples = []  # (sm_mhz, max_mhz, [active flags in NAMES order])
        self._stop = threading.Event()
        self._thr = None
        self._nvml = None
        try:
            import pynvml

            pynvml.nvmlInit()
            h = None
            try:
                import torch

                uuid = str(torch.cuda.get_device_properties(index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._nvml = (pynvml, h)
        except Exception:
            self._nvml = None

    def start(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()

    def _sample_nvml(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.samples.append((float(sm), float(mx), [bool(r & b) for b in self.BITS]))

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=5).stdout.strip()
        v = [x.strip() for x in out.split(",")]
        if len(v) == 6 and v[0].replace(".", "").isdigit() and v[1].replace(".", "").isdigit():
            self.samples.append((float(v[0]), float(v[1]), [x.lower() == "active" for x in v[2:]]))

    def _run(self):
        period = 0.02 if self._nvml else 0.2
        while not self._stop.is_set():
            try:
                self._sample_nvml() if self._nvml else self._sample_smi()
            except Exception:
                pass
            self._stop.wait(period)

    def stop(self):
        self._stop.set()
        if self._thr:
            self._thr.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples]
        reasons = sorted({self.NAMES[i] for s in self.samples for i in range(4) if s[2][i]})
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": reasons,
                "samples": len(self.samples), "source": "nvml" if self._nvml else "nvidia-smi"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        if not dist.is_initialized():
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


def make_inputs(device=None, dims=DIMS):
    # the eigendecompositions of the generator run on the host (torch CPU)
    # unless a device is given
    links = synthetic.asqtad_links(dims, seed=LINK_SEED, device=device)
    src = synthetic.gaussian_source(dims, seed=SRC_SEED, parity="even")
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
    lib.set_reliable_delta(RU_DELTA)  # the workload's reliable-update threshold
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

    # the timed solves: FP32 inner solve with 12-real Naik links (the
    # workload's long links are SU(3) times -1/24, so the third rows rebuild
    # exactly; the library checks that and reports it in links_compressed)
    lib.set_link_compression(True)
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
    compressed = bool(st.links_compressed)
    k1_bytes = DSLASH_BYTES_R12 if compressed else DSLASH_BYTES_F32
    lib.set_link_compression(False)

    # the same FP32 inner solve with 18-real links (warm-up, measured, instrumented)
    xr, _, _, _ = solve("single")
    lib.destroy_V("D", xr)
    ms18 = None
    for _ in range(2):
        xr, ms, res18, st18 = solve("single")
        ms18 = ms if ms18 is None else min(ms18, ms)
        xsol18 = lib.extract_V("D", xr, "even")[: Vh * 6]
        lib.destroy_V("D", xr)
    lib.set_kernel_timing(True)
    xr, _, _, st18i = solve("single")
    lib.destroy_V("D", xr)
    lib.set_kernel_timing(False)

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

    # end to end through the C ABI with host buffers, as MILC calls it on
    # every solve: create L from the raw host links (H2D of 4 x 72 reals per
    # site, the 12-real check and pack happen inside the solve), create b
    # and x (H2D from pinned host memory), solve, extract x (D2H), destroy.
    # All of it is inside the timed region.
    pinned_src = torch.from_numpy(src).pin_memory().numpy()
    pinned_zero = torch.zeros(src.shape, dtype=torch.float64).pin_memory().numpy()
    pinned_out = torch.zeros(src.shape, dtype=torch.float64).pin_memory().numpy()
    pinned_links = {k: torch.from_numpy(links[k]).pin_memory().numpy() for k in ("fat", "lng", "fatback", "lngback")}
    lib.set_inner_precision("single")
    lib.set_link_compression(True)  # as in the timed solves

    def e2e_step(with_links):
        barrier(pg)
        t0 = time.perf_counter()
        lib.timer_start()
        LL = lib.create_L("D", pinned_links) if with_links else L
        bb = lib.create_V("D", pinned_src, "even")
        xx = lib.create_V("D", pinned_zero, "even")
        it, info, res = lib.invert("D", LL, xx, bb, MASS, parity="even", max_iter=MAX_ITER, nrestart=NRESTART,
                                   resid=RESID)
        lib.extract_V("D", xx, "even", out=pinned_out)
        lib.destroy_V("D", bb)
        lib.destroy_V("D", xx)
        if with_links:
            lib.destroy_L("D", LL)
        ms_dev = lib.timer_stop()
        wall = (time.perf_counter() - t0) * 1e3
        assert info.status == 0, lib.last_error()
        return max(ms_dev, wall), res.final_rsq

    e2e_step(True)  # first upload of this size: pinned staging and pool growth
    n_e2e = max(1, min(args.steps, 5))
    e2e_runs = [e2e_step(True) for _ in range(n_e2e)]
    e2e = [t for t, _ in e2e_runs]
    e2e_rsq = max(r for _, r in e2e_runs)
    e2e_ms = max_over_ranks(pg, float(np.mean(e2e)))
    e2e_res = [e2e_step(False)[0] for _ in range(n_e2e)]
    e2e_res_ms = max_over_ranks(pg, float(np.mean(e2e_res)))
    link_bytes = 4 * V * 72 * 8
    lib.set_link_compression(False)

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
    tuning = {name: lib.tuning(name) for name in ("single", "single-r12", "double", "half", "half-links")}
    tuning_k2 = {name: lib.tuning(name, "mdagm") for name in ("single", "single-r12", "double", "half", "half-links")}
    lib.finalize()
    # the north-star size in the same run: 32^3x64, HISQ-shaped links,
    # m = 0.0012 -- FP64 and mixed CG, FP64 and mixed 12-shift multi-shift
    # (one GPU only: the scaling runs time the headline workload alone)
    target = None
    batch = None
    if not args.no_target and world == 1:
        t = multishift_workload(MS_DIMS, 2, {"fp64_cg", "mixed_cg_single", "fp64_multishift",
                                             "mixed_multishift_single"}, True, False, notes=False)
        target = {k: t[k] for k in ("workload", "lattice", "mass", "sigmas", "resid_sq", "reliable_delta",
                                    "fp64_cg", "mixed_cg_single", "fp64_multishift", "mixed_multishift_single")}
        target["timing"] = ("device time of each solve (CUDA events on the library stream), inputs resident, "
                            "the second of two solves; true residuals recomputed through the FP64 Dslash")
    if not args.no_batch and world == 1:
        bw = batch_workload(None, steps=1, warmup=1, sequential=True, notes=False)
        batch = {k: bw[k] for k in ("workload", "systems", "lattices", "batch_s", "sequential_s",
                                    "speedup_vs_sequential", "rhs_per_thread", "true_rsq_rel_max", "timing")}

    peak, peak_kind = peaks()
    k1_ms = dslash_ms / max(dslash_n, 1)
    achieved = k1_bytes * Vh / (k1_ms * 1e-3) / 1e9
    # K2 reads what K1 reads plus p and writes ttt: 24 more bytes per site
    k2_bytes = k1_bytes + 24
    k2_ms = mdagm_ms / max(mdagm_n, 1)
    k2_achieved = k2_bytes * Vh / (k2_ms * 1e-3) / 1e9
    err_vs_fp64 = float(np.abs(xs_last - xsol64).max() / np.abs(xsol64).max())
    err_half = float(np.abs(xsolh - xsol64).max() / np.abs(xsol64).max())
    err_hl = float(np.abs(xsoll - xsol64).max() / np.abs(xsol64).max())
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    cpu = cpu_baseline_sample(links, src) if world == 1 and not args.no_cpu_baseline else None
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
        "config": bench_config(world),
        "solve": {"ms_each": [round(t, 3) for t in times], "links_compressed": compressed,
                  "iterations": int(np.median(iters)), "reliable_updates": int(np.median(rus)),
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
        "mixed_cg_18real_links": {
            "s": ms18 / 1e3, "iterations": st18.iterations, "reliable_updates": st18.reliable_updates,
            "true_rsq_rel": res18.final_rsq,
            "err_vs_fp64_solution": float(np.abs(xsol18 - xsol64).max() / np.abs(xsol64).max()),
            "k1_us": st18i.dslash_ms / max(st18i.dslash_launches, 1) * 1e3,
            "k1_gbs": DSLASH_BYTES_F32 * Vh / (st18i.dslash_ms / max(st18i.dslash_launches, 1) * 1e-3) / 1e9,
            "speedup_vs_fp64": ms64 / ms18, "storage": "FP32 vectors and 18-real FP32 links"},
        "dslash": {"f32_us": ms_f32 * 1e3, "f32_gbs": DSLASH_BYTES_F32 * Vh / (ms_f32 * 1e-3) / 1e9,
                   "f64_us": ms_f64 * 1e3, "f64_gbs": DSLASH_BYTES_F64 * Vh / (ms_f64 * 1e-3) / 1e9,
                   "f32_gflops": DSLASH_FLOPS * Vh / (ms_f32 * 1e-3) / 1e9,
                   "bytes_per_site": {"f32": DSLASH_BYTES_F32, "f64": DSLASH_BYTES_F64},
                   "autotuner": {k: {"variant": VARIANTS[v] if v >= 0 else None,
                                     "us": [round(x, 2) for x in us]} for k, (v, us) in tuning.items()},
                   "autotuner_k2": {k: {"variant": VARIANTS[v] if v >= 0 else None,
                                        "us": [round(x, 2) for x in us]} for k, (v, us) in tuning_k2.items()}},
        "roofline": {"kernel": ("k_dslash<float, Recon12>" if compressed else "k_dslash<float, float>")
                               + " (K1) in a solve of the timed workload (CUDA events per launch)",
                     "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "algorithmic_bytes_per_site": k1_bytes,
                     # ncu dram__bytes_read+write per output site of one K1 launch
                     # (profiles/), times the sites of this lattice
                     "traffic": (None if (compressed and K1_TRAFFIC_PER_SITE_R12 is None) else
                                 (K1_TRAFFIC_PER_SITE_R12 if compressed else K1_TRAFFIC_PER_SITE_F32) * Vh),
                     "launches": int(dslash_n), "avg_launch_us": k1_ms * 1e3},
        "roofline_k2": {"kernel": ("k_dslash_mdagm<float, Recon12>" if compressed else "k_dslash_mdagm<float, float>")
                                  + " (K2: Dslash + M^dag M epilogue + p.Mp reduction) in a solve of the timed "
                                    "workload (CUDA events per launch)",
                        "bound": "hbm", "achieved": k2_achieved, "peak": peak, "unit": "GB/s",
                        "frac": k2_achieved / peak, "peak_source": peak_kind,
                        "algorithmic_bytes_per_site": k2_bytes, "launches": int(mdagm_n),
                        "avg_launch_us": k2_ms * 1e3},
        "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": link_bytes + 2 * Vh * 6 * 8,
                "d2h_bytes_per_step": Vh * 6 * 8, "steps": n_e2e, "true_rsq_rel": e2e_rsq,
                "what": "QPHIX_D3_asqtad_create_L_from_raw (raw FP64 links from pinned host memory), "
                        "create_V of b and x, invert (mixed, 12-real Naik check and pack included), "
                        "extract_V, destroy: every step, wall clock and device timer, the larger"},
        "e2e_links_resident": {"value": e2e_res_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * Vh * 6 * 8,
                               "d2h_bytes_per_step": Vh * 6 * 8, "steps": n_e2e,
                               "what": "as e2e with the link handle created once, outside the timed region"},
        "gpu_launches": None,
        "clocks": clk,
        "cpu_baseline": cpu,
        "target_32x32x32x64": target,
        "config4_batch": batch,
    }
    # our kernel launches per step: 4 per iteration + restart/reliable-update kernels
    line["gpu_launches"] = int(np.median(iters)) * 4 + 8 * int(np.median(rus)) + 8
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


# ------------------------------------------------------- reference (CPU) --
class _StdoutToStderr:
    """The reference host code prints progress lines to stdout; while it runs
    inside the GPU arm they go to stderr, so stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


class RefSolver:
    """The reference's own FP64 CG (QPHIX_D3_asqtad_invert of its host code
    plus the restated per-site kernel, oracle/_ref; OpenMP on all host
    cores) with the links resident, as the GPU arm's timed solves are."""

    def __init__(self, links, src, dims=DIMS):
        import orc

        self.ref = capi.QphixLib(orc.REF_LIB)
        with _StdoutToStderr():
            assert self.ref.init(dims) == 0
            self.L = self.ref.create_L("D", links)
            self.b = self.ref.create_V("D", src, "even")
        self.src = src

    def solve(self, max_iter=MAX_ITER, nrestart=NRESTART, mass=MASS):
        """One solve to |r|/|b| < 1e-10 (or max_iter * nrestart iterations):
        (seconds, iterations, final |r|^2/|b|^2)."""
        with _StdoutToStderr():
            x = self.ref.create_V("D", np.zeros_like(self.src), "even")
            t0 = time.perf_counter()
            it, info, res = self.ref.invert("D", self.L, x, self.b, mass, parity="even", max_iter=max_iter,
                                            nrestart=nrestart, resid=RESID)
            dt = time.perf_counter() - t0
            self.ref.destroy_V("D", x)
        return dt, res.final_iter, res.final_rsq

    def close(self):
        with _StdoutToStderr():
            self.ref.destroy_V("D", self.b)
            self.ref.destroy_L("D", self.L)
            self.ref.finalize()


def cpu_threads():
    n = os.environ.get("OMP_NUM_THREADS")
    return int(n) if n and n.isdigit() else os.cpu_count()


def cpu_baseline_sample(links=None, src=None):
    """One full FP64 CG solve of the reference solver on the benchmark input
    (measured, 10-30 s on 16 host cores)."""
    import orc

    if not os.path.exists(orc.REF_LIB):
        return None
    if links is None:
        links, src = make_inputs(None)
    r = RefSolver(links, src)
    try:
        dt, iters, rsq = r.solve()
    finally:
        r.close()
    return {"value": dt, "unit": "s", "cores": cpu_threads(), "kind": "reference",
            "sample": f"one full FP64 CG solve of the reference solver (its host code + the restated per-site "
                      f"kernel, OpenMP) on the full 24^3x48 lattice to |r|^2/|b|^2 = {rsq:.2e}: {iters} iterations "
                      f"in {dt:.1f} s, measured (not scaled)",
            "iterations": iters, "true_rsq_rel": rsq}


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path on
    the host cores.  Every timed step is one full FP64 CG solve of the
    benchmark input to |r|/|b| < 1e-10 by the reference's own solver
    (ks_d_congrad_fn.cpp:221-619); warm-up steps are bounded samples of
    --ref-iters iterations (they only warm the caches and the thread pool).
    Same metric, unit and config object as the GPU arm; the solver it runs
    (FP64 CG) is named in "solver"."""
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return
    import orc

    if not os.path.exists(orc.REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libqphix_ref.so was not built"}))
        return
    dims = tuple(int(v) for v in args.lattice.split("x")) if args.lattice else DIMS
    links = synthetic.asqtad_links(dims, seed=LINK_SEED)
    src = synthetic.gaussian_source(dims, seed=SRC_SEED, parity="even")
    r = RefSolver(links, src, dims)
    try:
        for _ in range(args.warmup):
            r.solve(max_iter=args.ref_iters, nrestart=1)
        runs = [r.solve() for _ in range(args.steps)]
    finally:
        r.close()
    v = float(np.mean([t for t, _, _ in runs]))
    iters = [i for _, i, _ in runs]
    sample = (f"every step one full FP64 CG solve of the reference solver (its host code + restated kernel, "
              f"OpenMP on {cpu_threads()} threads) on the full {'x'.join(map(str, dims))} lattice to |r|/|b| < 1e-10: "
              f"{iters[0]} iterations, measured (not scaled)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded random SU(3) links, Gaussian source)",
        "config": bench_config(world, dims),
        "solver": "FP64 CG with the reference's control flow (the reference has no mixed-precision solver)",
        "solve": {"s_each": [round(t, 3) for t, _, _ in runs], "iterations": iters,
                  "true_rsq_rel": max(q for _, _, q in runs)},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cpu_threads(), "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_reference_dslash(args, dims, links):
    """--mode dslash --impl reference: the reference's own Dslash
    (qphix_ks_dslash, ks_long_dslash.cpp:564-668, with the restated per-site
    kernel; OpenMP on all host cores), wall-clock timed over --reps calls
    after one warm-up call, GB/s by the same algorithmic bytes."""
    import orc

    V = int(np.prod(dims))
    ref = capi.QphixLib(orc.REF_LIB)
    out = {}
    with _StdoutToStderr():
        assert ref.init(dims) == 0
        for prec in ("F", "D"):
            L = ref.create_L(prec, links)
            vin = ref.create_V(prec, np.random.default_rng(1).standard_normal(V * 6))
            vout = ref.create_V(prec, np.zeros(V * 6))
            ref.dslash(prec, L, vout, vin, "even")
            t0 = time.perf_counter()
            for _ in range(args.reps):
                ref.dslash(prec, L, vout, vin, "even")
            dt = (time.perf_counter() - t0) / args.reps
            nbytes = (DSLASH_BYTES_F32 if prec == "F" else DSLASH_BYTES_F64) * (V // 2)
            out[prec] = {"us": dt * 1e6, "gbs": nbytes / dt / 1e9}
            ref.destroy_V(prec, vin)
            ref.destroy_V(prec, vout)
            ref.destroy_L(prec, L)
        ref.finalize()
    print(json.dumps({"mode": "dslash", "impl": "reference", "lattice": "x".join(map(str, dims)), "reps": args.reps,
                      "cores": os.cpu_count(), **out}))


def run_profile_dslash(args):
    """--mode dslash: one FP32 and one FP64 Dslash launch after a warm-up
    (small-lattice capture target for ncu); with --impl reference the
    reference's host Dslash on the same lattice instead."""
    dims = tuple(int(v) for v in (args.lattice or "16x16x16x32").split("x"))
    links = synthetic.asqtad_links(dims, seed=LINK_SEED)
    V = int(np.prod(dims))
    if args.impl == "reference":
        run_reference_dslash(args, dims, links)
        return
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
    print(json.dumps({"mode": "dslash", "lattice": "x".join(map(str, dims)), "reps": args.reps, **out}))


def run_profile_mixed(args):
    """--mode mixed: only the timed mixed-precision solves (ncu launch list);
    --lattice another lattice than the headline's (same link recipe, mass and
    tolerance), with its kernel timings and the autotuner's per-variant
    times."""
    import torch

    dims = tuple(int(v) for v in args.lattice.split("x")) if args.lattice else DIMS
    links, src = make_inputs("cuda" if torch.cuda.is_available() and args.lattice else None, dims)
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(dims) == 0, lib.last_error()
    lib.set_reliable_delta(RU_DELTA)
    lib.set_link_compression(args.compress)
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
    name = {"single": "single-r12" if args.compress else "single"}.get(args.inner, args.inner)
    lib_tuning = (lib.tuning(name), lib.tuning(name, "mdagm"))
    # K1 / K2 device time inside one more solve (not timed above)
    lib.set_kernel_timing(True)
    x = lib.create_V("D", np.zeros_like(src), "even")
    lib.invert("D", L, x, b, MASS, parity="even", max_iter=MAX_ITER, nrestart=NRESTART, resid=RESID)
    st = lib.last_stats()
    lib.set_kernel_timing(False)
    lib.destroy_V("D", x)
    lib.destroy_V("D", b)
    lib.destroy_L("D", L)
    lib.finalize()
    k1_us = st.dslash_ms / max(st.dslash_launches, 1) * 1e3
    k2_us = st.mdagm_ms / max(st.mdagm_launches, 1) * 1e3
    print(json.dumps({"mode": "mixed", "inner": args.inner, "lattice": "x".join(map(str, dims)), "solves": res_all,
                      "k1_us": k1_us, "k2_us": k2_us, "tuning_k1": lib_tuning[0], "tuning_k2": lib_tuning[1]}))


MS_DIMS = (32, 32, 32, 64)
MS_MASS = 0.0012
MS_SIGMAS = np.logspace(-5, 0, 12)  # RHMC-style shifts sigma_j
MS_WORKLOAD = ("asqtad CG and 12-shift multi-shift CG 32^3x64, HISQ-shaped links (smeared eps=0.2 fat, "
               "eps=0.3 Naik), m=0.0012, shifts log-spaced 1e-5..1, tol 1e-10")


def _true_rel_rsq(lib, L, x_raw, src, mass, V):
    """|b - (4m^2 - D_eo D_oe) x|^2 / |b|^2 on the even sites, with the FP64
    operator applied through QPHIX_D3_asqtad_dslash (independent of the
    solver's own residual)."""
    e = slice(0, V * 3)
    full = np.zeros(V * 6)
    full[e] = x_raw[e]
    hin = lib.create_V("D", full)
    tmp = lib.create_V("D", np.zeros(V * 6))
    out = lib.create_V("D", np.zeros(V * 6))
    lib.dslash("D", L, tmp, hin, "odd")
    lib.dslash("D", L, out, tmp, "even")
    dd = lib.extract_V("D", out)[e]
    for h in (hin, tmp, out):
        lib.destroy_V("D", h)
    r = src[e] - (4 * mass * mass * x_raw[e] - dd)
    return float(np.dot(r, r) / np.dot(src[e], src[e]))


def multishift_workload(dims=MS_DIMS, reps=2, which=None, compress=True, cpu_baseline=False, notes=True):
    """The 32^3x64 workload on one GPU, same input for every solve: the FP64
    CG (reference control flow), the mixed CG with FP32 and with 16-bit-link
    inner solves, the FP64 multi-shift CG with 12 shifts and the mixed
    multi-shift CG.  Every solution's FP64 true residual is recomputed
    through the FP64 Dslash, and its error against the FP64 solution
    reported.  `which`: subset of the solve names (None: all); the last of
    `reps` solves of each kind is reported.  Returns a dict."""
    import torch

    V = int(np.prod(dims))
    Vh = V // 2
    dev = "cuda" if torch.cuda.is_available() else None
    t0 = time.perf_counter()
    links = synthetic.asqtad_links(dims, seed=LINK_SEED, eps_fat=0.2, eps_long=0.3, fat_scale=0.9,
                                   smear=True, device=dev)
    src = synthetic.gaussian_source(dims, seed=SRC_SEED, parity="even")
    gen_s = time.perf_counter() - t0
    if dev:
        torch.cuda.empty_cache()
    masses = np.sqrt(MS_MASS ** 2 + MS_SIGMAS / 4)
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(dims) == 0, lib.last_error()
    lib.set_reliable_delta(0.2)
    lib.set_link_compression(compress)  # FP32 inner solves with 12-real Naik links
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    assert L and b, lib.last_error()
    zeros = np.zeros_like(src)
    out = {"mode": "multishift", "workload": MS_WORKLOAD, "lattice": "x".join(map(str, dims)),
           "mass": MS_MASS, "sigmas": [float(s) for s in MS_SIGMAS], "resid_sq": RESID,
           "reliable_delta": 0.2,
           "seeds": {"links": LINK_SEED, "source": SRC_SEED}, "field_generation_s": gen_s}

    def want(name):
        return which is None or name in which

    def cg(inner, n):
        lib.set_inner_precision(inner)
        for k in range(n):
            x = lib.create_V("D", zeros, "even")
            lib.timer_start()
            it, info, res = lib.invert("D", L, x, b, MS_MASS, parity="even", max_iter=MAX_ITER,
                                       nrestart=NRESTART, resid=RESID)
            ms = lib.timer_stop()
            st = lib.last_stats()
            assert info.status == 0, lib.last_error()
            sol = lib.extract_V("D", x, "even")
            lib.destroy_V("D", x)
        return ms, st, res, sol

    def multi(inner, n):
        lib.set_inner_precision(inner)
        for k in range(n):
            xs = [lib.create_V("D", zeros, "even") for _ in masses]
            lib.timer_start()
            it, info, res = lib.invert_multi("D", L, xs, b, masses, parity="even", max_iter=MAX_ITER,
                                             nrestart=NRESTART, resid=RESID)
            ms = lib.timer_stop()
            st = lib.last_stats()
            assert info.status == 0, lib.last_error()
            sols = [lib.extract_V("D", x, "even") for x in xs]
            for x in xs:
                lib.destroy_V("D", x)
        return ms, st, res, sols

    def rel(a, ref):
        e = slice(0, V * 3)
        return float(np.abs(a[e] - ref[e]).max() / np.abs(ref[e]).max())

    def note(name):
        if notes:
            print(json.dumps({name: out[name]}), file=sys.stderr, flush=True)

    note("field_generation_s")
    x64 = xs64 = None
    ms64 = ms64m = None
    if want("fp64_cg"):
        ms64, st64, res64, x64 = cg("double", reps)
        out["fp64_cg"] = {"s": ms64 / 1e3, "iterations": res64.final_iter,
                          "true_rsq_rel": _true_rel_rsq(lib, L, x64, src, MS_MASS, V)}
        note("fp64_cg")
    for inner in ("single", "half-links"):
        if not want(f"mixed_cg_{inner}"):
            continue
        ms, st, res, x = cg(inner, reps)
        d = {"s": ms / 1e3, "iterations": st.iterations, "reliable_updates": st.reliable_updates,
             "escalated": st.escalated, "links_compressed": st.links_compressed,
             "true_rsq_rel": _true_rel_rsq(lib, L, x, src, MS_MASS, V)}
        if x64 is not None:
            d["err_vs_fp64"] = rel(x, x64)
            d["speedup_vs_fp64_cg"] = ms64 / ms
        if inner == "single":
            # per-kernel CUDA-event durations from one more solve (not timed)
            lib.set_kernel_timing(True)
            _, sti, _, _ = cg(inner, 1)
            lib.set_kernel_timing(False)
            d["k1_us"] = sti.dslash_ms / max(sti.dslash_launches, 1) * 1e3
            d["k2_us"] = sti.mdagm_ms / max(sti.mdagm_launches, 1) * 1e3
            d["k1_launches"] = sti.dslash_launches
            k1_bytes = DSLASH_BYTES_R12 if sti.links_compressed == 1 else DSLASH_BYTES_F32
            peak, kind = peaks()
            d["k1_gbs"] = k1_bytes * Vh / (d["k1_us"] * 1e-6) / 1e9
            d["k1_frac"] = d["k1_gbs"] / peak
            d["k2_gbs"] = (k1_bytes + 24) * Vh / (d["k2_us"] * 1e-6) / 1e9
            d["k2_frac"] = d["k2_gbs"] / peak
            d["peak_source"] = kind
        out[f"mixed_cg_{inner}"] = d
        note(f"mixed_cg_{inner}")
    if want("fp64_multishift"):
        ms64m, st64m, res64m, xs64 = multi("double", reps)
        out["fp64_multishift"] = {"s": ms64m / 1e3, "iterations": st64m.iterations,
                                  "true_rsq_rel": [_true_rel_rsq(lib, L, x, src, m, V)
                                                   for x, m in zip(xs64, masses)]}
        note("fp64_multishift")
    for inner in ("single", "half-links"):
        if not want(f"mixed_multishift_{inner}"):
            continue
        ms, st, res, xs = multi(inner, reps)
        d = {"s": ms / 1e3, "iterations": st.iterations, "reliable_updates": st.reliable_updates,
             "links_compressed": st.links_compressed, "final_iter_per_shift": [r.final_iter for r in res],
             "true_rsq_rel": [_true_rel_rsq(lib, L, x, src, m, V) for x, m in zip(xs, masses)]}
        if xs64 is not None:
            d["err_vs_fp64"] = [rel(x, y) for x, y in zip(xs, xs64)]
            d["speedup_vs_fp64_multishift"] = ms64m / ms
        if ms64 is not None:
            d["speedup_vs_fp64_cg"] = ms64 / ms
        out[f"mixed_multishift_{inner}"] = d
        note(f"mixed_multishift_{inner}")
    lib.destroy_V("D", b)
    lib.destroy_L("D", L)
    out["autotuner"] = {k: lib.dslash_variant(k) for k in ("single", "single-r12", "double", "half-links")}
    lib.finalize()
    if cpu_baseline and "fp64_cg" in out:
        import orc

        if os.path.exists(orc.REF_LIB):
            # full FP64 solves of the reference solver on the host cores, measured
            r = RefSolver(links, src, dims)
            try:
                dt, iters, rsq = r.solve(mass=MS_MASS)
            finally:
                r.close()
            out["cpu_baseline_fp64_cg"] = {
                "s": dt, "iterations": iters, "true_rsq_rel": rsq, "cores": cpu_threads(), "kind": "reference",
                "sample": "one full FP64 CG solve of the reference solver on the full lattice, measured"}
            note("cpu_baseline_fp64_cg")
            if "fp64_multishift" in out:
                ref = capi.QphixLib(orc.REF_LIB)
                with _StdoutToStderr():
                    ref.init(dims)
                    RL = ref.create_L("D", links)
                    rb = ref.create_V("D", src, "even")
                    rxs = [ref.create_V("D", np.zeros_like(src), "even") for _ in masses]
                    t0 = time.perf_counter()
                    it, info, res = ref.invert_multi("D", RL, rxs, rb, masses, parity="even", max_iter=MAX_ITER,
                                                     nrestart=NRESTART, resid=RESID)
                    dt = time.perf_counter() - t0
                    for x in rxs:
                        ref.destroy_V("D", x)
                    ref.destroy_V("D", rb)
                    ref.destroy_L("D", RL)
                    ref.finalize()
                out["cpu_baseline_fp64_multishift"] = {
                    "s": dt, "iterations": it, "cores": cpu_threads(), "kind": "reference",
                    "sample": "one full FP64 multi-shift solve (12 shifts) of the reference solver on the full "
                              "lattice, measured"}
    return out


def run_multishift(args):
    """--mode multishift: multishift_workload on --lattice (default 32^3x64)
    with every solve and the measured CPU baselines; prints one JSON line."""
    dims = tuple(int(v) for v in args.lattice.split("x")) if args.lattice else MS_DIMS
    which = set(args.solves.split(",")) if args.solves else None
    reps = 1 + max(0, min(args.steps, 2) - 1)
    print(json.dumps(multishift_workload(dims, reps, which, not args.no_compress, not args.no_cpu_baseline)))


BATCH_BIG = (24, 24, 24, 48)
BATCH_NRHS = 16
BATCH_SMALL = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 32), (20, 20, 20, 40)]
BATCH_MASS = 0.02
BATCH_WORKLOAD = ("batched mixed CG: 16 Gaussian RHS on 24^3x48 + 8 lattices (8^4, 12^4, 16^3x32, 20^3x40, "
                  "two of each, one RHS each), m=0.02, tol 1e-10, one device run")


def batch_workload(lattice=None, steps=1, warmup=1, sequential=True, notes=True):
    """24 systems on 9 lattices in one QPHIX_B200_D3_batch_invert call (host
    buffers in and out), against the same systems solved one at a time
    through QPHIX_D3_asqtad_invert with the FP32 inner solve.  Every
    solution's FP64 true residual is checked through the FP64 Dslash.
    lattice: the 16 right-hand sides on that lattice alone (profiling
    target).  Returns a dict."""
    import torch

    dev = "cuda" if torch.cuda.is_available() else None
    t0 = time.perf_counter()
    big = tuple(int(v) for v in lattice.split("x")) if lattice else BATCH_BIG
    lats = [big] + ([] if lattice else [d for d in BATCH_SMALL for _ in range(2)])
    links = [synthetic.asqtad_links(d, seed=LINK_SEED + i, device=dev) for i, d in enumerate(lats)]
    systems = [(0, BATCH_MASS, synthetic.gaussian_source(big, seed=SRC_SEED + r, parity="even"))
               for r in range(BATCH_NRHS)]
    systems += [(l, BATCH_MASS, synthetic.gaussian_source(lats[l], seed=SRC_SEED + 100 + l, parity="even"))
                for l in range(1, len(lats))]
    gen_s = time.perf_counter() - t0
    if notes:
        print(json.dumps({"field_generation_s": gen_s}), file=sys.stderr, flush=True)
    if dev:
        torch.cuda.empty_cache()
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(big) == 0, lib.last_error()
    B = lib.batch_create_L(list(zip(lats, links)))
    assert B, lib.last_error()
    outs = [torch.zeros(s[2].shape, dtype=torch.float64).pin_memory().numpy() for s in systems]
    pinned_src = [torch.from_numpy(s[2]).pin_memory().numpy() for s in systems]
    psys = [(l, m, p) for (l, m, _), p in zip(systems, pinned_src)]

    batch_g = [0]

    def batch_solve():
        for o in outs:
            o[:] = 0.0
        lib.timer_start()
        w0 = time.perf_counter()
        it, info, res, xs = lib.batch_invert(B, psys, max_iter=MAX_ITER, nrestart=NRESTART, resid=RESID,
                                             outs=outs)
        wall = time.perf_counter() - w0
        ms = lib.timer_stop()
        batch_g[0] = lib.last_stats().batch_rhs_per_thread
        assert info.status == 0, lib.last_error()
        return max(ms / 1e3, wall), res, [x.copy() for x in xs]

    for _ in range(max(1, warmup)):
        batch_solve()
    times = []
    for _ in range(max(1, steps)):
        s, res, xs = batch_solve()
        times.append(s)
    s_batch = float(np.median(times))
    if notes:
        print(json.dumps({"batch_s": s_batch, "iterations": [r.final_iter for r in res]}), file=sys.stderr,
              flush=True)
    lib.batch_destroy_L(B)
    if not sequential:
        lib.finalize()
        return {"mode": "batch", "workload": BATCH_WORKLOAD, "batch_s": s_batch,
                "rhs_per_thread": batch_g[0], "batch_iterations": [r.final_iter for r in res]}

    # the same systems one at a time (FP32 inner, FP64 reliable updates)
    seq = 0.0
    seq_iters = []
    trues = []
    lib.finalize()
    for l, dims in enumerate(lats):
        mine = [k for k, s in enumerate(systems) if s[0] == l]
        assert lib.init(dims) == 0, lib.last_error()
        L = lib.create_L("D", links[l])
        lib.set_inner_precision("single")
        V = int(np.prod(dims))
        for rep in range(2):  # the first pass warms the autotuner and the graphs
            for k in mine:
                b = lib.create_V("D", systems[k][2], "even")
                x = lib.create_V("D", np.zeros_like(systems[k][2]), "even")
                lib.timer_start()
                it, info, r1 = lib.invert("D", L, x, b, BATCH_MASS, parity="even", max_iter=MAX_ITER,
                                          nrestart=NRESTART, resid=RESID)
                ms = lib.timer_stop()
                if rep == 1:
                    seq += ms / 1e3
                    seq_iters.append(lib.last_stats().iterations)
                lib.destroy_V("D", b)
                lib.destroy_V("D", x)
        for k in mine:
            trues.append(_true_rel_rsq(lib, L, xs[k], systems[k][2], BATCH_MASS, V))
        lib.destroy_L("D", L)
        lib.finalize()
    return {
        "mode": "batch", "workload": BATCH_WORKLOAD, "systems": len(systems), "lattices": len(lats),
        "field_generation_s": gen_s, "batch_s": s_batch, "batch_all_s": times,
        "rhs_per_thread": batch_g[0],
        "sequential_s": seq, "speedup_vs_sequential": seq / s_batch,
        "batch_iterations": [r.final_iter for r in res], "batch_reliable_updates": [r.final_restart for r in res],
        "sequential_iterations": seq_iters,
        "true_rsq_rel_max": max(trues), "true_rsq_rel": trues,
        "timing": "batch: one C-ABI call from pinned host buffers (H2D of sources and guesses, D2H of "
                  "solutions inside); sequential: device time of each QPHIX_D3_asqtad_invert on resident vectors",
    }


def run_batch(args):
    """--mode batch: batch_workload on its 9 lattices (or --lattice alone);
    prints one JSON line."""
    print(json.dumps(batch_workload(args.lattice, args.steps, args.warmup, not args.no_sequential)))


FORCE_DIMS = (16, 16, 16, 32)
FORCE_MASS = 0.05
FORCE_WORKLOAD = ("fermion force d/dU of phi^dag (4m^2 - D_eo D_oe)^-1 phi, 16^3x32, m=0.05, eps=0.3 links; "
                  "central finite differences h=1e-5 along 32 random su(3) directions dU = i T U")


def run_force(args):
    """--mode force: the fermion force on 16^3x32 through the C ABI.  Checks
    the FP64 force against central finite differences of S along 32 random
    su(3) perturbations of all fat and Naik links (every S from an FP64 solve),
    the FP32 force against the FP64 one, and times both."""
    dims = FORCE_DIMS
    V = int(np.prod(dims))
    lat = synthetic.Lattice(dims)
    links = synthetic.asqtad_links(dims, seed=LINK_SEED)
    phi = synthetic.gaussian_source(dims, seed=SRC_SEED, parity="even")
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(dims) == 0, lib.last_error()
    lib.set_inner_precision("double")

    def action(fat, lng, want_force=False):
        lk = {"fat": fat, "lng": lng, "fatback": synthetic.backlinks_raw(dims, fat, 1),
              "lngback": synthetic.backlinks_raw(dims, lng, 3)}
        L = lib.create_L("D", lk)
        b = lib.create_V("D", phi, "even")
        x = lib.create_V("D", np.zeros_like(phi), "even")
        it, info, res = lib.invert("D", L, x, b, FORCE_MASS, parity="even", max_iter=MAX_ITER,
                                   nrestart=NRESTART, resid=1e-26)
        assert info.status == 0, lib.last_error()
        xr = lib.extract_V("D", x, "even")
        S = float(np.dot(phi[: 3 * V], xr[: 3 * V]))
        out = (S,)
        if want_force:
            lib.force("D", L, [x], [1.0], "even")  # warm
            lib.timer_start()
            gf, gl = lib.force("D", L, [x], [1.0], "even")
            ms64 = lib.timer_stop()
            k64 = lib.last_stats().solve_ms
            Lf = lib.create_L("F", lk)
            xf = lib.create_V("F", xr, "even")
            lib.force("F", Lf, [xf], [1.0], "even")
            lib.timer_start()
            ff, fl = lib.force("F", Lf, [xf], [1.0], "even")
            ms32 = lib.timer_stop()
            k32 = lib.last_stats().solve_ms
            lib.destroy_V("F", xf)
            lib.destroy_L("F", Lf)
            out = (S, gf, gl, ff, fl, ms64, ms32, it, k64, k32)
        for h in (b, x):
            lib.destroy_V("D", h)
        lib.destroy_L("D", L)
        return out

    S0, gf, gl, ff, fl, ms64, ms32, iters, k64, k32 = action(links["fat"], links["lng"], True)
    gnorm = float(np.sqrt(gf @ gf + gl @ gl))
    rng = np.random.default_rng(3003)
    h = 1e-5
    errs, nerrs = [], []
    t0 = time.perf_counter()
    for _ in range(args.fd_dirs):
        dirs = []
        for key in ("fat", "lng"):
            U = synthetic.links_raw_to_lex(dims, links[key])
            a = rng.standard_normal(U.shape) + 1j * rng.standard_normal(U.shape)
            T = 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))
            T = T - (np.trace(T, axis1=-2, axis2=-1) / 3.0)[..., None, None] * np.eye(3)
            dirs.append(synthetic._to_raw_links(lat, 1j * T @ U))
        Sp = action(links["fat"] + h * dirs[0], links["lng"] + h * dirs[1])[0]
        Sm = action(links["fat"] - h * dirs[0], links["lng"] - h * dirs[1])[0]
        fd = (Sp - Sm) / (2 * h)
        an = float(gf @ dirs[0] + gl @ dirs[1])
        errs.append(abs(fd - an) / abs(an))
        nerrs.append(abs(fd - an) / (gnorm * float(np.sqrt(dirs[0] @ dirs[0] + dirs[1] @ dirs[1]))))
    fd_s = time.perf_counter() - t0
    scale = max(np.abs(gf).max(), np.abs(gl).max())
    lib.finalize()
    bytes64 = 2 * V * 72 * 8
    print(json.dumps({
        "mode": "force", "workload": FORCE_WORKLOAD, "lattice": "x".join(map(str, dims)), "mass": FORCE_MASS,
        "action": S0, "solve_iterations": iters, "fd_perturbations": len(errs), "fd_h": h,
        "fd_rel_err_max": max(errs) if errs else None,
        "fd_rel_err_median": float(np.median(errs)) if errs else None, "fd_wall_s": fd_s,
        "fp32_vs_fp64_max_rel": float(max(np.abs(ff - gf).max(), np.abs(fl - gl).max()) / scale),
        "fd_err_over_grad_times_dir_norm_max": max(nerrs) if nerrs else None,
        "force_call_ms": {"f64": ms64, "f32": ms32},
        "force_kernels_ms": {"f64": k64, "f32": k32},
        "force_kernels_gbs_f64": (bytes64 + DSLASH_BYTES_F64 * V // 2 + 2 * V * 48) / (k64 * 1e-3) / 1e9,
        "force_call_note": "one C-ABI call: D x, the outer-product kernel and the D2H copy of both "
                           f"gradient arrays ({bytes64 / 1e6:.0f} MB FP64)",
    }))


GF_WORKLOAD = ("Symanzik one-loop gauge force (6 plaquette, 18 rectangle, 24 parallelogram staples per link), "
               "momentum update of one checkerboard, random SU(3) links")


def run_gforce(args):
    """--mode gforce: QPHIX_{D3,F3}_symanzik_1loop_gauge_force on --lattice
    (default 32^3x64), one checkerboard per call, device time per call
    (CUDA events around the kernel, mean of --reps calls after one warm-up)
    and GFLOP/s by the call's own flop count (info.final_flop)."""
    import torch  # noqa: F401  (CUDA context through the library)

    dims = tuple(int(v) for v in args.lattice.split("x")) if args.lattice else MS_DIMS
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    lat = synthetic.Lattice(dims)
    rng = np.random.default_rng(LINK_SEED)
    # random SU(3) per link from QR of complex Gaussians (det fixed to 1)
    V = lat.V
    a = rng.standard_normal((V * 4, 3, 3)) + 1j * rng.standard_normal((V * 4, 3, 3))
    q, r = np.linalg.qr(a)
    q = q * (np.diagonal(r, axis1=1, axis2=2) / np.abs(np.diagonal(r, axis1=1, axis2=2)))[:, None, :]
    q = q / np.linalg.det(q)[:, None, None] ** (1.0 / 3.0)
    raw = np.empty((V * 4, 3, 3, 2))
    raw[..., 0], raw[..., 1] = q.real, q.imag
    Uraw = raw.reshape(-1)
    mom = np.zeros(V * 72)
    coeffs = {"plaquette": 1.0, "rectangle": -0.0545, "parallelogram": -0.0123}
    lib = capi.QphixLib(LIB_PATH)
    assert lib.init(dims) == 0, lib.last_error()
    out = {"mode": "gforce", "workload": GF_WORKLOAD, "lattice": "x".join(map(str, dims)), "coeffs": coeffs}
    for prec in ("D", "F"):
        g = lib.create_G(prec, Uraw, "even")
        f = lib.create_F(prec, mom, "even")
        info = lib.gauge_force(prec, g, f, coeffs, 0.01)  # warm-up (table upload, module load)
        assert info.status == 0, lib.last_error()
        ms = []
        for _ in range(max(1, args.reps)):
            info = lib.gauge_force(prec, g, f, coeffs, 0.01)
            ms.append(lib.last_stats().solve_ms)
        t = float(np.mean(ms))
        out[prec] = {"ms_per_call": t, "gflops": info.final_flop / (t * 1e-3) / 1e9,
                     "flop_per_call": info.final_flop, "links_per_call": 4 * V // 2}
        lib.destroy_G(prec, g)
        lib.destroy_F(prec, f)
    lib.finalize()
    print(json.dumps(out))


DD_WORKLOAD = ("domain-decomposed asqtad CG: the lattice cut into t slabs, one per GPU, faces over NCCL "
               "send/recv into each GPU's ghost buffer, FP64 sums by ncclAllReduce")


def run_dd(args):
    """--mode dd: the domain-decomposed path.  Under torchrun with N > 1 the
    --lattice (default 32^3x64) is cut into N t slabs, one per GPU; every
    rank solves its slab of the same system (FP64 CG, then mixed CG with
    12-real Naik links); device time per solve, max over ranks (strong
    scaling).  On one GPU: the headline mixed solve through the periodic
    path and through the loopback halo path, to measure the halo's cost."""
    import torch

    world, rank, local, pg = dist_setup()
    os.environ["QPHIX_GPU_DEVICE"] = str(local)
    torch.cuda.set_device(local)
    dims = tuple(int(v) for v in args.lattice.split("x")) if args.lattice else (MS_DIMS if world > 1 else DIMS)
    mass = MS_MASS if dims == MS_DIMS else MASS
    links = synthetic.asqtad_links(dims, seed=LINK_SEED, smear=dims == MS_DIMS,
                                   eps_fat=0.2 if dims == MS_DIMS else 0.3,
                                   device="cuda" if max(dims) > 16 else None)
    src = synthetic.gaussian_source(dims, seed=SRC_SEED, parity="even")
    lib = capi.QphixLib(LIB_PATH)
    if world > 1:
        from milc_qphix_b200 import decomp

        uid = [lib.comm_unique_id() if rank == 0 else None]
        pg.broadcast_object_list(uid, src=0)
        assert lib.comm_init(uid[0], world, rank) == 0, lib.last_error()
        assert lib.init(dims, (1, 1, 1, world), rank) == 0, lib.last_error()
        links = {k: decomp.scatter(dims, v, world, rank, 72) for k, v in links.items()}
        src = decomp.scatter(dims, src, world, rank, 6)
    else:
        assert lib.init(dims) == 0, lib.last_error()
    lib.set_reliable_delta(0.2 if dims == MS_DIMS else RU_DELTA)
    lib.set_link_compression(True)
    L = lib.create_L("D", links)
    b = lib.create_V("D", src, "even")
    zeros = np.zeros_like(src)

    def solve(inner, n):
        lib.set_inner_precision(inner)
        out = []
        for _ in range(n):
            x = lib.create_V("D", zeros, "even")
            barrier(pg)
            lib.timer_start()
            it, info, res = lib.invert("D", L, x, b, mass, parity="even", max_iter=MAX_ITER, nrestart=NRESTART,
                                       resid=RESID)
            ms = lib.timer_stop()
            assert info.status == 0, lib.last_error()
            st = lib.last_stats()
            out.append((max_over_ranks(pg, ms), st.iterations, res.final_rsq))
            lib.destroy_V("D", x)
        return out

    result = {"mode": "dd", "workload": DD_WORKLOAD, "lattice": "x".join(map(str, dims)), "mass": mass,
              "n_gpus": world, "scaling": "strong", "resid_sq": RESID}
    paths = [("decomposed", False)] if world > 1 else [("periodic", False), ("loopback_halo", True)]
    for name, loop in paths:
        if world == 1:
            lib.set_loopback_halo(loop)
        r64 = solve("double", 2)[-1]
        rmx = solve("single", 1 + max(1, args.steps))[1:]
        result[name] = {"fp64_cg": {"s": r64[0] / 1e3, "iterations": r64[1], "true_rsq_rel": r64[2]},
                        "mixed_cg": {"s": float(np.mean([t for t, _, _ in rmx])) / 1e3, "iterations": rmx[0][1],
                                     "true_rsq_rel": max(q for _, _, q in rmx)}}
    if world == 1:
        lib.set_loopback_halo(False)
        result["halo_cost_mixed"] = result["loopback_halo"]["mixed_cg"]["s"] / result["periodic"]["mixed_cg"]["s"]
    lib.destroy_V("D", b)
    lib.destroy_L("D", L)
    lib.finalize()
    if world > 1:
        lib.comm_finalize()
    if rank == 0:
        print(json.dumps(result))
    if pg is not None:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="bench",
                    choices=["bench", "dslash", "mixed", "multishift", "batch", "force", "dd", "gforce"],
                    help="bench: the benchmark line; dslash/mixed: small profiling targets; "
                         "multishift: the 32^3x64 CG and 12-shift multi-shift workload; "
                         "batch: 24 systems on 9 lattices in one batched solve; "
                         "force: the 16^3x32 fermion force against finite differences")
    ap.add_argument("--lattice", default=None)
    ap.add_argument("--solves", default=None,
                    help="multishift mode: comma-separated subset of fp64_cg, mixed_cg_single, "
                         "mixed_cg_half-links, fp64_multishift, mixed_multishift_single, "
                         "mixed_multishift_half-links")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--inner", default="single", choices=["single", "half", "half-links", "double"])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-iters", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="default run: skip the batched-solve workload (config 4) extra key")
    ap.add_argument("--no-target", action="store_true",
                    help="bench mode: skip the 32^3x64 solves reported beside the headline")
    ap.add_argument("--no-compress", action="store_true",
                    help="multishift mode: 18-real links in the FP32 inner solves")
    ap.add_argument("--compress", action="store_true",
                    help="mixed mode: FP32 inner solve with 12-real Naik links")
    ap.add_argument("--fd-dirs", type=int, default=32,
                    help="force mode: finite-difference directions (0: force only)")
    ap.add_argument("--no-sequential", action="store_true",
                    help="batch mode: skip the one-at-a-time comparison (profiling target)")
    args = ap.parse_args()
    if args.mode == "dslash":
        run_profile_dslash(args)
        return
    if args.mode == "mixed":
        run_profile_mixed(args)
        return
    if args.mode == "multishift":
        run_multishift(args)
        return
    if args.mode == "batch":
        run_batch(args)
        return
    if args.mode == "force":
        run_force(args)
        return
    if args.mode == "dd":
        run_dd(args)
        return
    if args.mode == "gforce":
        run_gforce(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
