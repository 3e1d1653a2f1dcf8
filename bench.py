#!/usr/bin/env python
"""bench.py -- throughput of the plenoptic depth hot path on B200.

One step = one 4080x3068 8-bit raw frame (pitch 23.2 px, three lens types with
blur sigma 0.6/1.0/1.4, 12 slanted planes, ~26.6 k micro-images) through the
whole path: micro-image slicing, random initialisation and 8 red-black
PatchMatch iterations with 12 neighbours and a 15x15 bilateral NCC (FP32),
the cycle check, the disparity filter and its reprojection-error map, and a
64-slice focal stack rendered to 2040x1534.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line (rank 0).  Under torchrun each rank processes its own
frame (frames are independent: weak scaling, replicas only); ranks meet only
for the barrier and the max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "plenoptic-for-depth_b200")

WORKLOAD = dict(width=4080, height=3068, pitch=23.2, n_planes=12, max_nb=12, patch_size=15, iterations=8,
                sigma_spatial=3.0, sigma_color=12.0, n_lens_types=3, blur_sigma=(0.6, 1.0, 1.4), seed=2026,
                slices=64, vd_range=(2.0, 12.0))


def metric() -> str:
    return "%dx%d depth frames/s" % (WORKLOAD["width"], WORKLOAD["height"])
FLOPS_PER_TAP = 24      # per in-bounds NCC tap: disparity 4, source coords 4, fractions 2, bilinear 6, moments 8


def load_pfd():
    name = "pfd_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def fp32_fma_rate(device: int) -> float:
    """FP32 FFMA throughput of the device (TFLOP/s), from the probe built into
    tests/_build (independent FFMA chains on every SM, best of three)."""
    import ctypes
    path = os.path.join(ROOT, "tests", "_build", "libfmaprobe.so")
    L = ctypes.CDLL(path)
    L.pfd_probe_fp32_fma_rate.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    v = ctypes.c_double()
    rc = L.pfd_probe_fp32_fma_rate(device, ctypes.byref(v))
    if rc != 0:
        raise RuntimeError("FP32 probe failed: CUDA error %d" % rc)
    return v.value


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pfd_oracle
    pfd_oracle.build()
    return pfd_oracle


def make_workload(pfd, rank: int):
    w = WORKLOAD
    return pfd.make_workload(w["width"], w["height"], w["pitch"], w["n_planes"], seed=w["seed"] + rank,
                             max_nb=w["max_nb"], n_lens_types=w["n_lens_types"], blur_sigma=w["blur_sigma"])


def stack_size():
    return WORKLOAD["width"] // 2, WORKLOAD["height"] // 2


def slice_vds():
    lo, hi = WORKLOAD["vd_range"]
    return np.linspace(lo, hi, WORKLOAD["slices"]).astype(np.float32)


def pm_params(pfd):
    w = WORKLOAD
    return pfd.PmParams(base=w["pitch"], patch_size=w["patch_size"], max_iterations=w["iterations"],
                        sigma_spatial=w["sigma_spatial"], sigma_color=w["sigma_color"])


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU baseline: the oracle restatement of the path on the host cores
# --------------------------------------------------------------------------
class CpuSample:
    """The oracle restatement of the whole path on the host cores, timed on a
    bounded sample of one frame and scaled to the frame:
      * SelectNeighbors + MISimilarityMeasure on every micro-image (threads
        over views, as the reference's OpenMP loop, SelectNeighbors.cpp:123);
      * PatchMatch: RandomInitializationForFrame on `blocks` blocks of views
        spread evenly over the frame, scaled by views; one late half-sweep
        (the last one, started from the converged state before it) on the same
        blocks, with its in-bounds NCC taps counted; every half-sweep of the
        run is then its own tap count (counted on the device in the
        calibration pass, equal to the oracle's count) times the sample's time
        per tap; the spread of the blocks' times per tap is reported;
      * the cycle check, the disparity filter and its reprojection map on the
        frame's converged state (one thread, like the reference's CPU code);
      * the focal stack: 4 of the slices, scaled to all of them (threads).
    The states come from the device run of the same frame, lists and seed,
    which is bit-identical to the oracle's (tests/test_gpu_config_parity.py)."""

    def __init__(self, pfd, oracle, w, params, seed, nthreads, sweep_taps, before_last, converged, blocks=8):
        self.pfd, self.oracle, self.w = pfd, oracle, w
        self.orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
        self.params, self.seed, self.nthreads = params, seed, nthreads
        self.sweep_taps = list(sweep_taps)
        self.before_last, self.converged = before_last, converged
        self.V = w.centers.shape[0]
        self.blocks = blocks
        self.bs = 16
        vds = slice_vds()
        self.sample_vds = vds[[len(vds) // 8, (3 * len(vds)) // 8, (5 * len(vds)) // 8, (7 * len(vds)) // 8]]

    def _ranges(self, bs):
        step = self.V // self.blocks
        return [(i * step + (step - bs) // 2, i * step + (step - bs) // 2 + bs) for i in range(self.blocks)]

    def _pm(self, bs):
        P, orc = self.params, self.orc
        it_last = P.max_iterations - 1
        t_init = t_sweep = 0.0
        taps = 0
        per_tap = []
        for v in self._ranges(bs):
            t0 = time.perf_counter()
            orc.init(P, self.seed, nthreads=self.nthreads, views=v)
            t1 = time.perf_counter()
            orc.sweep(P, self.seed, it_last, 1, self.before_last, nthreads=self.nthreads, views=v)
            t2 = time.perf_counter()
            _, tp = orc.sweep_taps(P, self.seed, it_last, 1, self.before_last, nthreads=self.nthreads, views=v)
            t_init += t1 - t0
            t_sweep += t2 - t1
            taps += tp
            per_tap.append((t2 - t1) / max(tp, 1))
        return t_init, t_sweep, taps, per_tap

    def calibrate(self, budget_s):
        bs = 16
        while True:
            ti, ts, _, _ = self._pm(bs)
            if ti + ts >= 0.5 * budget_s or bs * self.blocks * 2 > self.V:
                break
            bs = min(self.V // self.blocks, max(2 * bs, int(bs * 0.7 * budget_s / max(ti + ts, 1e-3))))
        self.bs = bs

    def run(self) -> dict:
        o, pfd, w = self.oracle, self.pfd, self.w
        t0 = time.perf_counter()
        o.select_neighbors(w.centers, w.tilekeys, w.frame.n_cols, w.frame.n_rows, w.frame.pitch, images=w.gray)
        t_sel = time.perf_counter() - t0
        ti, ts, taps, per_tap = self._pm(self.bs)
        nv = self.bs * self.blocks
        t_init = ti * self.V / nv
        s_per_tap = ts / max(taps, 1)
        t_sweeps = s_per_tap * sum(self.sweep_taps)
        st = {k: v.copy() for k, v in self.converged.items()}
        unit = WORKLOAD["pitch"]
        t0 = time.perf_counter()
        o.cycle_check(self.orc, pfd.CycleCfg(), unit, st)
        o.filter_global(self.orc, pfd.FilterCfg(), unit, st)
        o.reprojection_error(self.orc, pfd.FilterCfg(), unit, st)
        t1 = time.perf_counter()
        ow, oh = stack_size()
        o.refocus(self.orc, WORKLOAD["width"], WORKLOAD["height"], self.sample_vds, ow, oh)
        t2 = time.perf_counter()
        t_stack = (t2 - t1) * WORKLOAD["slices"] / len(self.sample_vds)
        rel = float(np.std(per_tap) / np.mean(per_tap)) if len(per_tap) > 1 else 0.0
        return {"frame_s": t_sel + t_init + t_sweeps + (t1 - t0) + t_stack, "t_select": t_sel, "views": nv,
                "t_init_sample": ti, "t_sweep_sample": ts, "sample_taps": taps, "t_init": t_init, "t_sweeps": t_sweeps,
                "pm_s": t_init + t_sweeps, "t_checks": t1 - t0, "t_stack": t_stack, "per_tap_spread": rel}

    def describe(self, s) -> str:
        return ("oracle SelectNeighbors on every view (%.2f s, %d threads); PatchMatch init on %d of %d micro-images in "
                "%d blocks spread over the frame (%.2f s, scaled by views) and the last half-sweep on them from the "
                "converged state (%.2f s, %.3g taps), the run's %d half-sweeps scaled by their device-counted taps "
                "(%.3g; blocks' time per tap spread %.1f%%): %.0f s; cycle check + filter + reprojection map of the "
                "converged frame (%.1f s, 1 thread); focal stack: 4 of %d slices (%.1f s scaled, %d threads)" %
                (s["t_select"], self.nthreads, s["views"], self.V, self.blocks, s["t_init_sample"], s["t_sweep_sample"],
                 s["sample_taps"], len(self.sweep_taps), sum(self.sweep_taps), 100 * s["per_tap_spread"], s["pm_s"],
                 s["t_checks"], WORKLOAD["slices"], s["t_stack"], self.nthreads))


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------------------
# engine arm
# --------------------------------------------------------------------------
STAGES = ("slice + neighbour selection", "init", "patchmatch sweeps", "cycle check", "filter", "reprojection map",
          "focal stack")


def job_time(local: float, world: int, device: str) -> float:
    """Time of the whole job over replicas: the slowest rank's (one all_reduce
    MAX over the process group; the local time when there is one rank)."""
    if world <= 1:
        return float(local)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(frames_per_rank: int, world: int, job_s: float) -> float:
    """Whole-job frames/s: every rank matched frames_per_rank frames of its own
    (replicas, no data exchanged) within the job time."""
    return world * frames_per_rank / job_s


def run_engine(args, rank, world, local_rank):
    import ctypes
    import torch
    import torch.distributed as dist

    pfd = load_pfd()
    torch.cuda.set_device(local_rank)
    w = make_workload(pfd, rank)
    params = pm_params(pfd)
    V = w.centers.shape[0]
    unit = WORKLOAD["pitch"]
    ow, oh = stack_size()
    vds = slice_vds()
    ccfg, fcfg = pfd.CycleCfg(), pfd.FilterCfg()
    ctx = pfd.Context(local_rank)
    ctx.set_sweep_fetch(pfd.FETCH_TEXTURE if args.fetch == "texture" else pfd.FETCH_SHARED)
    fid = ctx.frame_create(w.frame.raw.shape[1], w.frame.raw.shape[0], w.centers, w.tilekeys, w.mi, w.mi,
                           w.nb_ids, w.nb_counts)
    raw_dev = torch.from_numpy(w.frame.raw).to(f"cuda:{local_rank}")
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local_rank}")
    seed = WORKLOAD["seed"]

    def mark(ev, key):
        if ev is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record(stream)
            ev.setdefault(key, []).append(e)

    n_cols, n_rows = w.frame.n_cols, w.frame.n_rows

    def step(ev=None):
        """The whole path on one frame already resident in HBM."""
        mark(ev, "t0")
        ctx.frame_set_raw_device(fid, raw_dev.data_ptr(), raw_dev.shape[1])
        ctx.frame_select_neighbors(fid, n_cols, n_rows, WORKLOAD["pitch"])
        mark(ev, "ti")
        ctx.pm_init(fid, params, seed)
        mark(ev, "t1")
        for it in range(params.max_iterations):
            for ph in range(2):
                mark(ev, "sweep_a")
                ctx.pm_sweep(fid, params, seed, it, ph)
                mark(ev, "sweep_b")
        mark(ev, "t2")
        ctx.cycle_check(fid, ccfg, unit, maps=False, stats=False)
        mark(ev, "t3")
        ctx.filter(fid, fcfg, unit, download=False)
        mark(ev, "t4")
        ctx.reprojection_error(fid, fcfg, unit, download=False)
        mark(ev, "t5")
        ctx.refocus(fid, vds, ow, oh, download=False)
        mark(ev, "t6")
        ctx.cycle_check_stats(fid)            # the statistics, folded once the path is enqueued

    # calibration pass: in-bounds NCC taps per sweep launch (identical trajectory: same
    # seed and lists); the state before the last half-sweep and the converged state
    # are kept for the CPU baseline
    ctx.frame_set_raw_device(fid, raw_dev.data_ptr(), raw_dev.shape[1])
    sel_ids, sel_cnt = ctx.frame_select_neighbors(fid, n_cols, n_rows, WORKLOAD["pitch"], max_list=WORKLOAD["max_nb"])
    ctx.set_tap_counting(True)
    ctx.pm_init(fid, params, seed)
    ctx.read_tap_count()
    sweep_taps = []
    before_last = None
    for it in range(params.max_iterations):
        for ph in range(2):
            if it == params.max_iterations - 1 and ph == 1 and world == 1 and rank == 0:
                before_last = dict(zip(("plane", "cost", "disp", "sel"), ctx.download(fid)))
            ctx.pm_sweep(fid, params, seed, it, ph)
            sweep_taps.append(ctx.read_tap_count())
    ctx.set_tap_counting(False)
    converged = dict(zip(("plane", "cost", "disp", "sel"), ctx.download(fid)))
    depth = pfd.depth_error(w, converged["plane"], cost=converged["cost"])

    for _ in range(args.warmup):
        step()
    ctx.sync()
    fp32_tflops = fp32_fma_rate(local_rank)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev = {}
    launches0 = ctx.launch_count()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for _ in range(args.steps):
        step(ev)
    t_end.record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    clk = clocks.stop()
    ms = t_start.elapsed_time(t_end)
    sweep_ms = [a.elapsed_time(b) for a, b in zip(ev["sweep_a"], ev["sweep_b"])]
    stage_ms = {}
    for name, (a, b) in zip(STAGES, [("t0", "ti"), ("ti", "t1"), ("t1", "t2"), ("t2", "t3"), ("t3", "t4"),
                                     ("t4", "t5"), ("t5", "t6")]):
        stage_ms[name] = round(statistics.mean(x.elapsed_time(y) for x, y in zip(ev[a], ev[b])), 3)
    ms = job_time(ms, world, f"cuda:{local_rank}")
    if world > 1:
        dist.barrier()

    # the same step with the PatchMatch and the filter replayed from CUDA graphs
    graphs = None
    if world == 1:
        def step_graph():
            ctx.frame_set_raw_device(fid, raw_dev.data_ptr(), raw_dev.shape[1])
            ctx.frame_select_neighbors(fid, n_cols, n_rows, WORKLOAD["pitch"])
            ctx.patchmatch(fid, params, seed)
            ctx.cycle_check(fid, ccfg, unit, maps=False, stats=False)
            ctx.filter(fid, fcfg, unit, download=False)
            ctx.reprojection_error(fid, fcfg, unit, download=False)
            ctx.refocus(fid, vds, ow, oh, download=False)
            ctx.cycle_check_stats(fid)
        ctx.set_graphs(True)
        for _ in range(2):                       # uncaptured, then captured
            step_graph()
        ctx.sync()
        ga = torch.cuda.Event(enable_timing=True)
        gb = torch.cuda.Event(enable_timing=True)
        ga.record(stream)
        for _ in range(3):
            step_graph()
        gb.record(stream)
        ctx.sync()
        ctx.set_graphs(False)
        graphs = {"ms_per_step": round(ga.elapsed_time(gb) / 3, 2),
                  "covers": "the same step with pfd_patchmatch and the filter replayed from CUDA graphs"}

    # e2e through the public API with host buffers: pinned raw frame in; the
    # filtered per-pixel state (plane, cost, selected views) and the focal
    # stack out, every step
    pinned_raw = torch.from_numpy(w.frame.raw).pin_memory()
    px = V * w.mi * w.mi
    out_plane = torch.empty((px, 4), dtype=torch.float32).pin_memory()
    out_cost = torch.empty(px, dtype=torch.float32).pin_memory()
    out_sel = torch.empty(px, dtype=torch.int32).pin_memory()
    out_stack = torch.empty((len(vds), oh, ow), dtype=torch.float32).pin_memory()
    vd_host = np.ascontiguousarray(vds)
    L = pfd.lib()

    def e2e_step():
        ctx._check(L.pfd_frame_set_raw(ctx._h, fid, ctypes.c_void_p(pinned_raw.data_ptr()), pinned_raw.shape[1]),
                   "pfd_frame_set_raw")
        ctx.frame_select_neighbors(fid, n_cols, n_rows, WORKLOAD["pitch"])
        ctx.patchmatch(fid, params, seed)
        ctx.cycle_check(fid, ccfg, unit, maps=False, stats=False)
        ctx.filter(fid, fcfg, unit, download=False)
        ctx.reprojection_error(fid, fcfg, unit, download=False)
        ctx._check(L.pfd_refocus(ctx._h, fid, ctypes.c_void_p(vd_host.ctypes.data), len(vd_host), ow, oh,
                                 ctypes.c_void_p(out_stack.data_ptr())), "pfd_refocus")
        ctx._check(L.pfd_download(ctx._h, fid, ctypes.c_void_p(out_plane.data_ptr()), ctypes.c_void_p(out_cost.data_ptr()),
                                  None, ctypes.c_void_p(out_sel.data_ptr())), "pfd_download")
        ctx.cycle_check_stats(fid)

    e2e_step()
    e2e_steps = max(1, min(args.steps, 3))
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_s = job_time(e2e_s, world, f"cuda:{local_rank}")

    result = None
    if rank == 0:
        frames = world * args.steps
        value = replica_throughput(args.steps, world, ms / 1e3)
        # roofline of the dominant kernel (the red-black sweep)
        avg_sweep_ms = statistics.mean(sweep_ms)
        taps_per_launch = statistics.mean(sweep_taps)
        achieved = taps_per_launch * FLOPS_PER_TAP / (avg_sweep_ms * 1e-3) / 1e12
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "pm_sweep_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                tj = json.load(f)
            if tj.get("workload") == "4080x3068 pitch 23.2 K12 P15":
                traffic = tj.get("bytes_per_launch")
        result = {
            "metric": metric(), "value": round(value, 4), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded plenoptic raw frame)",
            "config": {"workload": workload_text(V, ow, oh),
                       "parallelism": "replicas" if world > 1 else "single",
                       "sweep_fetch": args.fetch,
                       "l2": "per-step working set %.2f GB > 126 MB L2 (state, tiles, focal stack)" %
                             (px * 40 * 2 / 1e9 + len(vds) * ow * oh * 4 / 1e9),
                       "stages": list(STAGES)},
            "stage_ms": stage_ms,
            "e2e": {"value": round(replica_throughput(e2e_steps, world, e2e_s), 4), "unit": "frames/s",
                    "h2d_bytes_per_step": int(w.frame.raw.nbytes),
                    "d2h_bytes_per_step": int(out_plane.numel() * 4 + out_cost.numel() * 4 + out_sel.numel() * 4 +
                                              out_stack.numel() * 4)},
            "roofline": {"bound": "fp32", "kernel": "pm_sweep_warp_kernel", "achieved": round(achieved, 3),
                         "peak": round(fp32_tflops, 2), "unit": "TFLOP/s", "frac": round(achieved / fp32_tflops, 4),
                         "peak_source": "measured FP32 FFMA rate on this device (tests/csrc/fma_probe.cu); "
                                        "MEASURED_PEAKS.json has no FP32 figure",
                         "algorithmic": "%d flops x %.3g in-bounds NCC taps per launch" %
                                        (FLOPS_PER_TAP, taps_per_launch),
                         "avg_launch_ms": round(avg_sweep_ms, 3), "traffic": traffic},
            "clocks": clk,
            "gpu_launches": launches,
        }
        if graphs is not None:
            result["graphs"] = graphs
        result["depth_error"] = dict({k: round(v, 4) for k, v in depth.items()},
                                     against="the scene's true virtual depth at each raw pixel (synthetic frame)")
        if world == 1 and not args.no_cpu_baseline:
            oracle = load_oracle()
            nth = cpu_threads()
            ws = pfd.Workload(w.frame, w.mi, w.centers, w.tilekeys, sel_ids, sel_cnt, w.gray)
            cs = CpuSample(pfd, oracle, ws, params, seed, nth, sweep_taps, before_last, converged)
            cs.calibrate(8.0)
            smp = cs.run()
            result["cpu_baseline"] = {"value": round(1.0 / smp["frame_s"], 8), "unit": "frames/s", "cores": nth,
                                      "kind": "port", "sample": cs.describe(smp)}
    if result is not None and world == 1:
        result["acmm"] = acmm_leg(pfd, ctx, fid, raw_dev, stream, seed)
    ctx.frame_free(fid)
    ctx.close()
    if result is not None:
        result["forms"] = ("batching (64 mixed frames) and serving (Poisson streams) are measured by "
                           "python bench.py --forms; profiles/forms_mixed_frames.md")
    return result


def acmm_leg(pfd, ctx, fid, raw_dev, stream, seed, reps=3):
    """The ACMM matcher (PFD_MATCHER_ACMM, one pyramid level) on the same
    resident frame with the parameters AdaptMIPMFrameACMM uses at one level
    (patch 5, 5 iterations, top_k 6, PatchMatchParamsLF's sigmas 5 and 3):
    initialisation, 10 half-sweeps and the post-refine pass, device-timed."""
    import torch
    P = pfd.PmParams(base=WORKLOAD["pitch"], patch_size=5, max_iterations=5, top_k=6, sigma_spatial=5.0,
                     sigma_color=3.0)
    ctx.set_matcher(True)
    try:
        ctx.frame_set_raw_device(fid, raw_dev.data_ptr(), raw_dev.shape[1])
        ctx.patchmatch(fid, P, seed)                  # warm-up
        ctx.sync()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            ctx.patchmatch(fid, P, seed)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b) / reps
    finally:
        ctx.set_matcher(False)
    return {"matcher": "AdaptMIPMFrameACMM, one pyramid level", "patch": 5, "iterations": 5, "top_k": 6,
            "ms_per_frame": round(ms, 2), "frames_per_s": round(1000.0 / ms, 3),
            "covers": "init + 10 half-sweeps + post-refine (matching only, no checks or focal stack)"}


# --------------------------------------------------------------------------
# batching and serving forms (python bench.py --forms)
# --------------------------------------------------------------------------
MIX = dict(sizes=((1024, 768), (2048, 1536), (4080, 3068)), pitch=(15.0, 30.0), K=(6, 18), planes=(3, 20),
           iters=(4, 12), patches=(11, 13, 15), seed=4242)


def mixed_frames(pfd, n, seed):
    """n distinct seeded frames of the mixed distribution: size uniform over
    1024x768 / 2048x1536 / 4080x3068, pitch U(15, 30) px, 6-18 neighbours, 3-20
    planes, patch 11/13/15, 4-12 PatchMatch iterations.  (workload, params, seed) each."""
    rs = np.random.RandomState(seed)
    out = []
    for i in range(n):
        W, H = MIX["sizes"][rs.randint(len(MIX["sizes"]))]
        pitch = float(np.float32(rs.uniform(*MIX["pitch"])))
        K = int(rs.randint(MIX["K"][0], MIX["K"][1] + 1))
        planes = int(rs.randint(MIX["planes"][0], MIX["planes"][1] + 1))
        iters = int(rs.randint(MIX["iters"][0], MIX["iters"][1] + 1))
        patch = int(rs.choice(MIX["patches"]))
        w = pfd.make_workload(W, H, pitch, planes, seed=seed * 1000 + i, max_nb=K)
        out.append((w, pfd.PmParams(base=pitch, patch_size=patch, max_iterations=iters), 5000 + i))
    return out


def _state_hash(st):
    import hashlib
    h = hashlib.sha1()
    for a in st:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _depth_tally(pfd, items, states):
    """Depth error of each frame's state against its scene: pooled matched
    fraction and fraction within 0.5 virtual depth, median of the frames'
    median errors."""
    meds, n_ok, w05, tot = [], 0.0, 0.0, 0
    for (w, _, _), st in zip(items, states):
        de = pfd.depth_error(w, st[0], cost=st[1])
        npx = st[0].shape[0]
        tot += npx
        n_ok += de["matched"] * npx
        w05 += de.get("within_0.5", 0.0) * de["matched"] * npx
        if "median_abs" in de:
            meds.append(de["median_abs"])
    return {"matched": round(n_ok / tot, 4), "within_0.5": round(w05 / max(n_ok, 1.0), 4),
            "median_abs_of_frames": round(float(np.median(meds)), 4) if meds else None}


def batching_leg(pfd, items):
    """The batching form on n resident frames (sizes, pitches, neighbour
    counts, patches and iteration counts all mixed), device-timed on one
    context's stream, every variant bit-identical per frame:
      plain     pfd_patchmatch frame after frame, default launch shape;
      graphs    the same from CUDA graphs (third repetition: captured, replayed);
      batched   pfd_patchmatch_batch, one persistent launch per half-sweep over
                all frames, autotuned launch shape (tuning in its first call);
    and the plain GPU method, the reference's own kernels (oracle/_ref) frame
    after frame, each frame timed on a block of 1024 of its views and scaled."""
    import torch
    ref_frame = load_ref_frame()
    out = {}
    with pfd.Context(0) as ctx:
        stream = torch.cuda.ExternalStream(ctx.stream, device="cuda:0")
        fids = [ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
                for w, _, _ in items]
        params = [P for _, P, _ in items]
        seeds = [sd for _, _, sd in items]

        def timed(fn):
            ctx.sync()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            return a.elapsed_time(b)

        def plain():
            for fid, P, sd in zip(fids, params, seeds):
                ctx.patchmatch(fid, P, sd)

        out["plain_ms"] = timed(plain)
        states = [ctx.download(f) for f in fids]
        want = [_state_hash(st) for st in states]
        out["depth_error"] = _depth_tally(pfd, items, states)
        del states
        ctx.set_graphs(True)
        timed(plain)                                  # uncaptured
        timed(plain)                                  # captured
        out["graphs_ms"] = timed(plain)
        same_g = all(_state_hash(ctx.download(f)) == h for f, h in zip(fids, want))
        ctx.set_graphs(False)
        ctx.set_sweep_shape(pfd.SHAPE_AUTOTUNE)
        out["batched_first_call_ms"] = timed(lambda: ctx.patchmatch_batch(fids, params, seeds))
        out["batched_ms"] = timed(lambda: ctx.patchmatch_batch(fids, params, seeds))
        same_b = all(_state_hash(ctx.download(f)) == h for f, h in zip(fids, want))
        out["tuned_shapes"] = sorted({int(ctx.tuned_sweep_shape(f, P)) for f, P in zip(fids, params)})
        for f in fids:
            ctx.frame_free(f)
    # the plain GPU method: the reference's kernels, one frame at a time
    ref_s = 0.0
    for w, P, sd in items:
        V = w.centers.shape[0]
        n = min(V, 1024)
        wb = block_first(pfd, w, n)
        with ref_frame.RefFrame(wb, philox=False) as ref:
            ms = ref.patchmatch_sample(P, sd, n)
        ref_s += (ms[0] + ms[1]) / 1e3 * V / n
    n_fr = len(items)
    counts = "/".join(str(sum(1 for w, _, _ in items if w.frame.raw.shape[1] == sz[0])) for sz in MIX["sizes"])
    best_ms = min(out["batched_ms"], out["plain_ms"], out["graphs_ms"])
    return {"config": "%d seeded frames, sizes uniform in 1024x768 / 2048x1536 / 4080x3068 (%s), pitch U(15, 30) px, "
                      "6-18 neighbours, 3-20 planes, patch 11-15, 4-12 iterations; u8 pixels (exact in FP16/BF16), "
                      "FP32 accumulation" % (n_fr, counts),
            "plain": {"ms": round(out["plain_ms"], 1), "frames_per_s": round(1e3 * n_fr / out["plain_ms"], 3)},
            "graphs": {"ms": round(out["graphs_ms"], 1), "frames_per_s": round(1e3 * n_fr / out["graphs_ms"], 3),
                       "bit_identical": same_g},
            "batched_autotuned": {"ms": round(out["batched_ms"], 1),
                                  "frames_per_s": round(1e3 * n_fr / out["batched_ms"], 3),
                                  "first_call_ms": round(out["batched_first_call_ms"], 1),
                                  "shapes_chosen": out["tuned_shapes"], "bit_identical": same_b},
            "plain_reference_gpu": {"s": round(ref_s, 1), "frames_per_s": round(n_fr / ref_s, 4),
                                    "how": "reference kernels (oracle/_ref, cuRAND, sync per launch) on 1024 views "
                                           "of each frame, scaled by views; matched depth error: the engine's equals "
                                           "the reference's on whole runs (tests/test_gpu_refpin.py)"},
            "depth_error": out["depth_error"],
            "speedup_vs_plain_reference_gpu": round(ref_s * 1e3 / best_ms, 2)}


def serving_leg(pfd, items, plain_fps, window_s=60.0, slots=4, seed=7):
    """The serving form: Poisson request streams of window_s seconds at rates
    below and above the plain method's throughput on the mix (plain_fps), each
    request a frame of the pool with its own 4-12 iterations and the filter,
    sent to a server with `slots` slots and a 150 GB budget and to a one-slot
    server (the plain method: one frame at a time).  frames/s over the makespan
    and p50/p99 latency (submission to result) for each; every result is the
    same bit for bit in both servers."""
    import time
    out = []
    for mult in (0.5, 1.0, 2.0):
        rate = mult * plain_fps
        rs = np.random.RandomState(seed + int(mult * 10))
        arrivals = []
        t = rs.exponential(1.0 / rate)
        while t < window_s:
            arrivals.append(t)
            t += rs.exponential(1.0 / rate)
        reqs = [(int(rs.randint(len(items))), int(rs.randint(4, 13)), 9000 + i) for i in range(len(arrivals))]

        def run(n_slots):
            with pfd.Server(0, hbm_budget=150 << 30, slots=n_slots) as srv:
                t0 = time.perf_counter()
                tickets = []
                for a, (idx, iters, sd) in zip(arrivals, reqs):
                    delay = t0 + a - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    w, P, _ = items[idx]
                    Q = pfd.PmParams(base=P.base, patch_size=P.patch_size, max_iterations=iters)
                    tickets.append(srv.submit(w, Q, sd, filter_cfg=pfd.FilterCfg(), baseline_unit=P.base))
                res = [srv.wait(tk) for tk in tickets]
                span = time.perf_counter() - t0
            lat = [r[4] for r in res]
            return ({"frames_per_s": round(len(res) / span, 3), "p50_ms": round(float(np.percentile(lat, 50)), 1),
                     "p99_ms": round(float(np.percentile(lat, 99)), 1), "makespan_s": round(span, 1)},
                    [_state_hash(r[:4]) for r in res])

        served, hs = run(slots)
        plain, hp = run(1)
        out.append({"rate_per_s": round(rate, 3), "requests": len(reqs), "served": dict(served, slots=slots),
                    "plain": plain, "bit_identical": hs == hp})
    return {"config": "Poisson streams of %.0f s from the %d-frame pool of the batching form, 4-12 iterations and the "
                      "filter per request, 150 GB budget; rates 0.5x / 1x / 2x the plain method's throughput on the mix "
                      "(%.3f frames/s)" % (window_s, len(items), plain_fps),
            "streams": out}


def run_forms(args):
    import torch
    torch.cuda.set_device(0)
    pfd = load_pfd()
    load_oracle()
    items = mixed_frames(pfd, args.forms_frames, MIX["seed"])
    out = {"forms": args.forms_legs}
    bat = batching_leg(pfd, items)
    out["batching"] = bat
    if "serving" in args.forms_legs:
        out["serving"] = serving_leg(pfd, items, bat["plain"]["frames_per_s"], window_s=args.forms_window)
    return out


def load_ref_frame():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_frame
    return ref_frame


def reference_workload(pfd, oracle, seed):
    """The frame of make_workload, built without the engine library: the
    synthetic raw frame (libpfd_synth.so), its windows cut on the host, and the
    oracle's SelectNeighbors lists (the first max_nb of each)."""
    wl = WORKLOAD
    fr = pfd.synth_frame(wl["width"], wl["height"], wl["pitch"], wl["n_planes"], seed,
                         n_lens_types=wl["n_lens_types"], blur_sigma=wl["blur_sigma"])
    mi = pfd.mi_window(wl["pitch"])
    keep = pfd.valid_views(fr, mi)
    centers = np.ascontiguousarray(fr.centers[keep])
    keys = np.ascontiguousarray(fr.tilekeys[keep])
    gray = pfd.slice_views(fr.raw, centers, mi)
    K = wl["max_nb"]
    ids, cnt, _ = oracle.select_neighbors(centers, keys, fr.n_cols, fr.n_rows, wl["pitch"], images=gray)
    nb_ids = np.ascontiguousarray(np.where(np.arange(K)[None, :] < np.minimum(cnt, K)[:, None], ids[:, :K], -1),
                                  np.int32)
    return pfd.Workload(fr, mi, centers, keys, nb_ids, np.minimum(cnt, K).astype(np.int32), gray)


def block_perm(V, n):
    """Views in the order of block_first: a block of n from the middle of the
    frame (key order) first, the rest after it."""
    v0 = max(0, V // 2 - n // 2)
    return np.concatenate([np.arange(v0, v0 + n), np.arange(0, v0), np.arange(v0 + n, V)])


def block_first(pfd, w, n):
    """w with a block of n views from the middle of the frame (key order)
    renumbered to the front, the rest after it, lists renumbered."""
    V = w.centers.shape[0]
    perm = block_perm(V, n)
    pos = np.empty(V, np.int64)
    pos[perm] = np.arange(V)
    ids = w.nb_ids[perm]
    ids = np.where(ids >= 0, pos[np.maximum(ids, 0)], -1).astype(np.int32)
    return pfd.Workload(w.frame, w.mi, np.ascontiguousarray(w.centers[perm]), np.ascontiguousarray(w.tilekeys[perm]),
                        np.ascontiguousarray(ids), np.ascontiguousarray(w.nb_counts[perm]),
                        np.ascontiguousarray(w.gray[perm]))


def run_reference(args, rank, world):
    """The reference's implementation of the path, on this box: its own frame
    PatchMatch kernels (MIStereo/CudaUtil.cu + AdaptMIPMFrame.cu +
    AdaptMIPMUtil.cu, compiled from its sources with its flags into
    oracle/_ref, launched by its RunPatchMatchCUDAForFrame_Impl with a device
    synchronisation after every launch, cuRAND seeded with a fixed seed), and
    the CPU restatements of its host-side stages (SelectNeighbors +
    MISimilarityMeasure with threads over views, MICycleCheckerCPU and
    MIDisparityFilterCPU on one thread, the focal stack with threads).  The
    engine library is never loaded.  Each step is a bounded sample: the
    selection and the checks on the whole frame (the checks on the state of the
    reference's own full run, made once before the steps), the PatchMatch on a
    block of views scaled to the frame, the focal stack on 4 of the slices
    scaled to all."""
    if rank != 0:
        return None
    pfd = load_pfd()
    oracle = load_oracle()
    ref_frame = load_ref_frame()
    if not ref_frame.available():
        return {"impl": "reference", "unavailable": "oracle/_ref is not built (make -C oracle/ref needs the "
                                                      "reference tree)"}
    import torch
    torch.cuda.set_device(0)
    nth = cpu_threads()
    seed = WORKLOAD["seed"]
    w = reference_workload(pfd, oracle, seed)
    params = pm_params(pfd)
    V = w.centers.shape[0]
    with ref_frame.RefFrame(w, philox=False) as ref:
        full_ms = ref.patchmatch(params, seed)
        plane, cost, disp, sel = ref.download()
    converged = dict(plane=plane, cost=cost, disp=disp, sel=sel)
    depth = pfd.depth_error(w, plane, cost=cost)
    full_s = (full_ms[0] + full_ms[1]) / 1e3
    n = int(min(V, max(1024, V * 2.0 / max(full_s, 1e-3))))
    wb = block_first(pfd, w, n)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    # the checks' sample: a quarter of the frame's views (a block in key order from
    # the middle), neighbours outside it dropped, scaled by views
    nchk = max(1, V // 4)
    pc = block_perm(V, nchk)[:nchk]
    wc = block_first(pfd, w, nchk)
    ids_c = np.ascontiguousarray(np.where(wc.nb_ids[:nchk] < nchk, wc.nb_ids[:nchk], -1), np.int32)
    orc_c = oracle.Oracle(wc.gray[:nchk], wc.centers[:nchk], ids_c, wc.nb_counts[:nchk])
    ppv = w.mi * w.mi
    conv_c = {k: np.ascontiguousarray(v.reshape((V, ppv) + v.shape[1:])[pc].reshape((nchk * ppv,) + v.shape[1:]))
              for k, v in converged.items()}
    unit = WORKLOAD["pitch"]
    ow, oh = stack_size()
    vds = slice_vds()
    svds = vds[[len(vds) // 4, (3 * len(vds)) // 4]]
    vals, rows = [], []
    with ref_frame.RefFrame(wb, philox=False) as refb:
        # a block of views fills fewer waves of the reference's grid than the frame,
        # so its time scaled by views overstates the frame's; the ratio of the
        # whole-frame run to the scaled block, measured once, corrects it
        ms0 = refb.patchmatch_sample(params, seed, n)
        calib = full_s / max((ms0[0] + ms0[1]) / 1e3 * V / n, 1e-9)
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            oracle.select_neighbors(w.centers, w.tilekeys, w.frame.n_cols, w.frame.n_rows, unit, images=w.gray)
            t_sel = time.perf_counter() - t0
            ms = refb.patchmatch_sample(params, seed, n)
            t_pm = (ms[0] + ms[1]) / 1e3 * V / n * calib
            st = {k: v.copy() for k, v in conv_c.items()}
            t1 = time.perf_counter()
            oracle.cycle_check(orc_c, pfd.CycleCfg(), unit, st)
            oracle.filter_global(orc_c, pfd.FilterCfg(), unit, st)
            oracle.reprojection_error(orc_c, pfd.FilterCfg(), unit, st)
            t_chk = (time.perf_counter() - t1) * V / nchk
            t2 = time.perf_counter()
            oracle.refocus(orc, WORKLOAD["width"], WORKLOAD["height"], svds, ow, oh)
            t_stack = (time.perf_counter() - t2) * len(vds) / len(svds)
            frame_s = t_sel + t_pm + t_chk + t_stack
            if i >= args.warmup:
                vals.append(1.0 / frame_s)
                rows.append((t_sel, t_pm, t_chk, t_stack))
    value = statistics.median(vals)
    med = [statistics.median(r[j] for r in rows) for j in range(4)]
    sample = ("reference PatchMatch kernels (oracle/_ref, compiled from the reference's sources, cuRAND, sync per "
              "launch) on %d of %d micro-images scaled to the frame by views and by the whole frame's measured ratio "
              "%.3f (%.2f s; the whole frame once: %.2f s init + %.2f s sweeps); oracle SelectNeighbors on every view "
              "(%.2f s, %d threads); cycle check + filter + reprojection map of the reference run's state on %d of the "
              "views, scaled (%.2f s, 1 thread); focal stack 2 of %d slices scaled (%.2f s, %d threads)" %
              (n, V, calib, med[1], full_ms[0] / 1e3, full_ms[1] / 1e3, med[0], nth, nchk, med[2], len(vds), med[3],
               nth))
    return {
        "metric": metric(), "value": round(value, 6), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "impl": "reference", "dtype": "f32",
        "data": "synthetic (seeded plenoptic raw frame)",
        "config": {"workload": workload_text(V, ow, oh)},
        "cpu_baseline": {"value": round(value, 6), "unit": "frames/s", "cores": nth, "kind": "reference",
                         "sample": sample},
        "plain_reference_gpu": {"frames_per_s": round(1.0 / full_s, 4), "init_ms": round(full_ms[0], 1),
                                "sweeps_ms": round(full_ms[1], 1),
                                "covers": "RunPatchMatchCUDAForFrame_Impl on the whole frame: init + %d half-sweeps"
                                          % (2 * WORKLOAD["iterations"])},
        "depth_error": dict({k: round(v, 4) for k, v in depth.items()},
                            against="the scene's true virtual depth at each raw pixel (reference's own run)"),
        "e2e": {"value": round(value, 6), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def workload_text(V, ow, oh) -> str:
    return ("%dx%d raw, pitch %.1f px, 3 lens types, %d planes, %d micro-images, K=%d neighbours chosen by "
            "SelectNeighbors (similarity), %dx%d bilateral NCC, %d PatchMatch iterations, FP32; cycle check, "
            "disparity filter + reprojection map; %d-slice focal stack to %dx%d" %
            (WORKLOAD["width"], WORKLOAD["height"], WORKLOAD["pitch"], WORKLOAD["n_planes"], V, WORKLOAD["max_nb"],
             WORKLOAD["patch_size"], WORKLOAD["patch_size"], WORKLOAD["iterations"], WORKLOAD["slices"], ow, oh))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", action="store_true", help="measure the batching and serving forms instead")
    ap.add_argument("--forms-frames", type=int, default=64)
    ap.add_argument("--forms-window", type=float, default=60.0)
    ap.add_argument("--forms-legs", default="batching,serving")
    ap.add_argument("--frame", default=None, help="WxH override (profiling captures of a smaller frame)")
    ap.add_argument("--iterations", type=int, default=None, help="PatchMatch iterations override (profiling)")
    ap.add_argument("--fetch", choices=["shared", "texture"], default="shared",
                    help="where the half-sweeps read neighbour samples (pfd_set_sweep_fetch)")
    args = ap.parse_args()
    if args.frame:
        wdt, hgt = args.frame.lower().split("x")
        WORKLOAD["width"], WORKLOAD["height"] = int(wdt), int(hgt)
    if args.iterations is not None:
        WORKLOAD["iterations"] = args.iterations
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.forms:
        print(json.dumps(run_forms(args)), flush=True)
        return
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_engine(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
