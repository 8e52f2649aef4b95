#!/usr/bin/env python3
"""Benchmark: MO VGL electron-points/s on B200 (config-1 molecule).

One step = one evaluation of AO VGL + MO VGL for every electron point of the
workload (walkers x electrons), the reference's qmckl_get_mo_basis_mo_vgl.

  value  device-resident throughput: coordinates already in HBM, outputs left
         in HBM, timed with CUDA events on the evaluation stream, L2 flushed
         (256 MB write) before every timed step.
  e2e    the same through the public host API: qmckl_set_electron_coord from
         pinned host memory + qmckl_get_mo_basis_mo_vgl into pinned host memory
         (both copies inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--form mixed|fp64]
  python bench.py --impl reference     # the CPU reference path on host cores

Under torchrun (N > 1) every rank evaluates its own full workload on its own
GPU (walkers are independent; no collective on the data path): weak scaling,
value = points of all ranks / max over ranks of the timed region.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MO VGL electron-points/s on 1 B200, mixed vs FP64 form at <=1e-6 rel err"
WORKLOAD = "config-1 molecule: 80 nuclei (40 C/N/O + 40 H), cc-pVTZ-shaped cartesian basis, 2000 AOs, 160 MOs, 318 electrons x 512 walkers"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            parts = dict(kv.split("=", 1) for kv in line.split() if "=" in kv)
            if "kernel" in parts and "bytes_per_launch" in parts:
                out[(parts["kernel"], parts.get("form", ""))] = float(parts["bytes_per_launch"])
    return out


class ClockSampler:
    """SM clock and throttle reasons sampled every ~10 ms (NVML) during the timed region."""

    # NVML clocks-event-reason bits
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.stop_flag = False
        self.thread = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.gpu]) if vis else self.gpu
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception as e:   # no NVML: report it, keep running
            self.err = str(e)
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        nv = self.nv
        while not self.stop_flag:
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for b, name in self.REASONS.items():
                    if bits & b:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable: " + getattr(self, "err", "")]}
        self.stop_flag = True
        self.thread.join(timeout=2)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "NVML, 10 ms polling"}


def cpu_baseline(sysd, seconds=15.0, nthreads=0):
    """Time the CPU oracle (a restatement of the reference's C HPC path) on a bounded sample."""
    from oracle import pyoracle as O
    pts = sysd["elec_coord"].reshape(-1, 3)
    b = O.Basis(sysd)
    nthreads = nthreads or os.cpu_count() or 1
    n = 64
    done, t_total = 0, 0.0
    while t_total < seconds and done < pts.shape[0]:
        chunk = pts[done:done + n]
        t0 = time.perf_counter()
        ao = O.ao_vgl(b, chunk, sysd["nucl_coord"], nthreads=nthreads)
        O.mo_vgl(sysd["mo_coef"], ao, nthreads=nthreads)
        t_total += time.perf_counter() - t0
        done += chunk.shape[0]
        n = min(2 * n, 4096)
    return {"value": done / t_total, "unit": "electron-points/s", "cores": nthreads, "kind": "port",
            "sample": f"{done} of {pts.shape[0]} points of the workload, AO VGL + MO VGL, {t_total:.1f} s"}


def run_reference(args):
    import torch.distributed as dist  # noqa: F401  (only for rank detection)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from qmckl_b200 import gen
    sysd = gen.config(1)
    P = sysd["elec_coord"].shape[0] * sysd["elec_coord"].shape[1]
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        base = cpu_baseline(sysd, seconds=max(2.0, 20.0 / max(1, args.steps)))
        if i >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "electron-points/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * P / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, qmckl_b200/gen.py)",
            "config": {"workload": WORKLOAD, "points": P, "form": "reference CPU path"},
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "electron-points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def profile_case(kind, walkers=64):
    """One evaluation of the config-1 molecule on `walkers` walkers, for ncu captures."""
    import torch
    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200.system import make_context
    d = gen.config(1, walk_num=walkers)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    ctx = make_context(d, points=False, form=pq.FORM_FP64 if kind == "fp64" else pq.FORM_MIXED)
    if kind != "fp64":
        pq.b200_set_mixed_kernel(ctx, kind == "fused")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    pq.context_destroy(ctx)
    print(f"profile case {kind}: {P} points")


def _events_time(stream, fn, steps, flush=None, after=None):
    """Median device time (ms) of fn() over `steps` calls, CUDA events on `stream`."""
    import torch
    ts = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        if after is not None:
            after()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts), ts


def case_batched(args):
    """Config 2: 256 independent molecules, one persistent launch (CUDA graph) vs a per-system launch loop."""
    import torch
    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200.system import make_context
    t0 = time.time()
    systems = gen.batch_config()
    ctxs = [make_context(s, points=False, form=pq.FORM_MIXED) for s in systems]
    P = [gen.points(s).shape[0] for s in systems]
    b = pq.b200_batch_create(ctxs, P)
    setup_s = time.time() - t0
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    pq.b200_batch_set_stream(b, stream.cuda_stream)
    co, oo, (ct, ot) = pq.b200_batch_layout(b, len(ctxs))
    coord = np.zeros(ct)
    for s, sysd in enumerate(systems):
        coord[co[s]:co[s] + 3 * P[s]] = gen.points(sysd).T.reshape(-1)
    d_coord = torch.tensor(coord, dtype=torch.float64, device="cuda")
    d_out = torch.empty(ot, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    best = pq.b200_batch_tune(b, d_coord.data_ptr(), d_out.data_ptr(), 2)
    tuning = pq.b200_batch_get_tuning(b)
    pq.b200_batch_set_graph(b, True)

    def persistent():
        pq.b200_batch_mo_vgl_device(b, d_coord.data_ptr(), d_out.data_ptr())

    def check():
        assert pq.b200_batch_synchronize(b) == 0

    def loop():
        pq.b200_batch_mo_vgl_loop_device(b, d_coord.data_ptr(), d_out.data_ptr())

    for _ in range(max(3, args.warmup)):
        persistent()
        check()
    n = max(3, min(args.steps, 10))
    t_p, _ = _events_time(stream, persistent, n, flush, check)
    for _ in range(2):
        loop()
    t_l, _ = _events_time(stream, loop, n, flush)
    flops = sum(10.0 * p * s["ao_num"] * s["mo_num"] for p, s in zip(P, systems))
    line = {"case": "batched systems: 256 molecules, 5-80 nuclei, cc-pVDZ/TZ shapes, 16-256 walkers",
            "systems": len(systems), "points": int(sum(P)), "form": "mixed",
            "persistent_ms": t_p, "loop_ms": t_l, "loop_over_persistent": t_l / t_p,
            "points_per_s": sum(P) / (t_p * 1e-3), "dense_equivalent_tflops": flops / (t_p * 1e-3) / 1e12,
            "tuning": {"producer_warps": tuning[0], "queue_order": tuning[1], "tuned_ms": best},
            "graph": True, "setup_s": setup_s, "steps": n,
            "timing": "CUDA events on the batch stream, median, 256 MB L2 flush before each step"}
    print(json.dumps(line))
    pq.b200_batch_destroy(b)
    for c in ctxs:
        pq.context_destroy(c)


def case_adjoint(args):
    """Config 3: forward MO VGL + adjoint (coefficient, nuclear, point gradients), config-1 molecule, 128 walkers."""
    import torch
    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200.system import make_context
    d = gen.config(3)
    pts = gen.points(d)
    P, A, M, N = pts.shape[0], d["ao_num"], d["mo_num"], d["nucl_num"]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    w = torch.randn((P, 5, M), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    out = torch.empty((P, 5, M), dtype=torch.float64, device="cuda")
    gc = torch.empty((M, A), dtype=torch.float64, device="cuda")
    gn = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    gr = torch.empty((3, P), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    res = {}
    for name, form in (("fp64", pq.FORM_FP64), ("mixed", pq.FORM_MIXED)):
        ctx = make_context(d, points=False, form=form)
        pq.b200_set_stream(ctx, stream.cuda_stream)
        fwd = lambda: pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        bwd = lambda: pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), w.data_ptr(), gc.data_ptr(),
                                                    gn.data_ptr(), gr.data_ptr())
        for _ in range(3):
            fwd()
            bwd()
        torch.cuda.synchronize()
        tf, _ = _events_time(stream, fwd, max(3, min(args.steps, 20)), flush)
        tb, _ = _events_time(stream, bwd, max(3, min(args.steps, 20)), flush)
        res[name] = {"forward_ms": tf, "backward_ms": tb, "points_per_s_fwd_bwd": P / ((tf + tb) * 1e-3)}
        pq.context_destroy(ctx)
    print(json.dumps({"case": "adjoint: config-1 molecule, 128 walkers, L = sum W * mo_vgl", "points": P,
                      "ao_num": A, "mo_num": M, "results": res,
                      "timing": "CUDA events, median, 256 MB L2 flush before each call"}))


def case_large(args):
    """Config 4: 200 nuclei, 5000 AOs, 350 MOs, 700 electrons x 256 walkers: fused mixed vs unfused FP64."""
    import torch
    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200.system import make_context
    d = gen.config(4)
    pts = gen.points(d)
    P, A, M = pts.shape[0], d["ao_num"], d["mo_num"]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    out = torch.empty((P, 5, M), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    res = {}
    ref = None
    for name, form in (("fp64_unfused", pq.FORM_FP64), ("mixed_fused", pq.FORM_MIXED)):
        ctx = make_context(d, points=False, form=form)
        pq.b200_set_stream(ctx, stream.cuda_stream)
        fn = lambda: pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        t, _ = _events_time(stream, fn, max(3, min(args.steps, 10)), flush)
        res[name] = {"ms": t, "points_per_s": P / (t * 1e-3)}
        if ref is None:
            ref = out.clone()
        else:
            diff = (out - ref).abs()
            res[name]["max_abs_over_max_ref"] = {
                n: float(diff[:, c, :].max() / ref[:, c, :].abs().max())
                for c, n in enumerate(["value", "grad_x", "grad_y", "grad_z", "laplacian"])}
        pq.context_destroy(ctx)
    res["speedup"] = res["fp64_unfused"]["ms"] / res["mixed_fused"]["ms"]
    print(json.dumps({"case": "large: 200 nuclei, 5000 AOs, 350 MOs, 700 electrons x 256 walkers", "points": P,
                      "ao_num": A, "mo_num": M, "results": res,
                      "timing": "CUDA events, median, 256 MB L2 flush before each call"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default=os.environ.get("QMCKL_B200_BENCH_FORM", "mixed"), choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--unfused", action="store_true",
                    help="mixed form with the AO pieces written to HBM and a separate tensor-core GEMM")
    ap.add_argument("--pieces", type=int, default=3, choices=[2, 3],
                    help="operand split of the mixed form: 3 bfloat16 pieces (default) or 2 float16 pieces")
    ap.add_argument("--profile", choices=["fused", "split", "fp64"],
                    help="run one evaluation of a small case (config-1 molecule, 64 walkers) for ncu; no timing")
    ap.add_argument("--case", choices=["batched", "adjoint", "large"],
                    help="measure another workload instead of the headline one (one JSON line)")
    args = ap.parse_args()
    if args.case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return {"batched": case_batched, "adjoint": case_adjoint, "large": case_large}[args.case](args)
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return profile_case(args.profile)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200 import replicas
    from qmckl_b200.system import make_context

    sysd = gen.config(1)
    W, E = sysd["elec_coord"].shape[:2]
    P, A, M = W * E, sysd["ao_num"], sysd["mo_num"]
    form = pq.FORM_MIXED if args.form == "mixed" else pq.FORM_FP64
    ctx = make_context(sysd, points=False, form=form)
    if form == pq.FORM_MIXED:
        pq.b200_set_split_terms(ctx, args.pieces)
        if args.unfused:
            pq.b200_set_mixed_kernel(ctx, False)
    stream = torch.cuda.Stream()          # evaluation stream shared by torch and the library
    torch.cuda.set_stream(stream)
    pq.b200_set_stream(ctx, stream.cuda_stream)

    coord_t = np.ascontiguousarray(gen.points(sysd).T)               # [3][P]
    d_coord = torch.tensor(coord_t, dtype=torch.float64, device="cuda")
    d_mo = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    d_ao = torch.empty(P * 5 * A, dtype=torch.float64, device="cuda") if form == pq.FORM_FP64 else None
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        pq.b200_mo_vgl_device(ctx, P, d_coord.data_ptr(), d_mo.data_ptr())

    # accuracy of the timed form against the FP64 form on the same points
    err = None
    if form == pq.FORM_MIXED:
        step()
        torch.cuda.synchronize()
        mixed = d_mo.clone()
        ctx64 = make_context(sysd, points=False, form=pq.FORM_FP64)
        pq.b200_set_stream(ctx64, stream.cuda_stream)
        pq.b200_mo_vgl_device(ctx64, P, d_coord.data_ptr(), d_mo.data_ptr())
        torch.cuda.synchronize()
        ref = d_mo.view(P, 5, M)
        diff = (mixed.view(P, 5, M) - ref).abs()
        err = {"max_abs_over_max_ref": {n: float(diff[:, c, :].max() / ref[:, c, :].abs().max())
                                         for c, n in enumerate(["value", "grad_x", "grad_y", "grad_z", "laplacian"])},
               "reference": "FP64 form on the GPU (itself checked against the CPU oracle in tests/)"}
        pq.context_destroy(ctx64)
        del mixed, ref, diff

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = pq.b200_kernel_launch_count()
    fused_path = form == pq.FORM_MIXED and not args.unfused
    if fused_path:
        pq.b200_get_kblock_stats(ctx, reset=True)
    times = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    launches = pq.b200_kernel_launch_count() - launches0
    kb_eval, kb_total = pq.b200_get_kblock_stats(ctx) if fused_path else (0, 0)
    # dominant-kernel timing: the AO kernel alone (same stream, same events)
    ao_times = []
    if form == pq.FORM_FP64:
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pq.b200_ao_vgl_device(ctx, P, d_coord.data_ptr(), d_ao.data_ptr())
            e1.record(stream)
            e1.synchronize()
            ao_times.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    ms = replicas.max_over_ranks(statistics.mean(times), device="cuda")

    # end to end through the public host API (pinned host buffers)
    h_coord = torch.from_numpy(np.ascontiguousarray(sysd["elec_coord"].reshape(-1))).pin_memory()
    h_out = torch.empty(P * 5 * M, dtype=torch.float64).pin_memory()
    ctx_e = make_context(sysd, points=True, form=form)
    pq.b200_set_stream(ctx_e, stream.cuda_stream)
    lib = pq.lib()
    import ctypes as C

    def e2e_step():
        rc = lib.qmckl_set_electron_coord(C.c_int64(ctx_e), C.c_char(b"N"), C.c_int64(W),
                                          C.c_void_p(h_coord.data_ptr()), C.c_int64(P * 3))
        assert rc == 0, pq.last_error(ctx_e)
        rc = lib.qmckl_get_mo_basis_mo_vgl(C.c_int64(ctx_e), C.c_void_p(h_out.data_ptr()), C.c_int64(P * 5 * M))
        assert rc == 0, pq.last_error(ctx_e)

    for _ in range(2):
        e2e_step()
    e2e_times = []
    for _ in range(max(3, args.steps // 2)):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        e2e_times.append(e0.elapsed_time(e1))
    pq.context_destroy(ctx_e)
    e2e_ms = replicas.max_over_ranks(statistics.mean(e2e_times), device="cuda")

    hbm, bf16, bf16_sus, peak_src = load_peaks()
    traffic = load_traffic()
    if form == pq.FORM_FP64:
        ao_ms = statistics.mean(ao_times)
        algo_bytes = 5.0 * P * A * 8 + 24.0 * P      # dense ao_vgl write + coordinates
        achieved = algo_bytes / (ao_ms * 1e-3) / 1e9
        roofline = {"kernel": "ao_f64_kernel<5> (AO VGL, FP64)", "bound": "hbm", "achieved": achieved,
                    "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": peak_src,
                    "traffic": traffic.get(("ao_f64_kernel", "fp64")), "ms_per_launch": ao_ms,
                    "algorithmic_bytes_per_launch": algo_bytes,
                    "other_kernel": {"kernel": "dgemm_kernel (MO VGL, FP64 mma.sync m8n8k4)",
                                     "ms_per_launch": ms - ao_ms,
                                     "tflops": 2.0 * 5 * P * A * M / ((ms - ao_ms) * 1e-3) / 1e12}}
    else:
        # fused kernel: 25 points x 5 components per 128-row MMA tile, MOs in
        # N tiles of n_tile columns, 64-AO K blocks (those that vanish over a
        # tile are skipped: the kernel counts the blocks it evaluates);
        # 6 split-BF16 products (3 for float16 x 2) per K step
        flops = 2.0 * 5 * P * A * M
        n_tiles = -(-M // 256)
        n_tile = -(-(-(-M // n_tiles)) // 16) * 16
        while n_tile > 160:
            n_tiles += 1
            n_tile = -(-(-(-M // n_tiles)) // 16) * 16
        nprod = 6 if args.pieces == 3 else 3
        executed = 2.0 * (kb_eval / args.steps) * 128 * n_tile * 64 * nprod
        t = traffic.get(("fused_mo_kernel", "mixed"))
        kname = ("fused_mo_kernel<3,5> (AO -> split-BF16 tcgen05 MO VGL" if args.pieces == 3 else
                 "fused_mo_kernel<2,5> (AO -> split-FP16 tcgen05 MO VGL") + "; step = 3 ordering kernels + tile plan + this)"
        if args.unfused:
            # AO pieces to HBM, then 128-row tiles of the 5P x A pieces matrix x 6 products
            executed = 2.0 * (-(-5 * P // 128) * 128) * (n_tile * n_tiles) * (-(-A // 64) * 64) * 6
            kname = "ao_tile_kernel<3,5> + tc_gemm_kernel<3,2> (unfused mixed form; whole step)"
            t = None
        achieved = executed / (ms * 1e-3) / 1e12
        roofline = {"kernel": kname,
                    "bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                    "frac": achieved / bf16, "peak_source": peak_src,
                    "traffic": t * P / 20352.0 if t else None,
                    "traffic_note": "ncu dram bytes of a 20,352-point launch scaled by points" if t else None,
                    "executed_tensor_flop_per_launch": executed,
                    "dense_equivalent_tflops": flops / (ms * 1e-3) / 1e12,
                    "k_blocks_evaluated_fraction": (kb_eval / kb_total) if kb_total else None,
                    "output_bytes_per_launch": 40.0 * P * M}

    value = world * P / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "electron-points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if form == pq.FORM_FP64 else ("f32/bf16x3" if args.pieces == 3 else "f32/f16x2"),
        "data": "synthetic (seeded generator qmckl_b200/gen.py, no dataset)",
        "config": {"workload": WORKLOAD, "points": P, "ao_num": A, "mo_num": M,
                   "form": args.form, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed (256 MB write) before every timed step; AO matrix >> L2"},
        "e2e": {"value": world * P / (e2e_ms * 1e-3), "unit": "electron-points/s",
                "h2d_bytes_per_step": int(P * 3 * 8), "d2h_bytes_per_step": int(P * 5 * M * 8),
                "ms_per_step": e2e_ms},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "roofline": roofline,
    }
    if err is not None:
        line["error_vs_fp64"] = err
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sysd)
    pq.context_destroy(ctx)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
