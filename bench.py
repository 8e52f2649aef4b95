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
                out[(parts["kernel"], parts.get("form", ""))] = (float(parts.get("points", 0)),
                                                                 float(parts["bytes_per_launch"]))
    return out


def _scaled_traffic(kernel, form, P):
    """Per-launch DRAM bytes of `kernel` at P points, from the capture in profiles/dram_traffic.txt."""
    cap = load_traffic().get((kernel, form))
    return cap[1] * P / cap[0] if cap and cap[0] > 0 else None


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


def physical_cores():
    """(physical cores, how counted): unique (core, socket) pairs of lscpu, else os.cpu_count()."""
    import subprocess
    try:
        out = subprocess.run(["lscpu", "-p=CORE,SOCKET"], capture_output=True, text=True, timeout=10).stdout
        pairs = {tuple(line.split(",")) for line in out.splitlines() if line and not line.startswith("#")}
        if pairs:
            return len(pairs), "physical (lscpu)"
    except Exception:
        pass
    return os.cpu_count() or 1, "logical (os.cpu_count)"


def _cpu_rate(evaluate, pts, seconds, first_chunk):
    """points/s of evaluate(chunk) over chunks of the workload's points until `seconds` have passed."""
    n, done, t_total = first_chunk, 0, 0.0
    while t_total < seconds and done < pts.shape[0]:
        chunk = pts[done:done + n]
        t0 = time.perf_counter()
        evaluate(chunk)
        t_total += time.perf_counter() - t0
        done += chunk.shape[0]
        n = min(2 * n, 8192)
    return done / t_total, done, t_total


def cpu_baseline(sysd, seconds=12.0, nthreads=0, single_thread_seconds=4.0):
    """Time the CPU path on a bounded sample of the workload's points: the
    reference's own C HPC kernels when they were built into oracle/_ref,
    else the oracle (a restatement of the same path); all physical cores,
    plus a 1-thread figure."""
    from oracle import pyoracle as O
    pts = sysd["elec_coord"].reshape(-1, 3)
    cores, how = physical_cores()
    nthreads = nthreads or cores
    ref = None
    try:
        from oracle import refpath
        ref = refpath.RefSystem(sysd) if refpath.available() else None
    except Exception:
        ref = None
    if ref is not None:
        kind, what = "reference", "the reference's C HAVE_HPC kernels (oracle/_ref)"
        evaluate = lambda c, t: ref.mo_vgl(c, nthreads=t)
    else:
        kind, what = "port", "the oracle (C restatement of the reference's HPC path)"
        b = O.Basis(sysd)
        evaluate = lambda c, t: O.mo_vgl(sysd["mo_coef"], O.ao_vgl(b, c, sysd["nucl_coord"], nthreads=t), nthreads=t)
    v, done, t = _cpu_rate(lambda c: evaluate(c, nthreads), pts, seconds, 16 * nthreads)
    v1, done1, t1 = _cpu_rate(lambda c: evaluate(c, 1), pts, single_thread_seconds, 64)
    return {"value": v, "unit": "electron-points/s", "cores": nthreads, "cores_counted": how, "kind": kind,
            "sample": f"{done} of {pts.shape[0]} points of the workload, AO VGL + MO VGL by {what}, {t:.1f} s",
            "single_thread": {"value": v1, "sample": f"{done1} points, {t1:.1f} s"}}


def workload_config(P, A, M, world):
    """The config dict both arms print (identical keys and values)."""
    return {"workload": WORKLOAD, "points": P, "ao_num": A, "mo_num": M,
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "GPU arm: L2 flushed (256 MB write) before every timed step; AO matrix >> L2"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from qmckl_b200 import gen
    sysd = gen.config(1)
    P = sysd["elec_coord"].shape[0] * sysd["elec_coord"].shape[1]
    vals = []
    base = None
    # each step: up to the whole workload (about 0.8 s on 16 cores), so that
    # the default 5 + 100 steps end in about three minutes
    per_step = max(1.0, 20.0 / max(1, args.warmup + args.steps))
    for i in range(args.warmup + args.steps):
        base = cpu_baseline(sysd, seconds=per_step, single_thread_seconds=0.5 if i < args.warmup + args.steps - 1 else 3.0)
        if i >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "electron-points/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * P / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, qmckl_b200/gen.py)",
            "config": workload_config(P, sysd["ao_num"], sysd["mo_num"], world),
            "form": "reference CPU path (" + base["kind"] + ")",
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": "electron-points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def profile_case(kind, walkers=64):
    """One evaluation of the config-1 molecule on `walkers` walkers, for ncu
    captures; "adjoint": the config-3 workload (config-1 molecule, 128
    walkers), mixed-form forward and MO VGL adjoint, called twice."""
    import torch
    from qmckl_b200 import gen
    from qmckl_b200 import qmckl as pq
    from qmckl_b200.system import make_context
    d = gen.config(3) if kind == "adjoint" else gen.config(1, walk_num=walkers)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    A, M, N = d["ao_num"], d["mo_num"], d["nucl_num"]
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    ctx = make_context(d, points=False, form=pq.FORM_FP64 if kind == "fp64" else pq.FORM_MIXED)
    if kind in ("fused", "split"):
        pq.b200_set_mixed_kernel(ctx, kind == "fused")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    if kind == "adjoint":
        w = torch.randn((P, 5, M), dtype=torch.float64, device="cuda",
                        generator=torch.Generator("cuda").manual_seed(3))
        gc = torch.empty((M, A), dtype=torch.float64, device="cuda")
        gn = torch.empty((N, 3), dtype=torch.float64, device="cuda")
        gr = torch.empty((3, P), dtype=torch.float64, device="cuda")
        for _ in range(2):
            pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), w.data_ptr(), gc.data_ptr(), gn.data_ptr(),
                                          gr.data_ptr())
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
    line = {"case": "config 2: 256 molecules, 5-80 nuclei, cc-pVDZ/TZ shapes, 16-256 walkers",
            "systems": len(systems), "points": int(sum(P)), "form": "mixed",
            "persistent_ms": t_p, "loop_ms": t_l, "loop_over_persistent": t_l / t_p,
            "points_per_s": sum(P) / (t_p * 1e-3), "dense_equivalent_tflops": flops / (t_p * 1e-3) / 1e12,
            "tuning": {"producer_warps": tuning[0], "queue_order": tuning[1], "tuned_ms": best},
            "graph": True, "setup_s": setup_s, "steps": n,
            "timing": "CUDA events on the batch stream, median, 256 MB L2 flush before each step"}
    pq.b200_batch_destroy(b)
    for c in ctxs:
        pq.context_destroy(c)
    return line


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
    return {"case": "config 3, adjoint: config-1 molecule, 128 walkers, L = sum W * mo_vgl", "points": P,
            "ao_num": A, "mo_num": M, "results": res, "steps": max(3, min(args.steps, 20)),
            "timing": "CUDA events, median, 256 MB L2 flush before each call"}


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
    return {"case": "config 4, large: 200 nuclei, 5000 AOs, 350 MOs, 700 electrons x 256 walkers", "points": P,
            "ao_num": A, "mo_num": M, "results": res, "steps": max(3, min(args.steps, 10)),
            "timing": "CUDA events, median, 256 MB L2 flush before each call"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default=os.environ.get("QMCKL_B200_BENCH_FORM", "mixed"), choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the configs 2, 3 and 4 measured after the headline workload")
    ap.add_argument("--unfused", action="store_true",
                    help="mixed form with the AO pieces written to HBM and a separate tensor-core GEMM")
    ap.add_argument("--pieces", type=int, default=3, choices=[2, 3],
                    help="operand split of the mixed form: 3 bfloat16 pieces (default) or 2 float16 pieces")
    ap.add_argument("--profile", choices=["fused", "split", "fp64", "adjoint"],
                    help="run one evaluation of a small case (config-1 molecule, 64 walkers) for ncu; no timing")
    ap.add_argument("--walkers", type=int, default=64, help="walkers of the --profile case (config-1 molecule)")
    ap.add_argument("--case", choices=["batched", "adjoint", "large"],
                    help="measure another workload instead of the headline one (one JSON line)")
    args = ap.parse_args()
    if args.case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps({"batched": case_batched, "adjoint": case_adjoint, "large": case_large}[args.case](args)))
        return
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return profile_case(args.profile, args.walkers)

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
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        pq.b200_mo_vgl_device(ctx, P, d_coord.data_ptr(), d_mo.data_ptr())

    for _ in range(args.warmup):
        step()
    pq.b200_synchronize(ctx)
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
    pq.b200_synchronize(ctx)   # also reports a bounded wait that gave up
    launches = pq.b200_kernel_launch_count() - launches0
    ks_eval, ks_total = pq.b200_get_kblock_stats(ctx) if fused_path else (0, 0)
    clocks = sampler.stop()
    ms = replicas.max_over_ranks(statistics.mean(times), device="cuda")

    # the FP64 form on the same GPU: the whole step and the FP64 AO kernel alone
    ctx64 = make_context(sysd, points=False, form=pq.FORM_FP64)
    pq.b200_set_stream(ctx64, stream.cuda_stream)
    d_ref = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    fp64_step = lambda: pq.b200_mo_vgl_device(ctx64, P, d_coord.data_ptr(), d_ref.data_ptr())
    for _ in range(3):
        fp64_step()
    pq.b200_synchronize(ctx64)
    n64 = max(3, min(args.steps, 10))
    fp64_ms, _ = _events_time(stream, fp64_step, n64, flush)
    d_ao = torch.empty(P * 5 * A, dtype=torch.float64, device="cuda")
    ao_step = lambda: pq.b200_ao_vgl_device(ctx64, P, d_coord.data_ptr(), d_ao.data_ptr())
    ao_step()
    ao_ms, _ = _events_time(stream, ao_step, n64, flush)
    del d_ao
    pq.b200_synchronize(ctx64)
    fp64_ms = replicas.max_over_ranks(fp64_ms, device="cuda")
    ao_ms = replicas.max_over_ranks(ao_ms, device="cuda")
    hbm, bf16, bf16_sus, peak_src = load_peaks()
    ao_bytes = 5.0 * P * A * 8 + 24.0 * P      # dense FP64 ao_vgl write + coordinates
    fp64_form = {"ms_per_step": fp64_ms, "points_per_s": world * P / (fp64_ms * 1e-3),
                 "ao_kernel": {"kernel": "ao_f64_kernel<5> (AO VGL, FP64)", "ms_per_launch": ao_ms,
                               "algorithmic_bytes_per_launch": ao_bytes,
                               "achieved_gbs": ao_bytes / (ao_ms * 1e-3) / 1e9,
                               "hbm_frac": ao_bytes / (ao_ms * 1e-3) / 1e9 / hbm,
                               "traffic": _scaled_traffic("ao_f64_kernel", "fp64", P)},
                 "mo_gemm_ms": fp64_ms - ao_ms,
                 "mo_gemm_traffic": _scaled_traffic("sparse_dgemm_kernel", "fp64", P),
                 "timing": f"CUDA events, median of {n64}, L2 flushed before each step"}

    # accuracy of the timed form: against the FP64 form on every point, and
    # against the CPU oracle on a fixed sample of the points
    err = None
    if form == pq.FORM_MIXED:
        step()
        fp64_step()
        pq.b200_synchronize(ctx)
        pq.b200_synchronize(ctx64)
        err = {"vs_fp64_gpu_all_points": device_error_report(d_mo.view(P, 5, M), d_ref.view(P, 5, M)),
               "vs_oracle_sample": None}
        if rank == 0:
            sample = np.arange(0, P, 39)
            err["vs_oracle_sample"] = oracle_error_report(sysd, sample, d_mo.view(P, 5, M), d_ref.view(P, 5, M))
    pq.context_destroy(ctx64)
    del d_ref

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
    # the floor of the end-to-end step: one plain copy of the same bytes from
    # the device into the same pinned buffer, and of the coordinates up
    d_src = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    d_crd = torch.empty(h_coord.numel(), dtype=torch.float64, device="cuda")
    copy_times = []
    for i in range(4):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            d_crd.copy_(h_coord, non_blocking=True)
            h_out.copy_(d_src, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            copy_times.append(e0.elapsed_time(e1))
    copy_ms = min(copy_times)
    del d_src, d_crd

    if form == pq.FORM_FP64:
        roofline = {"kernel": "ao_f64_kernel<5> (AO VGL, FP64)", "bound": "hbm",
                    "achieved": fp64_form["ao_kernel"]["achieved_gbs"], "peak": hbm, "unit": "GB/s",
                    "frac": fp64_form["ao_kernel"]["hbm_frac"], "peak_source": peak_src,
                    "traffic": _scaled_traffic("ao_f64_kernel", "fp64", P),
                    "traffic_note": "ncu capture at fewer points (profiles/dram_traffic.txt) scaled by the point count",
                    "ms_per_launch": ao_ms, "algorithmic_bytes_per_launch": ao_bytes,
                    "other_kernel": {"kernel": "f64_plan_kernel + sparse_dgemm_kernel (MO VGL, FP64 mma.sync "
                                               "m8n8k4 over each tile's live AOs)",
                                     "ms_per_launch": ms - ao_ms,
                                     "dense_equivalent_tflops": 2.0 * 5 * P * A * M / ((ms - ao_ms) * 1e-3) / 1e12}}
    else:
        roofline = mixed_roofline(args, P, A, M, ms, ks_eval, ks_total, bf16, peak_src)

    value = world * P / (ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "electron-points/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if form == pq.FORM_FP64 else ("f32/bf16x3" if args.pieces == 3 else "f32/f16x2"),
        "data": "synthetic (seeded generator qmckl_b200/gen.py, no dataset)",
        "config": workload_config(P, A, M, world),
        "form": args.form + (" (unfused)" if args.unfused else ""),
        "e2e": {"value": world * P / (e2e_ms * 1e-3), "unit": "electron-points/s",
                "h2d_bytes_per_step": int(P * 3 * 8), "d2h_bytes_per_step": int(P * 5 * M * 8),
                "ms_per_step": e2e_ms,
                "copy_floor_ms": copy_ms,
                "copy_floor_gbs": (P * 5 * M * 8 + P * 3 * 8) / (copy_ms * 1e-3) / 1e9,
                "fraction_of_copy_floor": copy_ms / e2e_ms,
                "note": "copy floor: the same H2D + D2H bytes as plain pinned copies on the device stream, no compute"},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "roofline": roofline,
        "fp64_form": fp64_form,
        "mixed_over_fp64": fp64_ms / ms if form == pq.FORM_MIXED else None,
    }
    if err is not None:
        line["error"] = err
    pq.context_destroy(ctx)
    del d_mo
    torch.cuda.empty_cache()
    if rank == 0 and not args.no_extras and world == 1:
        line["other_workloads"] = other_workloads(args)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sysd)
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def fused_n_tile(M):
    """MO tile width of the fused kernel's plan with 3 pieces (mo_tc.cu
    tc_plan_fused): tiles of up to 256 MOs when they take fewer tiles than
    tiles of up to 160, or as many with three A stages (up to 176 MOs)."""
    narrow = -(-M // 160)
    nt = -(-M // 256)
    n = -(-(-(-M // nt)) // 16) * 16
    fits3 = 1024 + 3 * (49152 + 4096) + 384 * n + 3072 <= 232448
    if nt < narrow or (nt == narrow and fits3):
        return n
    return -(-(-(-M // narrow)) // 16) * 16


def mixed_roofline(args, P, A, M, ms, ks_eval, ks_total, bf16, peak_src):
    """Roofline of the mixed step's dominant kernel against the bf16 tensor peak.

    The fused kernel evaluates 25 points x 5 components per 128-row MMA tile,
    MOs in N tiles of n_tile columns, 16-AO k-steps (the k-steps that vanish
    over a tile are skipped: the kernel counts the k-steps it issues);
    6 split-BF16 products (3 for float16 x 2) per k-step.  Reported two ways:
    the issued MMA flops and the algorithmic split count (3 x 10 P A M)."""
    flops = 2.0 * 5 * P * A * M
    n_tile = fused_n_tile(M) if args.pieces == 3 else -(-(-(-M // -(-M // 160))) // 16) * 16
    nprod = 6 if args.pieces == 3 else 3
    issued = 2.0 * (ks_eval / args.steps) * 128 * n_tile * 16 * nprod
    kname = ("fused_mo_kernel<3,5> (AO -> split-BF16 tcgen05 MO VGL" if args.pieces == 3 else
             "fused_mo_kernel<2,5> (AO -> split-FP16 tcgen05 MO VGL") + "; step = 3 ordering kernels + tile plan + this)"
    if args.unfused:
        # AO pieces to HBM, then 128-row tiles of the 5P x A pieces matrix x 6 products
        nt = -(-M // 160)
        issued = 2.0 * (-(-5 * P // 128) * 128) * (nt * (-(-(-(-M // nt)) // 16) * 16)) * (-(-A // 64) * 64) * 6
        kname = "ao_tile_kernel<3,5> + tc_gemm_kernel<3,2> (unfused mixed form; whole step)"
    split3 = 3.0 * flops
    achieved = issued / (ms * 1e-3) / 1e12
    traffic, traffic_note = None, "no ncu capture of this kernel in profiles/dram_traffic.txt"
    cap = load_traffic().get(("fused_mo_kernel", "mixed"))
    if cap and cap[0] > 0 and not args.unfused and args.pieces == 3:
        traffic = _scaled_traffic("fused_mo_kernel", "mixed", P)
        scaled = "" if int(cap[0]) == P else " scaled by the point count"
        traffic_note = (f"DRAM read + write bytes of one launch from an ncu capture at {int(cap[0])} points "
                        f"(profiles/dram_traffic.txt){scaled}; the algorithmic bytes are the "
                        f"{40.0 * P * M / 1e9:.3f} GB of mo_vgl written + 24 P bytes of coordinates, of which "
                        f"~59 MB are still dirty in L2 when the kernel ends (written back afterwards, "
                        f"uncounted in the launch)")
    return {"kernel": kname, "bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
            "frac": achieved / bf16, "peak_source": peak_src,
            "achieved_basis": "issued split-BF16 MMA flops per step / step time",
            "split3_count": {"flop_per_step": split3, "tflops": split3 / (ms * 1e-3) / 1e12,
                             "frac": split3 / (ms * 1e-3) / 1e12 / bf16,
                             "note": "3 x 10 P A M: the 3-term split of the dense contraction"},
            "traffic": traffic,
            "traffic_note": traffic_note,
            "executed_tensor_flop_per_launch": issued,
            "dense_equivalent_tflops": flops / (ms * 1e-3) / 1e12,
            "k_steps_issued_fraction": (ks_eval / ks_total) if ks_total else None,
            "output_bytes_per_launch": 40.0 * P * M}


def _torch_error_measures(got, ref):
    """The three error measures per component, on the device (torch tensors [P][5][M])."""
    import torch
    out = {"max_abs_over_max_ref": {}, "row_floored_rel": {}, "elementwise_rel": {}, "avg_bits": {}}
    for c, name in enumerate(COMPONENTS):
        g, r = got[:, c, :], ref[:, c, :]
        d = (g - r).abs()
        ar = r.abs()
        s = ar.max()
        out["max_abs_over_max_ref"][name] = float(d.max() / s)
        den = torch.maximum(ar, 1e-2 * ar.amax(dim=1, keepdim=True))
        den = torch.where(den == 0, torch.ones_like(den), den)
        out["row_floored_rel"][name] = float((d / den).max())
        m = ar > 1e-8 * s
        out["elementwise_rel"][name] = float((d[m] / ar[m]).max()) if bool(m.any()) else 0.0
        out["avg_bits"][name] = float(_torch_bits(g, r).double().mean())
    return out


def _torch_bits(a, b):
    """Bits of agreement of two FP64 tensors: the reference's
    qmckl_test_precision_64 (org/qmckl_numprec.org:384-430), on the device."""
    import torch
    x = a.contiguous().view(torch.int64)
    y = b.contiguous().view(torch.int64)
    same = (x < 0) == (y < 0)
    d = torch.where(same, (x - y).abs(), torch.zeros_like(x))
    e = torch.frexp(d.double())[1]
    bits = 53 - torch.clamp(e, max=53)
    zero = (a == 0) | (b == 0)
    return torch.where(same | zero, bits, torch.zeros_like(bits))


COMPONENTS = ("value", "grad_x", "grad_y", "grad_z", "laplacian")


def device_error_report(got, ref):
    rep = _torch_error_measures(got, ref)
    rep["points"] = int(got.shape[0])
    rep["reference"] = "FP64 form on the GPU"
    return rep


def oracle_error_report(sysd, sample, d_mixed, d_fp64):
    """Mixed and FP64 GPU results on the sampled points against the CPU oracle."""
    import torch
    from oracle import pyoracle as O
    pts = sysd["elec_coord"].reshape(-1, 3)[sample]
    ref = O.mo_vgl(sysd["mo_coef"], O.ao_vgl(O.Basis(sysd), pts, sysd["nucl_coord"]))
    idx = torch.tensor(sample, device=d_mixed.device)
    ref_t = torch.from_numpy(ref).to(d_mixed.device)
    rep = _torch_error_measures(d_mixed.index_select(0, idx), ref_t)
    f64 = d_fp64.index_select(0, idx)
    d = (f64 - ref_t).abs()
    den = torch.maximum(ref_t.abs(), 1e-2 * ref_t.abs().amax(dim=2, keepdim=True))
    den = torch.where(den == 0, torch.ones_like(den), den)
    rep["fp64_form_parity"] = float((d / den).max())
    rep["points"] = int(len(sample))
    rep["reference"] = "CPU oracle (restatement of the reference's HPC path), every 39th point"
    return rep


def other_workloads(args):
    """Configs 2, 3 and 4 at a few steps each (one line per workload)."""
    out = {}
    for name, fn in (("config4_large", case_large), ("config3_adjoint", case_adjoint), ("config2_batched", case_batched)):
        t0 = time.time()
        try:
            out[name] = fn(argparse.Namespace(steps=min(args.steps, 5), warmup=3))
        except Exception as e:   # reported, not fatal: the headline line still prints
            out[name] = {"error": repr(e)}
        out[name]["wall_s"] = time.time() - t0
    return out


if __name__ == "__main__":
    main()
