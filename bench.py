#!/usr/bin/env python
"""Benchmark of the a2afft_b200 pencil-decomposed 3D FFT on B200.

Workload: 512^3 complex64 C2C forward + inverse on a 64-rank virtual grid
(dims [4,4,4], 128^3 bricks), input U[-1,1) real/imag plus 3 pure tones of
amplitude 100 (seed 2) -- the precision-form configuration the headline metric
is quoted on.  One step = one forward + one inverse of the whole cube, in
place.  The 1 GiB buffer is larger than the 126 MB L2, so no flush is needed
between steps.

Printed (rank 0, one JSON line):
  value         ms per forward+inverse of the plain FP32 method, device-resident
                data, CUDA events on the launching stream (max over ranks; with
                N ranks, N independent replicas run and value = max time / N)
  methods       the same timing, per-pass times, roofline and accuracy for each
                method on the same input: plain, split_fp16 and split_bf16 (the
                split-precision tensor-core form), so the metric's comparison
                is in one line
  rel_l2_vs_fp64  per method: relative L2 error of the forward result against
                the oracle's complex128 transform of the same input (the
                reference's own check, np.fft.fftn, in FP64)
  e2e           the plain method through the public API with pinned HOST
                buffers: the H2D copy of the input and the D2H copy of the
                result are inside every timed step
  roofline      the dominant pass kernel: algorithmic bytes (2 x Ng^3 x 8 B per
                launch) / its mean CUDA-event duration, against the measured HBM
                copy bandwidth
  cpu_baseline  the reference's host step sequence (the oracle port's
                HostPipeline) on the full cube, on all host threads

``--impl reference`` times only that host pipeline (rank 0) on the full
workload, every step, and prints its line with "impl": "reference".

``--workload batch`` measures the batched form instead: 96 complex64 cubes with
edges drawn from 32 48 64 96 128 192 (seed 3) plus two 128x256x512 boxes, each
on 4 virtual ranks (dims [2,2,1]), N(0,1) input (seed 3); one step = one
batched forward + inverse, replayed from a CUDA graph in the schedule the
batch's make_plans picks (one persistent launch per direction, one per pass, or
the grouped schedule: each shape's boxes as one grid through the single-grid
pass kernels, shapes on parallel graph branches).  Its CPU baseline runs the
same step sequence on the host (oracle port) once per distinct shape, scaled by
the shape counts.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "512^3 C2C fwd+inv ms & %HBM peak: split-TC vs plain FP32 at L2 err<=1e-6"
NG = 512
RANKS = 64
SEED = 2
FALLBACK_HBM_GBS = 6650.0
CPU_BASELINE_STEPS = 2  # full-size host pipeline pairs timed for cpu_baseline
REF_BUDGET_S = 300.0  # timed seconds the reference arm may spend


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--method", choices=["all", "plain", "split_bf16", "split_fp16"], default="all",
                    help="cube workload: all = plain, split_fp16, split_bf16 where the split form exists")
    ap.add_argument("--ng", type=int, default=NG)
    ap.add_argument("--ranks", type=int, default=RANKS)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg")
    ap.add_argument("--no-vendor", action="store_true", help="skip the cuFFT context leg")
    ap.add_argument("--no-check", action="store_true", help="skip the accuracy check (profiling runs)")
    ap.add_argument("--workload", choices=["cube", "batch"], default="cube")
    ap.add_argument("--layout", choices=["replicas", "fused"], default="replicas",
                    help="N > 1: independent transforms per GPU (default), or one transform whose virtual ranks are "
                         "split over the GPUs and whose passes gather across them (peer loads/stores)")
    ap.add_argument("--batch-cubes", type=int, default=96, help="batch workload: number of drawn cubes")
    ap.add_argument("--batch-big", type=int, default=2, help="batch workload: number of 128x256x512 boxes")
    ap.add_argument("--batch-schedule", choices=["one-launch", "per-pass", "grouped"], default=None,
                    help="batch workload with --no-tune: this schedule instead of the default one-launch "
                         "(profiling runs)")
    ap.add_argument("--no-tune", action="store_true", help="batch workload: default plan, no make_plans timing "
                    "(profiling runs)")
    ap.add_argument("--precision", choices=["c64", "c128"], default="c64", help="cube workload element type")
    ap.add_argument("--seed", type=int, default=None, help="cube workload seed (default 2; 4 for the large sizes)")
    ap.add_argument("--variants", default=None,
                    help="Z,X,Y launch-variant indices instead of timing them all in make_plans (profiling runs)")
    return ap.parse_args()


def workload_name(ng, ranks, dims, precision="c64", seed=SEED, tones=3):
    cname = "complex128" if precision == "c128" else "complex64"
    inp = f"U[-1,1)+{tones} tones x100" if tones else "U[-1,1)"
    return f"{ng}^3 {cname} C2C forward+inverse, {ranks} virtual ranks (dims {dims}), {inp} seed {seed}"


def host_pipeline_ms(ng, ranks, steps, warmup, precision="c64", seed=SEED, tones=3, budget_s=None):
    """The reference's host step sequence (the oracle port's HostPipeline:
    19 passes per direction, every remap a multi-threaded strided copy, 1D
    transforms torch.fft on the host) on the full ng^3 cube, all host
    threads.  Times `steps` forward+inverse pairs after `warmup` untimed ones
    (fewer if `budget_s` of timed work would be exceeded); returns
    (mean ms, steps timed, threads, sample text)."""
    import torch

    import __graft_entry__ as entry

    O = entry.load_oracle()
    d = O.Decomp(ng, ranks)
    hp = O.HostPipeline(d, precision)
    real = torch.float64 if precision == "c128" else torch.float32
    hp.b1.copy_(synth_bricks(torch, ng, d.dims, seed, "cpu", real, tones))
    for _ in range(warmup):
        hp.run(False)
        hp.run(True)
    times = []
    t_start = time.perf_counter()
    for i in range(steps):
        t0 = time.perf_counter()
        hp.run(False)
        hp.run(True)
        times.append((time.perf_counter() - t0) * 1e3)
        if budget_s is not None and time.perf_counter() - t_start > budget_s:
            break
    cname = "complex128" if precision == "c128" else "complex64"
    sample = (f"the full {ng}^3 {cname} cube on {ranks} virtual ranks (dims {d.dims}), {len(times)} timed "
              f"forward+inverse pairs after {warmup} untimed; the reference's 19 passes per direction (alltoall, "
              f"pack/unpack, fast-axis changes, 1D transforms, copy/scale), remaps as multi-threaded strided "
              f"copies, 1D transforms torch.fft (pocketfft) on {hp.threads} threads")
    return statistics.mean(times), len(times), hp.threads, sample


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, torch_device_index):
        self.samples, self.reasons, self.max_mhz = [], 0, None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nv = pynvml
            import torch

            props = torch.cuda.get_device_properties(torch_device_index)
            h = None
            for attr in ("pci_bus_id",):
                bus = getattr(props, attr, None)
                if bus is not None:
                    try:
                        h = pynvml.nvmlDeviceGetHandleByPciBusId(f"{int(props.pci_domain_id):08x}:{int(bus):02x}:"
                                                                 f"{int(props.pci_device_id):02x}.0")
                    except Exception:
                        h = None
            if h is None:
                vis = os.environ.get("CUDA_VISIBLE_DEVICES")
                idx = int(vis.split(",")[torch_device_index]) if vis else torch_device_index
                h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self._h = h
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: clocks reported as unavailable
            self.error = str(e)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                self.reasons |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self._h))
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        names = [n for bit, n in self.REASONS.items() if self.reasons & bit and n != "gpu_idle"]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


def pipelined_e2e(torch, hin, houts, bufs, run, ke, dev):
    """End-to-end steps through the public API with pinned host buffers: each
    step copies its input host -> device, runs `run(buf, stream)` and copies
    the result device -> host.  Two or more device buffers (used in turn) and
    three streams let step i+1's upload overlap step i's download (the link is
    full duplex) and compute; returns ms per step over `ke` steps after two
    untimed ones."""
    s_in, s_run, s_out = (torch.cuda.Stream(device=dev) for _ in range(3))
    freed = [torch.cuda.Event() for _ in bufs]  # the buffer's last download is done
    for f in freed:
        f.record(s_out)

    def step(i):
        k = i % len(bufs)
        s_in.wait_event(freed[k])
        with torch.cuda.stream(s_in):
            bufs[k].copy_(hin, non_blocking=True)
        loaded = torch.cuda.Event()
        loaded.record(s_in)
        s_run.wait_event(loaded)
        run(bufs[k], s_run)
        done = torch.cuda.Event()
        done.record(s_run)
        s_out.wait_event(done)
        with torch.cuda.stream(s_out):
            houts[k].copy_(bufs[k], non_blocking=True)
        freed[k].record(s_out)

    for i in range(2):
        step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    for i in range(ke):
        step(i)
    e1.record(s_out)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / ke


def vendor_fft_ms(torch, buf, ng, steps, warmup):
    """cuFFT -- the library behind the reference's 1D transforms -- as a plain
    single-GPU 3D transform of a cube of the same size through torch.fft
    (fftn then ifftn, natural order, out of place, no virtual-rank bricks):
    context for the pass kernels' speed, not a run of the reference's pipeline.
    Returns ms per forward+inverse on the current stream."""
    cube = buf.view(ng, ng, ng)
    out, back = torch.empty_like(cube), torch.empty_like(cube)
    for _ in range(warmup):
        torch.fft.fftn(cube, out=out)
        torch.fft.ifftn(out, out=back)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        torch.fft.fftn(cube, out=out)
        torch.fft.ifftn(out, out=back)
    e1.record()
    torch.cuda.synchronize()
    del out, back
    return e0.elapsed_time(e1) / steps


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(kernel_key):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as fh:
            for line in fh:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel_key:
                    return float(parts[1])
    except OSError:
        pass
    return None


def synth_bricks(torch, ng, dims, seed, device, real=None, tones=3, kind="uniform"):
    """Seeded synthetic cube in the rank-major brick layout, generated on
    `device`: real and imaginary parts i.i.d. U[-1,1) (kind "uniform") or
    N(0,1) (kind "normal"), plus `tones` pure tones of amplitude 100 at random
    wave vectors."""
    real = real or torch.float32
    gen = torch.Generator(device=device).manual_seed(seed)
    shape = (ng, ng, ng)
    if kind == "normal":
        re = torch.randn(shape, generator=gen, device=device, dtype=real)
        im = torch.randn(shape, generator=gen, device=device, dtype=real)
    else:
        re = torch.rand(shape, generator=gen, device=device, dtype=real) * 2 - 1
        im = torch.rand(shape, generator=gen, device=device, dtype=real) * 2 - 1
    g = torch.complex(re, im)
    del re, im
    ks = torch.randint(0, ng, (tones, 3), generator=gen, device=device)
    idx = torch.arange(ng, device=device, dtype=torch.int64)
    for kx, ky, kz in ks.tolist():
        ph = ((kx * idx)[:, None, None] + (ky * idx)[None, :, None] + (kz * idx)[None, None, :]) % ng
        g += 100.0 * torch.polar(torch.ones((), device=device, dtype=real), ph.to(real) * (2 * math.pi / ng))
        del ph
    d0, d1, d2 = dims
    lx, ly, lz = ng // d0, ng // d1, ng // d2
    b = g.reshape(d0, lx, d1, ly, d2, lz).permute(0, 2, 4, 1, 3, 5).contiguous().reshape(-1)
    del g
    return b


BATCH_METRIC = "batch 96 cubes {32..192}^3 + 2x128x256x512 C2C fwd+inv ms, c64"
BATCH_RANKS = 4
BATCH_SEED = 3


def batch_shapes(pkg, args):
    return pkg.batch_shapes(cubes=args.batch_cubes, seed=BATCH_SEED, boxes=[(128, 256, 512)] * args.batch_big)


def batch_workload(shapes):
    from collections import Counter

    counts = Counter(shapes)
    drawn = ", ".join(f"{s[0]}x{s[1]}x{s[2]}: {c}" for s, c in sorted(counts.items()))
    return (f"{len(shapes)} independent complex64 boxes, C2C forward+inverse, {BATCH_RANKS} virtual ranks each "
            f"(dims [2,2,1]), N(0,1) seed {BATCH_SEED}; drawn: {drawn}")


def cpu_batch_ms(shapes, reps=1):
    """The reference's host step sequence (oracle port) once per distinct
    shape, scaled by how often the shape occurs: cubes through the six
    pencil steps and scipy line transforms, boxes (which the reference's
    pipeline does not take) through the separable 3D transform."""
    from collections import Counter

    import numpy as np

    import __graft_entry__ as entry

    O = entry.load_oracle()
    cores = os.cpu_count() or 1
    lines = O.scipy_lines(cores)
    total = 0.0
    wall = 0.0
    for shp, cnt in sorted(Counter(shapes).items()):
        d = O.Decomp(shp, BATCH_RANKS)
        g = O.make_input("normal", shp, seed=BATCH_SEED, dtype=np.complex64)
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            if shp[0] == shp[1] == shp[2]:
                b = O.global_to_bricks(g, d)
                f = O.forward(b, d, lines, np.complex64)
                O.inverse(f, d, lines, np.complex64)
            else:
                f = O.fft3_global(g, lines=lines)
                O.fft3_global(f, inverse=True, lines=lines)
            best = min(best, time.perf_counter() - t0)
        total += best * cnt
        wall += best * reps
    sample = (f"one forward+inverse per distinct shape ({len(Counter(shapes))} shapes), best of {reps}, "
              f"times the shape counts; cubes through the six pencil steps, boxes through the separable transform; "
              f"1D transforms scipy.fft workers={cores}")
    return total * 1e3, cores, sample, wall


def run_batch_reference(args, rank, world):
    if rank != 0:
        return
    import __graft_entry__ as entry

    shapes = batch_shapes(entry.load_package(), args)
    times = []
    steps = max(1, min(args.steps, 3))
    for i in range(min(args.warmup, 1) + steps):
        ms, cores, sample, _ = cpu_batch_ms(shapes)
        if i >= min(args.warmup, 1):
            times.append(ms)
    value = statistics.mean(times)
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": args.gpus,
        "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": round(value, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": batch_workload(shapes), "boxes": len(shapes), "world_size": BATCH_RANKS,
                   "precision": "c64"},
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch(args, rank, world, local_rank):
    import torch

    import __graft_entry__ as entry

    pkg = entry.load_package()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    shapes = batch_shapes(pkg, args)
    b = pkg.a2aBatch(shapes, BATCH_RANKS, "c64")
    if not args.no_tune:
        scratch, sviews = b.empty(dev)
        scratch.normal_()
        b.make_plans(sviews)  # tile heights per length, schedule, claim, prefetch
        del scratch, sviews
    elif args.batch_schedule:
        b.set_schedule(fused=args.batch_schedule != "per-pass", grouped=args.batch_schedule == "grouped")
    flat, views = b.empty(dev)
    gen = torch.Generator(device=dev).manual_seed(BATCH_SEED)
    flat.copy_(torch.complex(torch.randn(flat.numel(), generator=gen, device=dev),
                             torch.randn(flat.numel(), generator=gen, device=dev)))
    x0 = flat.clone()
    elems = sum(b.elements)
    nbytes = elems * 8
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        b.forward(views, stream=stream)
        b.inverse(views, stream=stream)
    stream.synchronize()
    b.check_device()
    plan_report = b.plan_report()  # after the first call bound the buffers (the grouped tables need them)

    rel_err = rt_err = None
    if (world == 1 or rank == 0) and not args.no_check:
        flat.copy_(x0)
        b.forward(views)
        b64 = pkg.a2aBatch(shapes, BATCH_RANKS, "c128")
        f64, v64 = b64.empty(dev)
        offs = b.offsets()
        for i in range(len(shapes)):
            v64[i].copy_(x0[offs[i]:offs[i] + b.elements[i]])
        b64.forward(v64)
        num = den = 0.0
        for i in range(len(shapes)):
            num += float(torch.linalg.vector_norm(views[i].to(torch.complex128) - v64[i]) ** 2)
            den += float(torch.linalg.vector_norm(v64[i]) ** 2)
        rel_err = math.sqrt(num / den)
        del f64, v64, b64
        b.inverse(views)
        rt_err = float(torch.linalg.vector_norm((flat - x0).to(torch.complex128)) /
                       torch.linalg.vector_norm(x0.to(torch.complex128)))
        torch.cuda.empty_cache()
    flat.copy_(x0)

    evs = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        evs[0].record(stream)
        k = 1
        for _ in range(args.steps):
            b.forward(views, stream=stream)
            evs[k].record(stream)
            b.inverse(views, stream=stream)
            evs[k + 1].record(stream)
            k += 2
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    b.check_device()
    total_ms = evs[0].elapsed_time(evs[-1])
    dirs = [[], []]
    for i in range(2 * args.steps):
        dirs[i % 2].append(evs[i].elapsed_time(evs[i + 1]))
    step_ms = total_ms / args.steps
    if world > 1:
        t = torch.tensor([step_ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_ms = float(t.item())

    e2e = None
    if not args.no_e2e:
        hin = x0.cpu().pin_memory()
        houts = [torch.empty_like(hin).pin_memory() for _ in range(2)]
        ke = max(1, min(args.steps, 10))
        # a second plan bound to the second device buffer (a plan keeps the
        # buffers it was last called with, so each buffer gets its own)
        b2 = pkg.a2aBatch(shapes, BATCH_RANKS, "c64")
        flat2, views2 = b2.empty(dev)
        if not args.no_tune:
            flat2.normal_()
            b2.make_plans(views2)
        plans = {flat.data_ptr(): (b, views), flat2.data_ptr(): (b2, views2)}

        def run(buf, st):
            bb, vv = plans[buf.data_ptr()]
            bb.forward(vv, stream=st)
            bb.inverse(vv, stream=st)

        e2e_ms = pipelined_e2e(torch, hin, houts, [flat, flat2], run, ke, dev)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": round(e2e_ms / world, 3), "unit": "ms", "h2d_bytes_per_step": flat.numel() * 8,
               "d2h_bytes_per_step": flat.numel() * 8, "steps": ke,
               "pipelined": "2 device buffers: step i+1's upload overlaps step i's download"}
        del hin, houts, b2, flat2, views2

    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    launches = b.launches_per_transform
    dir_ms = [statistics.mean(v) for v in dirs]
    dom = max(range(2), key=lambda i: dir_ms[i])
    alg_dir = 3 * 2.0 * nbytes  # every box read and written once per pass, 3 passes
    achieved = alg_dir / (dir_ms[dom] * 1e-3) / 1e9
    plan_line = plan_report.splitlines()[0]
    grouped = "schedule=grouped " in plan_line
    # DRAM bytes per direction from the committed ncu summary of the schedule in use
    traffic = profiled_traffic("batch98_grouped_c64_direction" if grouped else "batch98_c64_direction")
    kernel = (f"single-grid pass kernels over each shape's boxes as one grid ({launches} launches per direction, "
              "shapes on parallel graph branches)" if grouped
              else f"fft_batch_kernel ({launches} launch(es) per direction)")
    value = step_ms / world
    line = {
        "metric": BATCH_METRIC, "value": round(value, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(step_ms, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "a2afft_b200",
        "config": {"workload": batch_workload(shapes), "boxes": len(shapes), "world_size": BATCH_RANKS,
                   "precision": "c64", "elements": elems,
                   "l2": f"inputs {nbytes / 2**30:.2f} GiB > 126 MB L2 (no flush)", "replicas": world},
        "roofline": {"bound": "hbm", "kernel": kernel,
                     "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "algorithmic_bytes": alg_dir},
        "direction_ms": {"forward": round(dir_ms[0], 4), "inverse": round(dir_ms[1], 4)},
        "plan": plan_line,
        "plan_groups": [ln.strip() for ln in plan_report.splitlines() if ln.strip().startswith("group ")],
        "effective_gbs": round(2 * alg_dir / (step_ms * 1e-3) / 1e9, 1),
        "hbm_frac": round(2 * alg_dir / (step_ms * 1e-3) / 1e9 / peak, 4),
        "rel_l2_vs_fp64": rel_err, "roundtrip_rel_l2": rt_err,
        "clocks": clk.summary(),
        "gpu_launches": 2 * launches * args.steps,
        "e2e": e2e,
    }
    if world == 1 and not args.no_cpu:
        ms, cores, sample, _ = cpu_batch_ms(shapes)
        line["cpu_baseline"] = {"value": round(ms, 1), "unit": "ms", "cores": cores, "kind": "port",
                                "sample": sample}
    print(json.dumps(line), flush=True)


def cube_input(args):
    """(seed, tones) of the cube workload: the precision-form input (seed 2,
    3 tones) at 512^3 and below, plain U[-1,1) with seed 4 for the large
    sizes."""
    large = args.ng > 512 or args.precision == "c128"
    seed = args.seed if args.seed is not None else (4 if large else SEED)
    return seed, (0 if large else 3)


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "batch":
        run_batch_reference(args, rank, world)
        return
    ng, prec = args.ng, args.precision
    seed, tones = cube_input(args)
    # the full workload every step; a timed budget keeps an oversized
    # --steps request within a few minutes (the line reports what was timed)
    value, steps, cores, sample = host_pipeline_ms(ng, args.ranks, args.steps, args.warmup, precision=prec,
                                                   seed=seed, tones=tones, budget_s=REF_BUDGET_S)
    import __graft_entry__ as entry

    dims = entry.load_oracle().dims_create(args.ranks, 3)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "ms", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(value, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == "c128" else "f32", "data": "synthetic",
        "config": {"workload": workload_name(ng, args.ranks, dims, prec, seed, tones), "ng": ng,
                   "world_size": args.ranks, "dims": dims, "precision": prec, "method": "host pipeline"},
        "cpu_baseline": {"value": round(value, 3), "unit": "ms", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


TC_LENGTHS = (64, 128, 256, 512, 1024)


def cube_methods(args):
    """Methods timed on the cube workload: all three where the split
    tensor-core form exists (complex64, radix-16 lengths), else plain."""
    if args.method != "all":
        return [args.method]
    if args.precision == "c64" and args.ng in TC_LENGTHS:
        return ["plain", "split_fp16", "split_bf16"]
    return ["plain"]


PASS_NAMES = ["Z_fwd", "X_fwd", "Y_fwd", "Z_inv", "X_inv", "Y_inv"]


def time_method(pkg, torch, dist, method, x, stream, args, local_rank, world):
    """Plans (make_plans timing every launch variant on a scratch buffer, or
    the --variants choice), warms up, then times K forward+inverse steps on
    `x` with an event between every pass launch.  Returns the plan object,
    the step time (max over ranks), the per-pass means and the clocks."""
    dfft = pkg.a2adfft(dist, method=method)
    if args.variants:
        dfft.make_plans()
        for p, v in enumerate(int(t) for t in args.variants.split(",")):
            dfft.select_variant(p, v)
    else:
        scratch = dist.empty(x.device)  # make_plans times the pass variants on it
        dfft.make_plans(scratch)
        del scratch
        torch.cuda.empty_cache()

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            for inv in (0, 1):
                for p in range(3):
                    dfft.execute_pass(x, p, inv, stream)
    torch.cuda.synchronize()

    evs = [torch.cuda.Event(enable_timing=True) for _ in range(6 * args.steps + 1)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            evs[0].record(stream)
            k = 1
            for _ in range(args.steps):
                for inv in (0, 1):
                    for p in range(3):
                        dfft.execute_pass(x, p, inv, stream)
                        evs[k].record(stream)
                        k += 1
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    dfft.check_device()
    per_pass = [[] for _ in range(6)]
    for i in range(6 * args.steps):
        per_pass[i % 6].append(evs[i].elapsed_time(evs[i + 1]))
    step_ms = evs[0].elapsed_time(evs[-1]) / args.steps
    if world > 1:
        t = torch.tensor([step_ms], device=x.device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_ms = float(t.item())
    return dfft, step_ms, [statistics.mean(v) for v in per_pass], clk.summary()


def method_roofline(means, ng, esz, prec, peak, peak_kind, method):
    dom = max(range(6), key=lambda i: means[i])
    alg_bytes = 2.0 * float(ng) ** 3 * esz  # one read + one write of the cube per pass
    achieved = alg_bytes / (means[dom] * 1e-3) / 1e9
    traffic = profiled_traffic(["line", "batch", "batch"][dom % 3] + f"_{ng}_{prec}") if method == "plain" else \
        profiled_traffic(f"tc_{['line', 'batch', 'batch'][dom % 3]}_{ng}_{prec}")
    return {"bound": "hbm", "kernel": PASS_NAMES[dom], "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
            "traffic_source": "profiles/dram_traffic.txt (ncu capture of that kernel)" if traffic else None,
            "algorithmic_bytes": alg_bytes}


def run_ours(args, rank, world, local_rank):
    import torch

    import __graft_entry__ as entry

    pkg = entry.load_package()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ng, ranks = args.ng, args.ranks
    prec = args.precision
    seed, tones = cube_input(args)
    esz = 16 if prec == "c128" else 8
    dist = pkg.a2aDistribution(ranks, ng, 64, precision=prec)
    x = synth_bricks(torch, ng, dist.dims, seed, dev, torch.float64 if prec == "c128" else torch.float32, tones)
    x0 = x.clone()
    stream = torch.cuda.Stream(device=dev)
    nbytes_buf = x.numel() * x.element_size()
    peak, peak_kind = measured_peak()

    methods = cube_methods(args)
    results = {}
    for method in methods:  # the same input, each method timed on its own
        x.copy_(x0)
        results[method] = time_method(pkg, torch, dist, method, x, stream, args, local_rank, world)
    dfft, step_ms, means, clocks = results[methods[0]]

    # e2e through the public API with pinned host buffers (the first method)
    e2e = None
    if not args.no_e2e:
        x.copy_(x0)
        hin = x0.cpu().pin_memory()
        houts = [torch.empty_like(hin).pin_memory() for _ in range(3)]
        ke = max(1, min(args.steps, 10))

        def run(buf, st):
            dfft.forward(buf, st)
            dfft.inverse(buf, st)

        # three device buffers: step i+1's upload never waits for step i-1's
        # download, so both directions of the link stay busy
        e2e_ms = pipelined_e2e(torch, hin, houts, [x, torch.empty_like(x), torch.empty_like(x)], run, ke, dev)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": round(e2e_ms / world, 3), "unit": "ms", "h2d_bytes_per_step": nbytes_buf,
               "d2h_bytes_per_step": nbytes_buf, "steps": ke,
               "pipelined": "3 device buffers: step i+1's upload overlaps step i's compute and download"}
        del hin, houts
        torch.cuda.empty_cache()

    vendor = None
    if world == 1 and not args.no_vendor:
        vendor = {"library": "cuFFT via torch.fft.fftn + ifftn", "ms_per_step": None,
                  "layout": "one natural-order cube, out of place (no virtual-rank bricks)"}
        try:
            vendor["ms_per_step"] = round(vendor_fft_ms(torch, x, ng, min(args.steps, 20), max(args.warmup, 3)), 4)
        except RuntimeError as e:  # e.g. out of memory for the out-of-place buffers
            vendor["error"] = str(e).splitlines()[0]
        torch.cuda.empty_cache()

    if rank != 0:
        return

    # accuracy of every method, outside the timed regions: the forward result
    # against the oracle's complex128 transform of the same input (the
    # reference's own check, np.fft.fftn, in FP64), and the round trip
    acc = {m: {"rel_l2_vs_fp64": None, "roundtrip_rel_l2": None} for m in methods}
    if not args.no_check:
        O = entry.load_oracle()
        d = O.Decomp(ng, ranks)
        h0 = x0.cpu().numpy().reshape(ranks, -1)
        ref = O.global_to_bricks(O.fft3_fp64(O.bricks_to_global(h0, d)), d)
        for m in methods:
            f = results[m][0]
            x.copy_(x0)
            f.forward(x)
            acc[m]["rel_l2_vs_fp64"] = O.rel_l2_chunked(x.cpu().numpy(), ref)
            f.inverse(x)
            acc[m]["roundtrip_rel_l2"] = O.rel_l2_chunked(x.cpu().numpy(), h0)
        del ref, h0

    alg_total = 6 * 2.0 * float(ng) ** 3 * esz
    value = step_ms / world
    per_method = {}
    for m in methods:
        f, ms, mm, ck = results[m]
        per_method[m] = {
            "ms_per_step": round(ms / world, 4),
            "hbm_frac": round(alg_total / (ms * 1e-3) / 1e9 / peak, 4),
            "per_pass_ms": {n: round(v, 4) for n, v in zip(PASS_NAMES, mm)},
            "roofline": method_roofline(mm, ng, esz, prec, peak, peak_kind, m),
            "rel_l2_vs_fp64": acc[m]["rel_l2_vs_fp64"], "roundtrip_rel_l2": acc[m]["roundtrip_rel_l2"],
            "plan": [ln for ln in f.plan_report().splitlines()
                     if ("in use" in ln if m != "plain" else "chosen" in ln)],
            "clocks": ck, "gpu_launches": 6 * args.steps,
        }
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(step_ms, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == "c128" else "f32", "data": "synthetic",
        "impl": "a2afft_b200",
        "config": {"workload": workload_name(ng, ranks, dist.dims, prec, seed, tones), "ng": ng, "world_size": ranks,
                   "dims": dist.dims, "precision": prec, "method": methods[0], "methods": methods,
                   "l2": f"inputs {nbytes_buf / 2**30:.2f} GiB > 126 MB L2 (no flush)",
                   "replicas": world},
        "roofline": per_method[methods[0]]["roofline"],
        "per_pass_ms": per_method[methods[0]]["per_pass_ms"],
        "plan": per_method[methods[0]]["plan"],
        "effective_gbs": round(alg_total / (step_ms * 1e-3) / 1e9, 1),
        "hbm_frac": round(alg_total / (step_ms * 1e-3) / 1e9 / peak, 4),
        "fwd_inv_pairs_per_s": round(1e3 / step_ms * world, 2),
        "gflops": round(2 * 5 * float(ng) ** 3 * math.log2(float(ng) ** 3) / (step_ms * 1e-3) / 1e9, 1),
        "rel_l2_reference": "the oracle's complex128 transform (scipy pocketfft fftn) of the same input",
        "rel_l2_vs_fp64": acc[methods[0]]["rel_l2_vs_fp64"],
        "roundtrip_rel_l2": acc[methods[0]]["roundtrip_rel_l2"],
        "methods": per_method,
        "clocks": clocks,
        "gpu_launches": 6 * args.steps,
        "e2e": e2e,
        "vendor_fft": vendor,
    }
    if world == 1 and not args.no_cpu:
        ms, n, cores, sample = host_pipeline_ms(ng, ranks, CPU_BASELINE_STEPS, 1, precision=prec, seed=seed,
                                                tones=tones, budget_s=30)
        line["cpu_baseline"] = {"value": round(ms, 1), "unit": "ms", "cores": cores, "kind": "port",
                                "sample": sample}
    print(json.dumps(line), flush=True)


def run_fused(args, rank, world, local_rank):
    """One cube transform spread over the N processes (one per GPU): process g
    holds virtual ranks [g P/N, (g+1) P/N); every pass is one fused kernel per
    process over its share of the tiles, reading and writing the other GPUs'
    bricks through peer addresses, with a process-group barrier between
    passes.  Strong scaling: value = ms per forward+inverse of the one cube."""
    import importlib

    import torch
    import torch.distributed as tdist

    import __graft_entry__ as entry

    pkg = entry.load_package()
    dd = importlib.import_module(pkg.__name__ + ".distributed")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world == 1 and not tdist.is_initialized():
        import datetime

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29531")
        tdist.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=120))
    ng, ranks, prec = args.ng, args.ranks, args.precision
    seed, tones = cube_input(args)
    f = dd.FusedDistributedDfft(ranks, ng, prec)
    full = synth_bricks(torch, ng, f.dist.dims, seed, dev, torch.float64 if prec == "c128" else torch.float32, tones)
    mine = full[rank * f.block_elems:(rank + 1) * f.block_elems].clone()
    x0 = mine.clone()
    del full
    torch.cuda.empty_cache()
    f.bind(mine)
    for _ in range(max(args.warmup, 3)):
        f.forward()
        f.inverse()
    rt = float(torch.linalg.vector_norm((mine - x0).to(torch.complex128)) /
               torch.linalg.vector_norm(x0.to(torch.complex128)))
    tdist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record()
        for _ in range(args.steps):
            f.forward()
            f.inverse()
        e1.record()
        torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1) / args.steps
    t = torch.tensor([step_ms], device=dev if tdist.get_backend() == "nccl" else "cpu")
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    step_ms = float(t.item())
    f.release()
    if rank != 0:
        return
    esz = 16 if prec == "c128" else 8
    alg_total = 6 * 2.0 * float(ng) ** 3 * esz
    peak, peak_kind = measured_peak()
    line = {
        "metric": METRIC, "value": round(step_ms, 4), "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(step_ms, 4), "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64" if prec == "c128" else "f32", "data": "synthetic",
        "impl": "a2afft_b200",
        "config": {"workload": workload_name(ng, ranks, f.dist.dims, prec, seed, tones), "ng": ng,
                   "world_size": ranks, "precision": prec, "layout": "fused", "ranks_per_gpu": ranks // world,
                   "l2": "inputs > 126 MB L2 per GPU (no flush)"},
        "roofline": {"bound": "hbm", "kernel": "fft_mb_kernel (all passes)",
                     "achieved": round(alg_total / (step_ms * 1e-3) / 1e9 / world, 1), "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(alg_total / (step_ms * 1e-3) / 1e9 / world / peak, 4), "traffic": None,
                     "algorithmic_bytes": alg_total / world},
        "roundtrip_rel_l2": rt, "clocks": clk.summary(), "gpu_launches": 6 * args.steps, "e2e": None,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, local_rank)
        elif args.layout == "fused":
            run_fused(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
