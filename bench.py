#!/usr/bin/env python
"""Benchmark of the B200 FFT provider on the batched C2C workload.

Workload (one step): the three batched 1-D C2C plans of the headline configuration,
each executed forward then backward, in place, orthogonal normalization, inputs
uniform[-1, 1) from a seed, all device-resident (every plan's buffer exceeds the
126 MB L2, so no flush is needed between steps):
    complex<float>  N=4096  x batch 16384   (512 MiB)
    complex<float>  N=13440 x batch 4096    (420 MiB)
    complex<double> N=65536 x batch 512     (512 MiB)
value  = GFLOP/s over the step (5 N log2 N per transform), all ranks' work / max rank time.
e2e    = the same metric through the public plan API with pinned HOST buffers: every step
         runs, per plan, one streamed host-buffer call (syclfft_b200.execute_host: the batch
         moves through the device in chunks -- copy in, forward, backward, copy out -- with the
         two copy directions and the kernels overlapped) from a pinned input to a pinned output.
roofline: the dominant kernel's algorithmic bytes (2 * elements * sizeof(complex) per
         launch) / its CUDA-event launch time, against the measured HBM copy bandwidth.
cpu_baseline: the CPU restatement of the reference's portable provider (oracle/) on the
         host cores, on a bounded sample of the same workload.
--impl reference: times that CPU restatement alone (the reference's portable provider
         cannot be built here: no SYCL compiler), rank 0 only.

Multi-GPU: one process per GPU (torchrun); every rank runs the same per-GPU workload on
its own device (independent batches, no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sycl-fft_b200"))
sys.path.insert(0, ROOT)

WORKLOAD = [
    # (label, lengths, batch, double)
    ("c64_4096x16384", [4096], 16384, False),
    ("c64_13440x4096", [13440], 4096, False),
    ("c128_65536x512", [65536], 512, True),
]
METRIC = "batched C2C GFLOP/s (5N log2N), 1D fwd+bwd in-place orthogonal: c64 4096x16384, c64 13440x4096, c128 65536x512"
UNIT = "GFLOP/s"


def flops(lengths, batch):
    n = math.prod(lengths)
    return 5.0 * n * math.log2(n) * batch


def step_flops(workload=WORKLOAD):
    return sum(2 * flops(l, b) for _, l, b, _ in workload)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dram_traffic_record():
    """DRAM bytes per launch from an ncu capture, summarised in profiles/dram_traffic.json."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(values, world, device):
    """Element-wise maximum of per-rank floats: every multi-GPU time is the slowest rank's
    (the caller's process group: NCCL on GPUs, gloo in the CPU tests)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def cpu_baseline(sample_div: int = 2, repeats: int = 10):
    """Oracle (CPU restatement of the portable provider) on 1/sample_div of each batch."""
    import numpy as np
    from oracle import portable
    portable.build()
    threads = portable.max_threads()
    portable.set_threads(threads)
    total_flops, total_t = 0.0, 0.0
    for label, lengths, batch, dbl in WORKLOAD:
        b = max(1, batch // sample_div)
        n = math.prod(lengths)
        rng = np.random.default_rng(n)
        dt = np.complex128 if dbl else np.complex64
        x = (rng.uniform(-1, 1, n * b) + 1j * rng.uniform(-1, 1, n * b)).astype(dt)
        plans = [portable.OraclePlan(lengths, b, d, "orthogonal", dbl) for d in (-1, 1)]
        y = plans[0].execute(x)
        plans[1].execute(y)
        t0 = time.perf_counter()
        for _ in range(repeats):
            y = plans[0].execute(x)
            plans[1].execute(y)
        total_t += time.perf_counter() - t0
        total_flops += repeats * 2 * flops(lengths, b)
    return {
        "value": total_flops / total_t / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
        "sample": f"1/{sample_div} of each batch ({', '.join(f'{l} x {max(1, b // sample_div)}' for _, l, b, _ in WORKLOAD)}),"
                  f" fwd+bwd, {repeats} repeats, {total_t:.1f} s; CPU restatement of src/sycl/sycl.cpp"
                  f" (portable provider), g++ -O3 -fopenmp",
    }


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import portable
    portable.build()
    threads = portable.max_threads()
    portable.set_threads(threads)
    # one step = fwd+bwd of each sub-config on a bounded sample sized so K steps take ~1 minute
    div = 256
    setups = []
    for label, lengths, batch, dbl in WORKLOAD:
        n = math.prod(lengths)
        rng = np.random.default_rng(n)
        dt = np.complex128 if dbl else np.complex64
        setups.append((lengths, batch, dbl, dt, rng))

    def build(div):
        out = []
        for lengths, batch, dbl, dt, rng in setups:
            b = max(1, batch // div)
            n = math.prod(lengths)
            x = (rng.uniform(-1, 1, n * b) + 1j * rng.uniform(-1, 1, n * b)).astype(dt)
            out.append((x, [portable.OraclePlan(lengths, b, d, "orthogonal", dbl) for d in (-1, 1)], lengths, b))
        return out

    def one_step(sets):
        for x, plans, _, _ in sets:
            plans[1].execute(plans[0].execute(x))

    sets = build(div)
    one_step(sets)
    t0 = time.perf_counter()
    one_step(sets)
    t1 = time.perf_counter() - t0
    budget = 60.0
    while div < 16384 and t1 * args.steps > budget:
        div *= 2
        t1 /= 2
    sets = build(div)
    for _ in range(args.warmup):
        one_step(sets)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one_step(sets)
    elapsed = time.perf_counter() - t0
    fl = sum(2 * flops(l, b) for _, _, l, b in sets)
    value = fl * args.steps / elapsed / 1e9
    sample = f"1/{div} of each batch ({', '.join(f'{l} x {b}' for _, _, l, b in sets)}) fwd+bwd per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
        "data": "synthetic", "config": {"workload": "config2_batched_c2c", "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample + "; CPU restatement of the portable provider (src/sycl/sycl.cpp), "
                                            "the SYCL reference itself cannot be built here (no SYCL compiler)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    import syclfft_b200 as sf

    world, rank, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device (the provider has no CPU path)")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.orthogonal,
                           split_precision=args.split)
    plans, bufs, hosts = [], [], []
    workload = [w for w in WORKLOAD if not args.only or w[0] == args.only]
    if args.plan:
        # ad-hoc plans "N[xM[xK]]:batch:c64|c128", comma separated (profiling and tuning runs)
        workload = []
        for spec in args.plan.split(","):
            shape, batch, kind = spec.split(":")
            lengths = [int(v) for v in shape.split("x")]
            workload.append((f"{kind}_{shape}x{batch}", lengths, int(batch), kind == "c128"))
    workload = [(l, s, max(1, b // args.batch_div), d) for l, s, b, d in workload]
    for label, lengths, batch, dbl in workload:
        n = math.prod(lengths)
        g = torch.Generator(device=dev).manual_seed(1000 * rank + n)
        fdt = torch.float64 if dbl else torch.float32
        re = torch.rand(n * batch, device=dev, generator=g, dtype=fdt) * 2 - 1
        im = torch.rand(n * batch, device=dev, generator=g, dtype=fdt) * 2 - 1
        x = torch.complex(re, im)
        del re, im
        kind = "double" if dbl else "float"
        f = sf.plan_many_dft(kind, lengths, batch, sf.direction.forward, opts)
        b = sf.plan_many_dft(kind, lengths, batch, sf.direction.backward, opts)
        plans.append((label, lengths, batch, dbl, f, b))
        bufs.append(x)
    stream = torch.cuda.current_stream(dev)
    launches_per_step = sum(f.launches() + b.launches() for _, _, _, _, f, b in plans)

    def step(s, record=None):
        for i, (label, lengths, batch, dbl, f, b) in enumerate(plans):
            if record is not None:
                record[i][0].record(s)
            f.execute(bufs[i], stream=s)
            if record is not None:
                record[i][1].record(s)
            b.execute(bufs[i], stream=s)
            if record is not None:
                record[i][2].record(s)

    for _ in range(args.warmup):
        step(stream)
    torch.cuda.synchronize()
    # The batched form: one step (every plan's forward and backward execute) captured once into
    # a CUDA graph and replayed, so the timed region has no host launch work between kernels.
    graph = None
    if not args.no_graph:
        cap = torch.cuda.Stream(dev)
        cap.wait_stream(stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cap):
            step(cap)
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            graph.replay()
        torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    start.record(stream)
    for k in range(args.steps):
        if graph is not None:
            graph.replay()
        else:
            step(stream)
    end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    graph = None  # released before any process-group teardown
    barrier()
    # per-execute events on plain launches of the same step (for the per-plan times and the
    # roofline of the dominant kernel)
    n_ev = min(args.steps, 100)
    ev = [[[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in plans] for _ in range(n_ev)]
    for k in range(n_ev):
        step(stream, ev[k])
    torch.cuda.synchronize()
    elapsed_ms = max_over_ranks([start.elapsed_time(end)], world, dev)[0]
    total_flops = step_flops(workload) * args.steps * world
    value = total_flops / (elapsed_ms / 1e3) / 1e9

    # per-plan execute times inside the timed region
    per_plan = {}
    for i, (label, lengths, batch, dbl, f, b) in enumerate(plans):
        fw = [ev[k][i][0].elapsed_time(ev[k][i][1]) for k in range(n_ev)]
        bw = [ev[k][i][1].elapsed_time(ev[k][i][2]) for k in range(n_ev)]
        nbytes = 2 * math.prod(lengths) * batch * (16 if dbl else 8)
        per_plan[label] = {"fwd_ms": statistics.mean(fw), "bwd_ms": statistics.mean(bw),
                           "launches_per_execute": f.launches(),
                           "gbs_alg": nbytes / (statistics.mean(fw + bw) / 1e3) / 1e9}
    # Dominant kernel: the launch with the largest device time per step. A plan with L
    # launches per execute is split evenly over its L kernels (its passes move equal bytes).
    peak, peak_kind = measured_peaks()
    step_ms = elapsed_ms / args.steps
    kernels = []
    for label, lengths, batch, dbl, f, b in plans:
        pp = per_plan[label]
        L = pp["launches_per_execute"]
        launch_ms = (pp["fwd_ms"] + pp["bwd_ms"]) / 2 / L
        nbytes = 2 * math.prod(lengths) * batch * (16 if dbl else 8)  # one launch reads + writes every element
        kinds = [ps["kind"] for ps in f.describe()["passes"]]
        for k in kinds:
            kernels.append({"plan": label, "pass": k, "launch_ms": launch_ms, "bytes": nbytes,
                            "share": 2 * launch_ms / step_ms,
                            "gbs": nbytes / (launch_ms / 1e3) / 1e9})
    dom = max(kernels, key=lambda k: k["launch_ms"])
    traffic = dram_traffic_record()
    tr = None
    if traffic:
        tr = traffic.get("kernels", {}).get(f"{dom['plan']}:{dom['pass']}")
    roofline = {"bound": "hbm", "achieved": round(dom["gbs"], 1), "peak": peak, "unit": "GB/s",
                "frac": round(dom["gbs"] / peak, 4), "peak_source": peak_kind,
                "kernel": f"{dom['plan']} {dom['pass']} pass (largest device-time share, {dom['share']:.2f})",
                "alg_bytes_per_launch": dom["bytes"], "launch_ms": round(dom["launch_ms"], 4),
                "traffic": tr,
                "kernels": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in kk.items()}
                            for kk in kernels]}

    # e2e through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host_in = [torch.empty(x.numel(), dtype=x.dtype, pin_memory=True) for x in bufs]
        host_out = [torch.empty_like(h, pin_memory=True) for h in host_in]
        for h, x in zip(host_in, bufs):
            h.copy_(x)
        h2d = sum(h.numel() * h.element_size() for h in host_in)

        # one stream per plan: a plan's copy-in may start while the previous plan's last chunks
        # are still copied out (the copies share the provider's two copy streams, in order)
        e2e_streams = [stream] * len(plans) if args.e2e_serial else [torch.cuda.Stream(dev) for _ in plans]

        def e2e_step():
            for i, (_, _, _, _, f, b) in enumerate(plans):
                sf.execute_host([f, b], host_in[i], host_out[i], stream=e2e_streams[i])

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier()
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record(stream)
        for s in e2e_streams:
            s.wait_event(s2)
        for _ in range(args.e2e_steps):
            e2e_step()
        for s in e2e_streams:
            stream.wait_stream(s)
        e2.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks([s2.elapsed_time(e2)], world, dev)[0]
        e2e = {"value": step_flops(workload) * args.e2e_steps * world / (e2e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d, "steps": args.e2e_steps,
               "ms_per_step": e2e_ms / args.e2e_steps,
               "api": "syclfft_b200.execute_host([forward plan, backward plan], pinned in, pinned out) per plan"
                      + ("" if args.e2e_serial else ", one CUDA stream per plan"),
               "pcie_gbs_per_direction": round(h2d / (e2e_ms / args.e2e_steps / 1e3) / 1e9, 1)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and not args.only and not args.plan and args.batch_div == 1:
        cpu = cpu_baseline()

    if rank == 0:
        alg_bytes_step = sum(2 * 2 * math.prod(l) * b * (16 if d else 8) for _, l, b, d in workload)
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 (complex64, complex128)",
            "data": "synthetic (seeded uniform[-1,1) complex)",
            "config": {"workload": "config2_batched_c2c" if len(workload) == len(WORKLOAD) and args.batch_div == 1
                       and not args.plan
                       else "subset", "plans": [f"{w[0]} (batch {w[2]})" for w in workload],
                       "placement": "in_place", "normalization": "orthogonal", "directions": "forward+backward",
                       "parallelism": f"replicas x{world} (independent batches per GPU)",
                       "l2": "inputs larger than L2 (no flush)",
                       "execution": "plain launches" if args.no_graph else "CUDA graph of one step, replayed",
                       "split_precision": args.split},
            "gbs_alg": round(alg_bytes_step * world * args.steps / (elapsed_ms / 1e3) / 1e9, 1),
            "per_plan": per_plan,
            "roofline": roofline,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _plane_wave_input(shape, seed, dtype):
    """uniform[-1,1) complex plus a sum of 8 random plane waves (integer wave vectors)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = math.prod(shape)
    x = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).reshape(shape)
    idx = np.indices(shape, dtype=np.float64)
    for _ in range(8):
        k = [int(rng.integers(-s // 2, s // 2)) for s in shape]
        amp, ph = rng.uniform(0.5, 2.0), rng.uniform(0, 2 * np.pi)
        arg = sum(2 * np.pi * k[a] * idx[a] / shape[a] for a in range(len(shape)))
        x = x + amp * np.exp(1j * (arg + ph))
    return x.reshape(-1).astype(dtype)


def _errors(got, ref):
    import numpy as np
    d = got.astype(np.complex128) - ref
    return {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref)),
            "max_rel": float(np.abs(d).max() / np.abs(ref).max())}


def run_config(args):
    """Secondary configurations, one JSON line each (device-resident, CUDA-event timed):
    3: Bluestein primes N in {1009, 4099, 65537}, c64 and c128, batch 256, out of place,
       forward normalization, complex Gaussian inputs; errors against an FP64 direct DFT
       (N=1009) or an FP64 FFT (others), on the first 8 lines.
    4: 3D c64 256^3 in place forward+backward with backward normalization (split-precision
       tensor-core path and pure FP32) and 2D c128 2048^2 out of place forward+backward;
       inputs uniform plus 8 plane waves; errors of the forward result against FP64."""
    import numpy as np
    import torch
    import syclfft_b200 as sf
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    peak, peak_kind = measured_peaks()

    def timed(fn, reps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    cases = []
    reps = max(5, min(args.steps, 200))
    if args.config == 3:
        for n in (1009, 4099, 65537):
            for dbl in (False, True):
                batch = 256
                rng = np.random.default_rng(n + dbl)
                dt = np.complex128 if dbl else np.complex64
                x = (rng.standard_normal(n * batch) + 1j * rng.standard_normal(n * batch)).astype(dt)
                opts = sf.plan_options(placement=sf.placement.out_of_place, normalization=sf.normalization.forward)
                p = sf.plan_many_dft("double" if dbl else "float", [n], batch, sf.direction.forward, opts)
                xi = torch.from_numpy(x).to(dev)
                out = torch.empty_like(xi)
                ms = timed(lambda: p.execute(xi, out), reps)
                got = out[: 8 * n].cpu().numpy().reshape(8, n)
                xs = x[: 8 * n].reshape(8, n).astype(np.complex128)
                if n == 1009:
                    k = np.arange(n)
                    ref = xs @ np.exp(-2j * np.pi * np.outer(k, k) / n) / n
                else:
                    ref = np.fft.fft(xs, axis=1) / n
                nbytes = 2 * n * batch * (16 if dbl else 8)
                cases.append({"case": f"{'c128' if dbl else 'c64'}_N{n}x{batch}", "ms": round(ms, 4),
                              "gflops": round(flops([n], batch) / ms / 1e6, 1),
                              "gbs_alg": round(nbytes / ms / 1e6, 1),
                              "frac_of_peak": round(nbytes / ms / 1e6 / peak, 4),
                              "launches": p.launches(),
                              "passes": [ps["kind"] for ps in p.describe()["passes"]],
                              "oracle": "fp64 direct DFT" if n == 1009 else "fp64 FFT",
                              **_errors(got.reshape(-1), ref.reshape(-1))})
    else:
        shape = [256, 256, 256]
        x = _plane_wave_input(shape, 404, np.complex64)
        ref = np.fft.fftn(x.reshape(shape).astype(np.complex128)).reshape(-1)
        for split in (True, False):
            opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.backward,
                                   split_precision=split)
            f = sf.plan_many_dft("float", shape, 1, sf.direction.forward, opts)
            b = sf.plan_many_dft("float", shape, 1, sf.direction.backward, opts)
            buf = torch.from_numpy(x).to(dev)
            f.execute(buf)
            fwd = buf.cpu().numpy()
            b.execute(buf)
            back = buf.cpu().numpy()
            ms = timed(lambda: (f.execute(buf), b.execute(buf)), reps)
            nbytes = 2 * 2 * x.size * 8
            tc = sum(1 for ps in f.describe()["passes"] if ps.get("tc_id", -1) >= 0)
            cases.append({"case": f"c64_256^3_{'split_bf16' if split else 'fp32'}", "ms_fwd_bwd": round(ms, 4),
                          "gflops": round(2 * flops(shape, 1) / ms / 1e6, 1), "gbs_alg": round(nbytes / ms / 1e6, 1),
                          "launches": f.launches() + b.launches(), "tensor_core_passes": tc,
                          "forward": _errors(fwd, ref), "round_trip": _errors(back, x.astype(np.complex128))})
        shape = [2048, 2048]
        x = _plane_wave_input(shape, 2048, np.complex128)
        ref = np.fft.fftn(x.reshape(shape)).reshape(-1)
        opts = sf.plan_options(placement=sf.placement.out_of_place)
        f = sf.plan_many_dft("double", shape, 1, sf.direction.forward, opts)
        b = sf.plan_many_dft("double", shape, 1, sf.direction.backward, opts)
        xi = torch.from_numpy(x).to(dev)
        y = torch.empty_like(xi)
        z = torch.empty_like(xi)
        f.execute(xi, y)
        fwd = y.cpu().numpy()
        ms = timed(lambda: (f.execute(xi, y), b.execute(y, z)), reps)
        nbytes = 2 * 2 * x.size * 16
        cases.append({"case": "c128_2048^2_out_of_place", "ms_fwd_bwd": round(ms, 4),
                      "gflops": round(2 * flops(shape, 1) / ms / 1e6, 1), "gbs_alg": round(nbytes / ms / 1e6, 1),
                      "launches": f.launches() + b.launches(), "forward": _errors(fwd, ref)})
    total_flops = sum(c["gflops"] * c.get("ms", c.get("ms_fwd_bwd")) for c in cases)
    total_ms = sum(c.get("ms", c.get("ms_fwd_bwd")) for c in cases)
    line = {"metric": f"config {args.config}: GFLOP/s (5N log2N) and accuracy vs FP64", "unit": UNIT,
            "value": round(total_flops / total_ms, 1), "higher_is_better": True, "n_gpus": 1,
            "data": "synthetic (seeded)", "peak_gbs": peak, "peak_source": peak_kind,
            "config": {"workload": "config3_bluestein" if args.config == 3 else "config4_multidim",
                       "l2": "inputs larger than L2 except where a case's buffer is smaller"},
            "cases": cases}
    print(json.dumps(line), flush=True)
    return 0


def run_table(args):
    """Every configuration's rows on one GPU, one JSON line (the per-configuration table):
    P  the provider's plain per-plan execute (estimate planning), device-resident, CUDA events;
    A  autotuned plans (planning_mode::measure) replayed from a captured CUDA graph;
    C  cuFFT through torch.fft as a black box (informational);
    CPU the CPU restatement of the reference's portable provider on a bounded sample, all host
        threads; accuracy of P: relative L2 and max error against FP64 on sampled lines."""
    import numpy as np
    import torch
    import syclfft_b200 as sf
    from oracle import portable
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    portable.build()
    threads = portable.max_threads()
    portable.set_threads(threads)
    peak, _ = measured_peaks()
    N = sf.normalization
    cases = [
        # (row, shape, batch, double, in_place, normalization, directions, input, cpu sample lines)
        ("1: c64 N=1024 B=1 fwd oop", [1024], 1, False, False, "none", (-1,), "uniform", 1),
        ("2a: c64 4096x16384 fwd+bwd ip ortho", [4096], 16384, False, True, "orthogonal", (-1, 1), "uniform", 256),
        ("2b: c64 13440x4096", [13440], 4096, False, True, "orthogonal", (-1, 1), "uniform", 64),
        ("2c: c128 65536x512", [65536], 512, True, True, "orthogonal", (-1, 1), "uniform", 8),
        ("3: c64 N=1009 x256 oop fwd-norm", [1009], 256, False, False, "forward", (-1,), "gaussian", 64),
        ("3: c128 N=1009 x256", [1009], 256, True, False, "forward", (-1,), "gaussian", 64),
        ("3: c64 N=4099 x256", [4099], 256, False, False, "forward", (-1,), "gaussian", 16),
        ("3: c128 N=4099 x256", [4099], 256, True, False, "forward", (-1,), "gaussian", 16),
        ("3: c64 N=65537 x256", [65537], 256, False, False, "forward", (-1,), "gaussian", 2),
        ("3: c128 N=65537 x256", [65537], 256, True, False, "forward", (-1,), "gaussian", 2),
        ("4a: 3D c64 256^3 ip fwd+bwd bwd-norm", [256, 256, 256], 1, False, True, "backward", (-1, 1), "waves", 1),
        ("4b: 2D c128 2048^2 oop fwd+bwd", [2048, 2048], 1, True, False, "none", (-1, 1), "waves", 1),
    ]

    cases = [c for c in cases if c[0].startswith(args.table_rows)]

    def timed(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = []
    for row, shape, batch, dbl, ip, norm, dirs, kind, cpu_lines in cases:
        n = math.prod(shape)
        dt = np.complex128 if dbl else np.complex64
        rng = np.random.default_rng(n + batch)
        if kind == "waves":
            x = _plane_wave_input(shape, n, dt)
        elif kind == "gaussian":
            x = (rng.standard_normal(n * batch) + 1j * rng.standard_normal(n * batch)).astype(dt)
        else:
            x = (rng.uniform(-1, 1, n * batch) + 1j * rng.uniform(-1, 1, n * batch)).astype(dt)
        fl = flops(shape, batch) * len(dirs)
        nbytes = 2 * n * batch * (16 if dbl else 8) * len(dirs)
        scalar = "double" if dbl else "float"
        out = {"row": row}
        for form, planning in (("P", sf.planning_mode.estimate), ("A", sf.planning_mode.measure)):
            opts = sf.plan_options(placement=sf.placement.in_place if ip else sf.placement.out_of_place,
                                   normalization=getattr(N, norm), planning=planning)
            plans = [sf.plan_many_dft(scalar, shape, batch, sf.direction(d), opts) for d in dirs]
            a = torch.from_numpy(x).to(dev)
            b = a if ip else torch.empty_like(a)
            c = a if ip else torch.empty_like(a)
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())

            def step():
                plans[0].execute(a) if ip else plans[0].execute(a, b)
                if len(plans) > 1:
                    plans[1].execute(a) if ip else plans[1].execute(b, c)

            if form == "P":
                if len(dirs) == 1 or not ip:
                    step()
                    got = (a if ip else b).cpu().numpy() if len(dirs) == 1 else b.cpu().numpy()
                else:
                    plans[0].execute(a)
                    got = a.cpu().numpy()
                    a.copy_(torch.from_numpy(x).to(dev))
                lines = min(batch, 8)
                xs = x[: lines * n].astype(np.complex128)
                if shape == [1009]:
                    k = np.arange(n)
                    ref = (xs.reshape(lines, n) @ np.exp(-2j * np.pi * np.outer(k, k) / n)).reshape(-1)
                else:
                    ref = np.fft.fftn(xs.reshape([lines] + shape), axes=tuple(range(1, len(shape) + 1))).reshape(-1)
                scale = {"none": 1.0, "forward": 1.0 / n, "backward": 1.0, "orthogonal": n ** -0.5}[norm]
                ref = ref * scale
                d = got[: lines * n].astype(np.complex128) - ref
                out["rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(ref))
                out["max_rel"] = float(np.abs(d).max() / np.abs(ref).max())
                with torch.cuda.stream(s):
                    ms = timed(step)
            else:
                with torch.cuda.stream(s):
                    step()
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=s):
                    step()
                ms = timed(g.replay)
                out["A_tuning"] = [p.describe().get("tuning") for p in plans][0]
                del g
            out[form] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1), "gbs": round(nbytes / ms / 1e6, 1),
                         "frac": round(nbytes / ms / 1e6 / peak, 4)}
            del plans, a, b, c
        # C: cuFFT via torch (informational)
        xt = torch.from_numpy(x).to(dev).view([batch] + shape)
        tn = {"none": "backward", "forward": "forward", "backward": "backward", "orthogonal": "ortho"}[norm]
        dims = tuple(range(1, len(shape) + 1))

        def cufft():
            y = torch.fft.fftn(xt, dim=dims, norm=tn)
            if len(dirs) > 1:
                torch.fft.ifftn(y, dim=dims, norm=tn)

        ms = timed(cufft)
        out["C_torch_cufft"] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1)}
        del xt
        # CPU restatement on a sample of lines
        cb = max(1, min(batch, cpu_lines))
        xs = x[: cb * n]
        cps = [portable.OraclePlan(shape, cb, d, norm, dbl) for d in dirs]
        t0 = time.perf_counter()
        y = cps[0].execute(xs)
        if len(cps) > 1:
            cps[1].execute(y)
        t = time.perf_counter() - t0
        out["CPU"] = {"gflops": round(flops(shape, cb) * len(dirs) / t / 1e9, 2), "sample_lines": cb, "s": round(t, 3)}
        rows.append(out)
        print(json.dumps(out), file=sys.stderr, flush=True)
    rows.extend(_real_rows(sf, torch, dev, peak, timed, args.table_rows))
    rows.extend(_layout_rows(sf, torch, dev, peak, timed, args.table_rows))
    torch.cuda.empty_cache()
    print(json.dumps({"metric": "per-configuration rows (P, A, C, CPU) and accuracy", "cpu_threads": threads,
                      "peak_gbs": peak, "rows": rows}), flush=True)
    return 0


def _real_rows(sf, torch, dev, peak, timed, prefix=""):
    """Real transforms (R2C then C2R, backward normalization): P = the provider's plans, C = torch.fft
    rfft/irfft (cuFFT). GFLOP/s counts 2.5 N log2 N per real transform; bytes are the algorithmic
    N reals + (N/2 + 1) complex per line and direction. The reference has no real transform, so
    there is no CPU row."""
    import numpy as np
    rows = []
    for row, n, batch, dbl in (("R: r2c+c2r f32 N=8192 x16384 (one pass)", 8192, 16384, False),
                               ("R: r2c+c2r f32 N=16384 x8192", 16384, 8192, False),
                               ("R: r2c+c2r f32 N=26880 x4096", 26880, 4096, False),
                               ("R: r2c+c2r f64 N=131072 x512", 131072, 512, True)):
        if not row.startswith(prefix):
            continue
        rs, cs = (8, 16) if dbl else (4, 8)
        h = n // 2 + 1
        fl = 2 * 2.5 * n * math.log2(n) * batch
        nbytes = 2 * (n * rs + h * cs) * batch
        rng = np.random.default_rng(n)
        x = rng.uniform(-1, 1, (batch, n)).astype(np.float64 if dbl else np.float32)
        scalar = "double" if dbl else "float"
        opts = sf.plan_options(normalization=sf.normalization.backward)
        f = sf.plan_dft_r2c_1d(scalar, n, batch, opts)
        b = sf.plan_dft_c2r_1d(scalar, n, batch, opts)
        a = torch.from_numpy(x).to(dev)
        spec = torch.empty(batch * h, dtype=f.dtype, device=dev)
        back = torch.empty_like(a)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())

        def step():
            f.execute(a, spec, stream=s)
            b.execute(spec, back, stream=s)

        out = {"row": row}
        with torch.cuda.stream(s):
            step()
        torch.cuda.synchronize()
        lines = min(batch, 8)
        ref = np.fft.rfft(x[:lines].astype(np.float64), axis=1)
        got = spec[: lines * h].cpu().numpy().reshape(lines, h)
        d = got - ref
        out["rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(ref))
        out["max_rel"] = float(np.abs(d).max() / np.abs(ref).max())
        out["round_trip_rel_l2"] = float(torch.linalg.vector_norm(back - a) / torch.linalg.vector_norm(a))
        with torch.cuda.stream(s):
            ms = timed(step)
        out["P"] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1), "gbs": round(nbytes / ms / 1e6, 1),
                    "frac": round(nbytes / ms / 1e6 / peak, 4), "launches": f.launches() + b.launches()}

        def cufft():
            y = torch.fft.rfft(a, dim=1, norm="backward")
            torch.fft.irfft(y, n=n, dim=1, norm="backward")

        ms = timed(cufft)
        out["C_torch_cufft"] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1)}
        out["CPU"] = None
        rows.append(out)
        print(json.dumps(out), file=sys.stderr, flush=True)
        del f, b, a, spec, back
    return rows


def _layout_rows(sf, torch, dev, peak, timed, prefix=""):
    """Strided layouts: transforms down the columns of a row-major matrix (input stride = row
    length, distance 1), written as contiguous rows or back into the columns in place. P = the
    provider's strided plan; C = torch.fft.fft along dim 0 (cuFFT's strided plan). Bytes are the
    algorithmic 2 E cs."""
    import numpy as np
    rows = []
    for row, n, cols, ip in (("S: c64 4096-pt columns of 4096x16384 -> rows", 4096, 16384, False),
                             ("S: c64 4096-pt columns of 4096x16384 in place", 4096, 16384, True),
                             ("S: c64 1024-pt columns of 1024x65536 -> rows", 1024, 65536, False)):
        if not row.startswith(prefix):
            continue
        fl = 5 * n * math.log2(n) * cols
        nbytes = 2 * n * cols * 8
        lay = sf.data_layout((cols,), 1, (cols,) if ip else (1,), 1 if ip else n)
        opts = sf.plan_options(placement=sf.placement.in_place if ip else sf.placement.out_of_place)
        p = sf.plan_many_dft("float", [n], cols, sf.direction.forward, opts, layout=lay)
        g = torch.Generator(device=dev)
        g.manual_seed(n)
        a = torch.randn(n * cols, dtype=torch.complex64, device=dev, generator=g)
        keep = a.clone()
        o = None if ip else torch.empty_like(a)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        out = {"row": row}
        with torch.cuda.stream(s):
            p.execute(a) if ip else p.execute(a, o)
        torch.cuda.synchronize()
        res = (a.view(n, cols).t() if ip else o.view(cols, n))[:8].cpu().numpy()
        ref = np.fft.fft(keep.view(n, cols)[:, :8].cpu().numpy().astype(np.complex128), axis=0).T
        d = res - ref
        out["rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(ref))
        out["max_rel"] = float(np.abs(d).max() / np.abs(ref).max())
        with torch.cuda.stream(s):
            ms = timed(lambda: p.execute(a) if ip else p.execute(a, o))
        out["P"] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1), "gbs": round(nbytes / ms / 1e6, 1),
                    "frac": round(nbytes / ms / 1e6 / peak, 4), "launches": p.launches()}
        xm = keep.view(n, cols)
        ms = timed(lambda: torch.fft.fft(xm, dim=0))
        out["C_torch_cufft"] = {"ms": round(ms, 4), "gflops": round(fl / ms / 1e6, 1)}
        out["CPU"] = None
        rows.append(out)
        print(json.dumps(out), file=sys.stderr, flush=True)
        del p, a, keep, o
    return rows


def run_serve_devtime(args):
    """Device time of the serving stream's requests: every request executed back to back on
    one stream (no admission loop), CUDA events around each; one JSON line per plan shape
    (requests, device ms, share, algorithmic GB/s) and a total. The floor of any loop that runs
    these requests on these kernels without overlapping them."""
    import collections
    import ctypes
    import torch
    from syclfft_b200 import _provider, serving
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    torch.cuda.set_device(0)
    reqs = serving.make_request_stream(count=args.requests, rate=args.rate, seed=5)
    biggest = {}
    for r in reqs:
        k = (r.lengths[0], r.double)
        biggest[k] = max(biggest.get(k, 0), r.batch)
    plans, shape = {}, {}
    desc = ctypes.create_string_buffer(1 << 16)
    for (n, dbl), b in biggest.items():
        cfg = _provider.make_config([n], b, -1, dbl, False, 0, False, 0)
        h = lib.syclfft_b200_create_ex(ctypes.byref(cfg), _provider.CREATE_STREAM_SCRATCH, err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        plans[(n, dbl)] = h
        lib.syclfft_b200_describe_plan(h, desc, len(desc))
        passes = json.loads(desc.value.decode())["passes"]
        shape[(n, dbl)] = ("c128 " if dbl else "c64 ") + "+".join(
            q["kind"] + ("(lean)" if q.get("lean") else
                         "(general)" if max(q["fixed_id"], q["blue_id"], q["piped_id"], q["cluster_id"], q["tc_id"]) < 0
                         else "") for q in passes)
    most = {False: 0, True: 0}
    for r in reqs:
        most[r.double] = max(most[r.double], r.elements)
    bufs = {d: [torch.zeros(most[d], dtype=torch.complex128 if d else torch.complex64, device="cuda") for _ in range(2)]
            for d in (False, True)}
    s = torch.cuda.Stream()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(reqs) + 1)]
    for record in (False, True):
        if record:
            evs[0].record(s)
        for i, r in enumerate(reqs):
            x, y = bufs[r.double]
            if lib.syclfft_b200_execute_ex(plans[(r.lengths[0], r.double)], x.data_ptr(), y.data_ptr(), r.batch,
                                           r.direction, r.normalization, s.cuda_stream, err, 1024):
                raise RuntimeError(err.value.decode())
            if record:
                evs[i + 1].record(s)
        torch.cuda.synchronize()
    agg = collections.defaultdict(lambda: [0, 0.0, 0.0])
    for i, r in enumerate(reqs):
        a = agg[shape[(r.lengths[0], r.double)]]
        a[0] += 1
        a[1] += evs[i].elapsed_time(evs[i + 1])
        a[2] += 2 * r.elements * (16 if r.double else 8)
    total = sum(a[1] for a in agg.values())
    for k, (c, ms, b) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        print(json.dumps({"shape": k, "requests": c, "device_ms": round(ms, 1), "share": round(ms / total, 3),
                          "gbs_alg": round(b / ms / 1e6, 1)}))
    print(json.dumps({"metric": "serving stream device time, requests back to back on one stream", "unit": "ms",
                      "value": round(total, 1), "requests": len(reqs), "plans": len(plans)}))
    for h in plans.values():
        _provider.provider(lib).destroy(h)


def run_serve(args):
    """Serving configuration: the mixed request stream through the continuous-batching loop
    and through per-request plain executes; one JSON line with both."""
    # request buffers of every size come and go: expandable segments keep the allocator's
    # pool from fragmenting under the 120 GB admission budget
    os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")
    import torch
    from syclfft_b200 import serving
    torch.cuda.set_device(0)
    reqs = serving.make_request_stream(count=args.requests, rate=args.rate, seed=5)
    out = {"metric": "FFT serving stream: throughput (GFLOP/s, 5N log2N) and p50/p99 latency (arrival to completion)",
           "unit": "GFLOP/s", "higher_is_better": True, "n_gpus": 1, "data": "synthetic (seeded uniform[-1,1))",
           "config": {"workload": "serving_stream", "requests": len(reqs), "arrival_rate_per_s": args.rate,
                      "lengths": "1/3 pow2 2^6..2^20, 1/3 7-smooth, 1/3 primes 257..65537",
                      "batch": "log-uniform 1..512", "precision": "80% c64 / 20% c128",
                      "hbm_budget_gb": args.budget_gb, "plan_workers": args.plan_workers,
                      "warmup": "2000-request stream of the same distribution (seed 11), served, untimed"}}
    # untimed warm-up: a shorter stream of the same distribution (another seed) through the
    # served mode, so the timed modes do not pay the process's first launches of each kernel
    warm = serving.make_request_stream(count=min(2000, args.requests), rate=args.rate, seed=11)
    srv = serving.Server(budget_bytes=args.budget_gb * 1e9, streams=4, plan_workers=args.plan_workers)
    try:
        srv.run(warm, mode="served")
    finally:
        srv.close()
    for mode in ("served", "plain", "plan_per_request"):
        srv = serving.Server(budget_bytes=args.budget_gb * 1e9, streams=4, plan_workers=args.plan_workers)
        try:
            st = srv.run([serving.Request(**{k: getattr(r, k) for k in ("rid", "lengths", "batch", "double",
                                                                         "direction", "normalization", "seed",
                                                                         "arrival")}) for r in reqs], mode=mode)
        finally:
            srv.close()
        out[mode] = {k: (round(v, 4) if isinstance(v, float) else v) for k, v in st.items()}
    out["value"] = out["served"]["throughput_gflops"]
    # the plain per-plan form: a plan per request (the plan API's usage); the resident-plan
    # sequential form beside it
    out["speedup_vs_plain"] = round(out["served"]["throughput_gflops"] /
                                    out["plan_per_request"]["throughput_gflops"], 3)
    out["speedup_vs_plain_resident_plans"] = round(out["served"]["throughput_gflops"] /
                                                   out["plain"]["throughput_gflops"], 3)
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-serial", action="store_true", help="e2e: every plan's streamed call on one stream")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only", default="", help="run one plan of the workload (profiling)")
    ap.add_argument("--batch-div", type=int, default=1, help="divide batch counts (profiling small cases)")
    ap.add_argument("--plan", default="", help="replace the workload: N[xM[xK]]:batch:c64|c128[,...]")
    ap.add_argument("--no-graph", action="store_true",
                    help="time plain launches of the step instead of its captured CUDA graph")
    ap.add_argument("--split", action="store_true",
                    help="complex<float> plans on the split-precision tensor-core path where it applies")
    ap.add_argument("--serve", action="store_true", help="run the serving-stream benchmark instead")
    ap.add_argument("--serve-devtime", action="store_true",
                    help="the serving stream's device time by plan shape (requests back to back, one stream)")
    ap.add_argument("--table", action="store_true", help="every configuration's rows (plain, autotuned, cuFFT via torch, CPU)")
    ap.add_argument("--table-rows", default="", help="with --table: only the rows whose name starts with this")
    ap.add_argument("--config", type=int, choices=[3, 4], default=0,
                    help="run a secondary configuration instead (3: Bluestein primes, 4: 3D/2D)")
    ap.add_argument("--requests", type=int, default=20000)
    ap.add_argument("--rate", type=float, default=50000.0)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--plan-workers", type=int, default=2, help="--serve: threads creating plans ahead of admission")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.serve_devtime:
        return run_serve_devtime(args)
    if args.serve:
        return run_serve(args)
    if args.config:
        return run_config(args)
    if args.table:
        return run_table(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
