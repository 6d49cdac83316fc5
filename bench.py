#!/usr/bin/env python
"""bench.py -- throughput of the NeMo simulation step on the B200 backend.

Workload: the reference's random Izhikevich network (src/examples/random.cpp,
synthetic and seeded) at 100,000 neurons x 1000 outgoing synapses (100M
synapses; 80/20 excitatory/inhibitory; excitatory delays uniform 1-44 ms,
inhibitory 1 ms; Gaussian input noise sigma 5/2) with STDP on the excitatory
synapses (20 + 20 ms exponential window, A+ = 0.1, A- = -0.12, tau = 20 ms,
weights in [0, 10]) and applyStdp(1.0) every 100 ms.  The maximum delay is 44
rather than 64 because the reference rejects max delay + postfire window > 64
(src/nemo/StdpFunction.cpp:51-60).

One bench "step" is one STDP period: 100 simulated milliseconds followed by
applyStdp(1.0).  The metric is synaptic events per second (spike arrivals:
the sum of the out-degrees of the neurons that fired, as the reference's
benchmark counts them, src/examples/common.cpp:94-99) and simulated ms per
wall second.

  value    device-resident run through the native run loop (CUDA events)
  e2e      the reference-facing C ABI, nemo_step once per ms with host
           buffers: a one-neuron firing stimulus goes host->device and the
           fired neuron ids come back every step (src/examples/common.cpp
           --fstim), plus nemo_apply_stdp every 100 ms; nemo_step runs
           through the resident step loop (--no-resident: two kernel
           launches per call)
  roofline the step loop's algorithmic bytes per launch / its measured
           average duration (CUDA events around each launch), against the
           measured HBM copy bandwidth; the persistent loop runs one period
           per launch
  --impl reference  the CPU oracle (a restatement of the reference CPU
           backend; the reference itself cannot be built here) on the host

Multi-GPU: independent replicas, one per GPU (the path does not shard);
value = events of all ranks / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NEURONS = 100_000
SYNAPSES = 1000
DMAX = 44
WINDOW_MS = 100
METRIC = "synaptic events/s (100k x 1k Izhikevich, STDP)"
UNIT = "events/s"
BATCH_DMAX = 20  # delays 1-20 ms in the batched configuration

# algorithmic bytes (per neuron-step, per fired neuron, per event, per STDP
# entry) of the step kernel
B_NEURON = 60 + 16   # Izhikevich u,v r/w, a,b,sigma, RNG r/w + history r/w
B_FIRED = 8          # c, d on a spike
B_EVENT = 8          # {target, weight} per delivered synapse
B_STDP = 12          # {source,delay} + accumulator r/w per walked entry
B_APPLY = 20         # per plastic synapse per applyStdp


def config(args) -> dict:
    return {
        "workload": "izhikevich-100k-x1000-stdp",
        "neurons": args.neurons,
        "synapses_per_neuron": SYNAPSES,
        "synapses": args.neurons * SYNAPSES,
        "max_delay_ms": DMAX,
        "stdp": "20+20 ms exponential window, A+=0.1, A-=-0.12, weights [0,10], applyStdp(1.0) every 100 ms",
        "step": f"{WINDOW_MS} simulated ms + applyStdp",
        "generator": "random::construct (src/examples/random.cpp), mt19937 seed 5489",
        "cache": "inputs larger than L2: 0.8 GB forward matrix + 1 GB reverse matrix streamed per period",
        "parallelism": f"replicas x{args.gpus}",
    }


def stdp_conf(mod):
    conf = mod.Configuration()
    dt = np.arange(1, 21, dtype=np.float32)
    pre = (np.float32(0.1) * np.exp(-dt / np.float32(20.0))).astype(np.float32)
    post = (np.float32(-0.12) * np.exp(-dt / np.float32(20.0))).astype(np.float32)
    conf.set_stdp_function(pre, post, -10.0, 10.0)
    return conf


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region: the
    sampler is running (its first row has arrived) before the region starts,
    and only rows that arrive inside the region are summarised."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    INTERVAL_MS = 50

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []  # (arrival time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.INTERVAL_MS)], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 10
            while not self.rows and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.monotonic(), [x.strip() for x in line.split(",")]))

    def __exit__(self, *exc):
        self.t1 = time.monotonic()
        # a region shorter than the sampling interval: wait for the next row
        deadline = self.t1 + 4 * self.INTERVAL_MS / 1e3
        while self.proc and not any(self.t0 <= t for t, _ in self.rows) and time.monotonic() < deadline:
            time.sleep(0.005)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self) -> dict:
        inside = [r for t, r in self.rows if self.t0 <= t <= self.t1]
        extra = {}
        if not inside:
            # the region was shorter than the interval: the first row after it
            after = [(t, r) for t, r in self.rows if t > self.t1]
            if not after:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"], "samples": 0}
            inside = [after[0][1]]
            extra = {"row_after_region_ms": round((after[0][0] - self.t1) * 1e3, 1)}
        sm = [float(r[1]) for r in inside if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in inside:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(inside), "interval_ms": self.INTERVAL_MS, **extra}


def dist_setup(args):
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def _reduce(x: float, world: int, op: str) -> float:
    """All-reduce one number over the ranks (NCCL on the GPUs; gloo on CPU)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return float(t.item())


def dist_max(x: float, world: int) -> float:
    return _reduce(x, world, "MAX")


def dist_sum(x: float, world: int) -> float:
    return _reduce(x, world, "SUM")


def replica_throughput(events: float, run_ms: float, world: int) -> tuple:
    """Whole-job events/s of N independent replicas: all ranks' events over
    the slowest rank's device time.  Returns (events/s, max ms)."""
    ms = dist_max(run_ms, world)
    return dist_sum(events, world) / (ms / 1e3), ms


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_model() -> str:
    """The host CPU's model name (Linux), for the CPU-baseline records."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# what the CPU baseline parallelises: the reference's OpenMP loops (the
# neuron updates); delivery and STDP accumulation are serial loops there
CPU_THREADS_NOTE = "neuron updates on OpenMP threads; delivery and STDP accumulation serial, as in the reference"


def cpu_sample(neurons: int, warm_ms: int, ms: int, stdp_period: int = WINDOW_MS) -> dict:
    """Time the oracle (the reference CPU backend restated, OpenMP on the
    neuron update as in the reference) on the same network."""
    import oracle as O
    t0 = time.perf_counter()
    net = O.example_random(neurons, SYNAPSES, DMAX, True)
    sim = O.Simulation(net, stdp_conf(O))
    build_s = time.perf_counter() - t0
    sim.run(warm_ms, stdp_period, 1.0, max_ids=warm_ms * neurons)
    t0 = time.perf_counter()
    counts, _ = sim.run(ms, stdp_period, 1.0, max_ids=ms * neurons)
    el = time.perf_counter() - t0
    events = float(counts.sum()) * SYNAPSES
    return {"events_per_s": events / el, "sim_ms_per_s": ms / el, "seconds": el, "build_s": build_s,
            "fired": int(counts.sum())}


def run_reference(args, rank, world):
    """--impl reference: the oracle on the host cores, same metric/config."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    # each bench step is a bounded sample of the 100 ms period so that the
    # whole run stays within a few minutes
    per_ms = 0.03 * args.neurons / 100_000  # ~30 ms per simulated ms at 100k on one socket
    budget = 150.0
    window = max(5, min(WINDOW_MS, int(budget / max(1, args.steps + args.warmup) / per_ms)))
    import oracle as O
    t0 = time.perf_counter()
    net = O.example_random(args.neurons, SYNAPSES, DMAX, True)
    sim = O.Simulation(net, stdp_conf(O))
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        sim.run(window, window, 1.0, max_ids=window * args.neurons)
    t0 = time.perf_counter()
    fired = 0
    for _ in range(args.steps):
        counts, _ = sim.run(window, window, 1.0, max_ids=window * args.neurons)
        fired += int(counts.sum())
    el = time.perf_counter() - t0
    value = fired * SYNAPSES / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32+f64+int64", "data": "synthetic",
        "config": config(args),
        "sim_ms_per_s": args.steps * window / el,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} steps of {window} simulated ms (+applyStdp) after "
                                   f"{args.warmup} warm-up steps; network build {build_s:.1f} s untimed",
                         "cpu_model": cpu_model(), "threads": CPU_THREADS_NOTE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def phase_summary(trace) -> dict:
    """Per-phase times of the persistent step loop from its %globaltimer
    trace ([steps, CTAs, 5] ns): each point relative to the step's start
    (the earliest CTA), as the median over the steps (the first and the
    last left out) of the median or the last CTA."""
    t = trace.astype(np.int64)
    if t.shape[0] > 4:
        t = t[1:-1]
    rel = (t - t[:, :, :1].min(axis=1, keepdims=True)) / 1e3

    def over_steps(x):
        return round(float(np.median(x)), 2)
    return {
        "prephase_done_median_cta": over_steps(np.median(rel[:, :, 1], axis=1)),
        "prephase_done_last_cta": over_steps(rel[:, :, 1].max(axis=1)),
        "barrier_seen_median_cta": over_steps(np.median(rel[:, :, 2], axis=1)),
        "update_done_median_cta": over_steps(np.median(rel[:, :, 3], axis=1)),
        "update_done_last_cta": over_steps(rel[:, :, 3].max(axis=1)),
        "step_end_last_cta": over_steps(rel[:, :, 4].max(axis=1)),
        "steps": int(t.shape[0]), "ctas": int(t.shape[1]),
    }


def run_b200(args, rank, world, local):
    import nemosim_b200 as nb

    t0 = time.perf_counter()
    net = nb.example_random(args.neurons, SYNAPSES, DMAX, True)
    gen_s = time.perf_counter() - t0
    conf = stdp_conf(nb)
    conf.set_cuda_backend(local)
    if args.host_construction:
        conf.set_device_construction(False)
    t0 = time.perf_counter()
    sim = nb.Simulation(net, conf)
    build_s = time.perf_counter() - t0
    del net
    if args.no_graphs:
        sim.set_graphs(False)
    if args.no_persistent:
        sim.set_persistent(False)
    W = args.window

    # warm-up, then the launch-shape autotuner (its trial steps start from a
    # snapshot of the state and leave it unchanged)
    sim.run(W * args.warmup, W, 1.0, ids=False)
    tuned_us = sim.autotune(50) if not args.no_autotune else None
    launch = sim.launch()

    # timed: K periods, device-resident, CUDA events inside the run loop
    barrier(world)
    with ClockSampler(local) as clk:
        sim.run(W * args.steps, W, 1.0, ids=False)
    st = sim.run_stats()
    barrier(world)
    value, run_ms = replica_throughput(float(st["events"]), st["run_ms"], world)
    sim_ms_per_s = args.steps * W / (run_ms / 1e3)

    # profiled pass: per-kernel CUDA events for the roofline
    sim.set_profiling(True)
    kp = max(1, min(args.steps, 5))
    sim.run(W * kp, W, 1.0, ids=False)
    sim.set_profiling(False)
    ps = sim.run_stats()
    steps_p = kp * W
    persistent = ps["kernel_launches"]["run"] > 0
    if persistent:
        # one launch of the persistent step loop per STDP period
        nl = ps["kernel_launches"]["run"]
        run_bytes = (args.neurons * B_NEURON * steps_p + ps["fired"] * B_FIRED + ps["events"] * B_EVENT
                     + ps["stdp_entries"] * B_STDP) / nl
        kernels = {"run_kernel": (run_bytes, ps["kernel_ms"]["run"] / nl)}
    else:
        nsteps_p = max(1, ps["kernel_launches"]["step"])
        upd_ms = ps["kernel_ms"]["step"] / nsteps_p
        dlv_ms = ps["kernel_ms"]["stdp"] / max(1, ps["kernel_launches"]["stdp"])
        # algorithmic bytes per launch of each kernel of the step
        upd_bytes = (args.neurons * B_NEURON * nsteps_p + ps["fired"] * B_FIRED) / nsteps_p
        dlv_bytes = (ps["events"] * B_EVENT + ps["stdp_entries"] * B_STDP) / nsteps_p
        kernels = {"update_kernel": (upd_bytes, upd_ms), "deliver_kernel": (dlv_bytes, dlv_ms)}
    dominant = max(kernels, key=lambda k: kernels[k][1])
    alg_bytes, step_ms = kernels[dominant]
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_gbs()
    apply_ms = ps["kernel_ms"]["apply"] / max(1, ps["kernel_launches"]["apply"])
    apply_gbs = ps["plastic_synapses"] * B_APPLY / (apply_ms / 1e3) / 1e9 if apply_ms else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "step_kernel_traffic.json")
    if os.path.exists(tfile):
        with open(tfile) as f:
            tj = json.load(f).get(dominant, {})
        # scale the captured bytes per launch to this run's per-launch work
        if tj.get("alg_bytes_per_launch"):
            traffic = tj["dram_bytes_per_launch"] * alg_bytes / tj["alg_bytes_per_launch"]
    per_kernel = {k: {"alg_bytes_per_launch": v[0], "avg_launch_us": v[1] * 1e3,
                      "achieved_gbs": v[0] / (v[1] / 1e3) / 1e9 if v[1] else None} for k, v in kernels.items()}
    per_kernel["apply_kernel"] = {"avg_launch_us": apply_ms * 1e3, "achieved_gbs": apply_gbs,
                                  "alg_bytes_per_launch": ps["plastic_synapses"] * B_APPLY}
    # where a step's time goes: one traced launch of the persistent loop
    phases = None
    if persistent:
        phases = phase_summary(sim.trace_phases(W))

    # e2e through the C ABI with host buffers, the calls a C program makes:
    # nemo_step once per ms (a one-neuron firing stimulus from host memory,
    # the fired ids returned in host memory) and nemo_apply_stdp once per
    # period, the loop itself in C (nemo_b200_bench_step_loop, the
    # reference's benchmark() loop); then the same calls from a Python loop
    # through ctypes
    import ctypes as C
    L = nb.lib()
    c_step = C.CDLL(nb.library_path()).nemo_step
    c_step.restype = C.c_int
    c_step.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                       C.c_void_p]
    rng = np.random.default_rng(rank)
    ke = max(1, min(args.steps, args.e2e_steps))
    stim = rng.integers(0, args.neurons, size=2 * ke * W).astype(np.uint32)
    resident = persistent and not args.no_resident
    if not resident:
        sim.set_resident_step(0)
    ev0 = sim.step_events()
    fired_c, secs = C.c_uint64(), C.c_double()
    barrier(world)
    nb._check(L.nemo_b200_bench_step_loop(sim._h, stim[: ke * W], 1, ke * W, W, 1.0, C.byref(fired_c),
                                          C.byref(secs)))
    barrier(world)
    e2e_s = dist_max(secs.value, world)
    e2e_events = dist_sum(float(sim.step_events() - ev0), world)
    fired_total = fired_c.value
    # the Python loop over the same C calls
    no_u32, no_f32 = np.zeros(1, np.uint32), np.zeros(1, np.float32)
    fired, nfired = C.POINTER(C.c_uint)(), C.c_size_t()
    h, pf, pn = sim._h, C.addressof(fired), C.addressof(nfired)
    p_stim, p_i, p_v = stim.ctypes.data + 4 * ke * W, no_u32.ctypes.data, no_f32.ctypes.data
    ev1 = sim.step_events()
    t0 = time.perf_counter()
    k = 0
    for _ in range(ke):
        for _ in range(W):
            rc = c_step(h, p_stim + 4 * k, 1, p_i, p_v, 0, pf, pn)
            if rc:
                nb._check(rc)
            k += 1
        nb._check(L.nemo_apply_stdp(sim._h, 1.0))
    py_loop_s = time.perf_counter() - t0
    py_loop_events = float(sim.step_events() - ev1)
    # the same loop through the Python wrapper (fired ids as a list)
    t0 = time.perf_counter()
    for k in range(W):
        sim.step([int(stim[k])])
    sim.apply_stdp(1.0)
    py_step_us = (time.perf_counter() - t0) / W * 1e6
    words = (args.neurons + 31) // 32

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        c = cpu_sample(args.neurons, args.cpu_warm_ms, args.cpu_ms)
        cpu = {"value": c["events_per_s"], "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"{args.cpu_ms} simulated ms (after {args.cpu_warm_ms} warm-up ms) of the same "
                         f"network on the oracle; build {c['build_s']:.0f} s untimed",
               "sim_ms_per_s": c["sim_ms_per_s"], "cpu_model": cpu_model(), "threads": CPU_THREADS_NOTE}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": run_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32+f64+int64", "data": "synthetic",
            "config": config(args),
            "sim_ms_per_s": sim_ms_per_s,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": dominant, "alg_bytes_per_launch": alg_bytes,
                         "avg_launch_us": step_ms * 1e3, "kernels": per_kernel},
            "cpu_baseline": cpu,
            # nemo_step through the resident loop: per ms a 16-byte request
            # and the one-neuron stimulus in its line (8 bytes) in, the fired
            # ids and a 16-byte reply out (two launches: a 4-byte stimulus in
            # and the fired bit-vector out instead)
            "e2e": {"value": e2e_events / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": (8 + 16) * W if resident else (4 + 16) * W,
                    "d2h_bytes_per_step": (round(4 * fired_total / ke) + 16 * W) if resident else 4 * words * W,
                    "api": "nemo_step + nemo_apply_stdp (C ABI), loop in C (nemo_b200_bench_step_loop)",
                    "python_loop_value": py_loop_events / py_loop_s,
                    "step_path": "resident step loop" if resident else "two launches per nemo_step",
                    "sim_ms_per_s": ke * W / e2e_s, "fired_per_ms": fired_total / (ke * W),
                    "python_step_us": py_step_us},
            # per period: the persistent loop (or 100 update + deliver launches,
            # plus the graph's cycle-counter kernel), then applyStdp's kernel
            "gpu_launches": args.steps * ((1 if persistent else 2 * W + (W // 100)) + 1),
            "clocks": clk.summary(),
            # network generation (the random example's own loop, on the host)
            # and the simulation's construction from it, both untimed
            "network_gen_s": gen_s,
            "build_s": build_s,
            "built_on_device": sim.connectivity_digest()[1],
            "phases_us": phases,
            "launch": {"partition": launch[0], "threads": launch[1],
                       "autotuned_us_per_step": tuned_us,
                       "step_loop": "persistent cooperative launch per period" if persistent
                       else "two launches per step" + ("" if args.no_graphs else ", CUDA graphs of 100 steps")},
            "spikes_per_neuron_s": st["fired"] / args.neurons / (args.steps * W / 1e3),
        }
    del sim
    if rank == 0:
        if world == 1 and not args.no_secondary:
            # the batched and differentiable configurations, measured in the
            # same run (their own lines: --workload batch256 / bptt)
            b = run_batch(args, local, emit=False)
            d = run_bptt(args, local, emit=False, reps=5)
            line["secondary"] = {
                "batch256": {k: b[k] for k in ("metric", "value", "unit", "batch_ms", "sequential_ms",
                                               "bitexact_vs_individual_runs", "mismatched_networks",
                                               "batch_events_per_s", "batch_build_s", "launch", "clocks")},
                "bptt": {k: d[k] for k in ("metric", "value", "unit", "adjoint_ms", "state_dtype",
                                           "adjoint_fp32_state_ms", "torch_autograd_ms", "torch_autograd_reps",
                                           "steps", "clocks")},
            }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_batch(args, local, emit=True):
    """The batched configuration: networks of uneven size, each with its own
    generator seed and input-noise sigma, advanced together by one Batch,
    against the same networks run one after another as plain Simulations
    on the same GPU (device time of the runs; construction untimed).  Every
    network's fire stream in the batch is compared with its own run."""
    import nemosim_b200 as nb

    rng = np.random.default_rng(args.batch_seed)
    specs = [dict(n=int(rng.integers(args.batch_min_neurons, args.batch_max_neurons + 1)),
                  f=int(rng.integers(args.batch_min_fanout, args.batch_max_fanout + 1)),
                  seed=1000 + 17 * k, sigma=float(rng.uniform(2.0, 8.0)))
             for k in range(args.batch_networks)]
    conf = nb.Configuration()
    conf.set_cuda_backend(local)
    ms = args.batch_ms

    def make(sp):
        return nb.example_random(sp["n"], sp["f"], BATCH_DMAX, False, seed=sp["seed"],
                                 sigma_exc=sp["sigma"], sigma_inh=sp["sigma"])

    # one throwaway network first, so that no timed run pays one-time setup
    warm = nb.Simulation(make(specs[0]), conf)
    warm.run(ms, ids=False)
    del warm

    t0 = time.perf_counter()
    nets, seq_ms, seq = [], 0.0, []
    for sp in specs:
        net = make(sp)
        sim = nb.Simulation(net, conf)
        c, _, ids = sim.run(ms, max_ids=sp["n"] * ms // 10)  # room for 100 Hz
        seq_ms += sim.run_stats()["run_ms"]
        seq.append((c, ids))
        del sim
        nets.append(net)
    seq_wall = time.perf_counter() - t0

    t0 = time.perf_counter()
    batch = nb.Batch(nets, conf)
    del nets
    build_s = time.perf_counter() - t0
    if args.batch_launch:
        batch.set_launch(*(int(x) for x in args.batch_launch.split(",")))
        tuned_us = None
    else:
        tuned_us = batch.autotune(20)
    launch = batch.launch()
    neurons = sum(sp["n"] for sp in specs)
    with ClockSampler(local) as clk:
        counts, events, ids = batch.run(ms, max_ids=neurons * ms // 10)
    st = batch.run_stats()
    batch_ms = st["run_ms"]
    streams = batch.streams(counts, ids)
    mismatched = sum(1 for (c1, i1), (c2, i2) in zip(streams, seq)
                     if not (np.array_equal(c1, c2) and np.array_equal(i1, i2)))
    # the same batch continued with each step loop in turn (the default
    # above is the persistent loop unless the batch has more than two neurons
    # per resident thread)
    loop_ms = {}
    for persistent in (True, False):
        batch.set_persistent(persistent)
        batch.run(ms, ids=False)
        loop_ms["persistent" if persistent else "two_launch_graphs"] = batch.run_stats()["run_ms"]
    synapses = sum(sp["n"] * sp["f"] for sp in specs)
    # algorithmic bytes of the checked run (no STDP): neuron-steps, the
    # fired neurons' c and d, synaptic events
    alg = neurons * B_NEURON * ms + st["fired"] * B_FIRED + st["events"] * B_EVENT
    peak, peak_kind = measured_peak_gbs()
    achieved = alg / (batch_ms / 1e3) / 1e9
    line = {
        "metric": "batched speedup vs sequential plain runs", "value": seq_ms / batch_ms, "unit": "x",
        "n_gpus": 1, "higher_is_better": True, "dtype": "fp32+f64+int64", "data": "synthetic",
        "config": {"workload": f"batch-{args.batch_networks}-izhikevich", "networks": args.batch_networks,
                   "neurons": [args.batch_min_neurons, args.batch_max_neurons],
                   "fanout": [args.batch_min_fanout, args.batch_max_fanout], "max_delay_ms": BATCH_DMAX,
                   "sigma": [2.0, 8.0], "ms": ms, "total_neurons": neurons, "total_synapses": synapses,
                   "generator": "random::construct (src/examples/random.cpp) per network, own seed and sigma"},
        "batch_ms": batch_ms, "sequential_ms": seq_ms, "sequential_wall_s": seq_wall,
        "continued_runs_ms": loop_ms,
        "batch_events_per_s": st["events"] / (batch_ms / 1e3),
        "bitexact_vs_individual_runs": mismatched == 0, "mismatched_networks": mismatched,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "alg_bytes": alg},
        "launch": {"partition": launch[0], "threads": launch[1], "autotuned_us_per_step": tuned_us},
        "batch_build_s": build_s, "clocks": clk.summary(),
    }
    del batch
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_floor(args, local):
    """The scattered-update floor under the step's delivery: the step at
    100k neurons issues about 660k reductions into 100k 16-byte accumulator
    slots.  The same count at pseudo-random indices, as 64-bit reductions,
    32-bit reductions and 8-byte loads, from 1 to 16 CTAs of 256 threads
    per SM, timed with CUDA events (mean of `--steps` launches)."""
    import nemosim_b200 as nb
    ops, slots = 660_000, NEURONS
    sms = torch_sms(local)
    rows = []
    for kind, name in ((0, "red.add.u64"), (1, "red.add.u32"), (2, "ld.u64")):
        for per_sm in (1, 2, 4, 8, 16):
            us = nb.scatter_probe(ops, slots, kind, per_sm * sms, local, max(1, min(args.steps, 1000)))
            rows.append({"op": name, "ctas": per_sm * sms, "us": us, "gops_per_s": ops / us / 1e3})
    best = max(r["gops_per_s"] for r in rows if r["op"] == "red.add.u64")
    line = {"metric": "scattered 64-bit reductions per second (delivery floor)", "value": best * 1e9,
            "unit": "ops/s", "n_gpus": 1, "higher_is_better": True, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "scatter-floor", "ops": ops, "slots": slots, "slot_bytes": 16},
            "steps": args.steps, "sweep": rows,
            "step_floor_us": ops / (best * 1e3)}
    print(json.dumps(line), flush=True)


def torch_sms(local):
    import torch
    return torch.cuda.get_device_properties(local).multi_processor_count


def run_bptt(args, local, emit=True, reps=None):
    """The differentiable configuration at full size: one gradient step
    (forward + hand-written adjoint) against PyTorch float32 autograd of
    the same unrolled dynamics on the same GPU (the baseline leg)."""
    import torch
    from nemosim_b200.bptt import DifferentiableNetwork
    from oracle import bptt_torch as baseline

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    N, F, T, B, R, CK = 4096, 200, 500, 16, 256, 50
    net = DifferentiableNetwork.random(N, F, max_delay=10, seed=1)
    teacher = DifferentiableNetwork.random(N, F, max_delay=10, seed=101)
    g = torch.Generator(device="cpu").manual_seed(1)
    noise = (5.0 * torch.randn((T, B, N), generator=g)).to(dev)
    Wt, at, bt = teacher.tensors(dev, requires_grad=False)
    target = teacher.model(B, T, R, CK).readout_trains(Wt, at, bt, noise)

    def ours(dtype, reps):
        m = net.model(B, T, R, CK, False, state_dtype=dtype)
        W, a, b = net.tensors(dev)
        for _ in range(args.warmup):
            W.grad = a.grad = b.grad = None
            m.loss(W, a, b, noise, target).backward()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        for _ in range(reps):
            W.grad = a.grad = b.grad = None
            m.loss(W, a, b, noise, target).backward()
        end.record()
        torch.cuda.synchronize()
        return start.elapsed_time(end) / reps

    with ClockSampler(local) as clk:
        nrep = reps if reps is not None else args.steps
        ms32 = ours(torch.float32, nrep)
        ms64 = ours(torch.float64, nrep)
    W, a, b = net.tensors(dev)
    c, d = net.constants(dev)
    st = baseline.Structure(net.source, net.target, net.delay, N, dev)
    torch_reps = 2
    for _ in range(max(1, min(args.warmup, 2))):  # warm-up: allocator, kernels' first launches
        W.grad = a.grad = b.grad = None
        baseline.loss(W, a, b, c, d, noise, target, st, R, False).backward()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for _ in range(torch_reps):
        W.grad = a.grad = b.grad = None
        baseline.loss(W, a, b, c, d, noise, target, st, R, False).backward()
    end.record()
    torch.cuda.synchronize()
    torch_ms = start.elapsed_time(end) / torch_reps
    line = {
        # the default mode: float32 inputs and gradients, float64 neuron state
        "metric": "BPTT gradient step speedup vs PyTorch autograd (same GPU)", "value": torch_ms / ms64,
        "unit": "x", "n_gpus": 1, "higher_is_better": True, "dtype": "fp32 tensors, f64 state", "data": "synthetic",
        "config": {"workload": "bptt-izhikevich-4096x200", "neurons": N, "synapses_per_neuron": F,
                   "ms": T, "substeps": 4 * T, "trials": B, "readout": R, "checkpoint_ms": CK,
                   "delays_ms": [1, 10], "noise_sigma": 5.0},
        "adjoint_ms": ms64, "state_dtype": "float64", "adjoint_fp32_state_ms": ms32, "torch_autograd_ms": torch_ms,
        "speedup_fp32_state": torch_ms / ms32, "steps": nrep, "warmup": args.warmup,
        "torch_autograd_reps": torch_reps,
        "clocks": clk.summary(),
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--neurons", type=int, default=NEURONS)
    ap.add_argument("--window", type=int, default=WINDOW_MS, help=argparse.SUPPRESS)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-resident", action="store_true",
                    help="nemo_step with two kernel launches per call instead of the resident step loop")
    ap.add_argument("--cpu-ms", type=int, default=200)
    ap.add_argument("--cpu-warm-ms", type=int, default=50)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--no-persistent", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="leave out the batched and differentiable configurations of the default line")
    ap.add_argument("--host-construction", action="store_true",
                    help="build the connectivity on the host instead of the device")
    ap.add_argument("--workload", choices=["headline", "batch256", "bptt", "floor"], default="headline",
                    help="headline: the 100k x 1k STDP network (default); batch256: batched networks "
                         "against sequential runs; bptt: differentiable mode against PyTorch autograd; "
                         "floor: the scattered-reduction floor under delivery")
    ap.add_argument("--batch-networks", type=int, default=256)
    ap.add_argument("--batch-min-neurons", type=int, default=1000)
    ap.add_argument("--batch-max-neurons", type=int, default=32000)
    ap.add_argument("--batch-min-fanout", type=int, default=100)
    ap.add_argument("--batch-max-fanout", type=int, default=1000)
    ap.add_argument("--batch-ms", type=int, default=1000)
    ap.add_argument("--batch-seed", type=int, default=0)
    ap.add_argument("--batch-launch", default="",
                    help="neurons per CTA and threads per CTA of the batch's step loop (instead of the autotuner)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        # the CPU reference needs no process group: rank 0 runs, the others exit
        rank = int(os.environ.get("RANK", 0))
        args.gpus = int(os.environ.get("WORLD_SIZE", args.gpus))
        run_reference(args, rank, 1)
        return
    if args.workload != "headline":
        local = int(os.environ.get("LOCAL_RANK", 0))
        if int(os.environ.get("RANK", 0)) != 0:
            return  # these comparisons run on one GPU
        {"batch256": run_batch, "bptt": run_bptt, "floor": run_floor}[args.workload](args, local)
        return
    rank, world, local = dist_setup(args)
    args.gpus = world if world > 1 else args.gpus
    run_b200(args, rank, world, local)


if __name__ == "__main__":
    main()
