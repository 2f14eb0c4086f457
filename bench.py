#!/usr/bin/env python
"""Benchmark driver: prints ONE JSON line (rank 0).

Workloads
  kernels   the kernel-level sweep: circle-FFT evaluate + interpolate of one
            M31 column at log sizes 16..26, Blake2s Merkle commit (leaves +
            all node layers) of 64 M31 columns at log size 20, and a QM31
            fold_line of a 2^22 line evaluation. metric: algorithmic GB/s.
  poseidon  (default once the prover is built) full Poseidon2 proof, 2^18
            instances; metric: proof ms.

Multi-GPU: every rank runs the same workload on its own GPU (independent
replicas, no collective on the data path); value = work of all ranks / the
slowest rank's time ("scaling": "weak").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nitroozk-stwo_b200"))

import numpy as np  # noqa: E402

P = (1 << 31) - 1
L2_BYTES = 126 * (1 << 20)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled DURING the timed region: NVML
    read every 10 ms from a thread (reads only), nvidia-smi as a fallback."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device_index):
        self.dev = device_index
        self.sm, self.smax, self.reasons = [], [], set()
        self.handle = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.source = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            return pynvml.nvmlDeviceGetHandleByUUID(uuid.encode())
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def _sample_nvml(self, pynvml):
        self.sm.append(pynvml.nvmlDeviceGetClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        self.smax.append(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        for name, const in self.REASONS:
            if bits & getattr(pynvml, const, 0):
                self.reasons.add(name)

    def _loop_nvml(self):
        import pynvml
        while True:
            try:
                self._sample_nvml(pynvml)
            except Exception:
                pass
            if self.stop_flag.wait(0.01):
                break

    def start(self):
        try:
            self.handle = self._handle()
            self.source = "nvml"
            self.thread = threading.Thread(target=self._loop_nvml, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.handle = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), "--query-gpu=clocks.sm,clocks.max.sm,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi"
            self.thread = threading.Thread(target=self._read_smi, daemon=True)
            self.thread.start()
        except Exception:
            self.source = None

    def _read_smi(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            try:
                self.sm.append(float(parts[0]))
                self.smax.append(float(parts[1]))
            except (ValueError, IndexError):
                continue
            for (name, _), v in zip(self.REASONS, parts[2:6]):
                if v.lower() == "active":
                    self.reasons.add(name)

    def stop(self):
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        if self.source == "nvml":
            self.stop_flag.set()
            self.thread.join(timeout=2)
        else:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                "sm_max_mhz": max(self.smax) if self.smax else None,
                "reasons": sorted(self.reasons), "samples": len(self.sm), "source": self.source}


# ------------------------------------------------------------ distributed
def dist_setup(args, backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------ kernel sweep
FFT_LOGS = list(range(16, 27))
MERKLE_LOG, MERKLE_COLS = 20, 64
FOLD_LOG = 22


def sweep_bytes():
    fft = {n: 16 * (1 << n) for n in FFT_LOGS}            # evaluate 8*2^n + interpolate 8*2^n
    merkle_leaf = (4 * MERKLE_COLS + 32) * (1 << MERKLE_LOG)
    merkle_nodes = sum(96 * (1 << L) for L in range(MERKLE_LOG))
    fold = 24 * (1 << FOLD_LOG)
    return fft, merkle_leaf, merkle_nodes, fold


class KernelSweep:
    def __init__(self, seed):
        import torch
        from gpustark.backend import GpuBackend, to_device, Context
        self.torch = torch
        self.B = GpuBackend
        self.stream = torch.cuda.current_stream()
        self.ctx = Context(self.stream)
        rng = np.random.default_rng(seed)
        self.tw = self.B.precompute_twiddles(max(FFT_LOGS), ctx=self.ctx)
        self.tw_fold = self.B.precompute_twiddles(FOLD_LOG + 1, ctx=self.ctx)
        self.host_fft = {n: rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32) for n in FFT_LOGS}
        self.fft_in = {n: to_device(self.host_fft[n]) for n in FFT_LOGS}
        self.fft_buf = {n: torch.empty(1 << n, dtype=torch.int32, device="cuda") for n in FFT_LOGS}
        self.host_cols = [rng.integers(0, P, 1 << MERKLE_LOG, dtype=np.int64).astype(np.uint32) for _ in range(MERKLE_COLS)]
        self.cols = [to_device(c) for c in self.host_cols]
        self.layers = [torch.empty((1 << L) * 8, dtype=torch.int32, device="cuda") for L in range(MERKLE_LOG + 1)]
        self.host_fold = rng.integers(0, P, (1 << FOLD_LOG, 4), dtype=np.int64).astype(np.uint32)
        self.fold_in = [to_device(self.host_fold[:, i].copy()) for i in range(4)]
        self.alpha = rng.integers(0, P, 4).tolist()
        self.flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
        self.groups = ["fft%d" % n for n in FFT_LOGS] + ["merkle_leaf", "merkle_nodes", "fold_line"]
        self.times = {g: [] for g in self.groups}

    def flush_l2(self):
        self.flush.zero_()

    def step(self, record=True):
        torch = self.torch
        ev = {}

        def mark(name):
            e = torch.cuda.Event(enable_timing=True)
            e.record(self.stream)
            ev[name] = e

        for n in FFT_LOGS:
            mark("fft%d_s" % n)
            self.B.evaluate_polynomials([self.fft_in[n]], n, self.tw, out=[self.fft_buf[n]], ctx=self.ctx)
            self.B.interpolate_columns([self.fft_buf[n]], n, self.tw, ctx=self.ctx)
            mark("fft%d_e" % n)
        mark("merkle_leaf_s")
        self.B.commit_on_layer(MERKLE_LOG, None, self.cols, ctx=self.ctx, out=self.layers[MERKLE_LOG])
        mark("merkle_leaf_e")
        mark("merkle_nodes_s")
        self.B.commit_node_layers(self.layers, ctx=self.ctx)
        mark("merkle_nodes_e")
        mark("fold_line_s")
        self.B.fold_line(self.fold_in, FOLD_LOG, self.alpha, self.tw_fold, ctx=self.ctx)
        mark("fold_line_e")
        if record:
            self.stream.synchronize()
            for g in self.groups:
                self.times[g].append(ev[g + "_s"].elapsed_time(ev[g + "_e"]))
        return ev

    def e2e_step(self, pinned):
        """The same work through the C ABI with host buffers: inputs copied from
        pinned host memory, results (FFT outputs, root, fold) copied back."""
        torch = self.torch
        h2d = d2h = 0
        for n in FFT_LOGS:
            self.fft_in[n].copy_(pinned["fft%d" % n], non_blocking=True)
            h2d += 4 << n
        for i, c in enumerate(self.cols):
            c.copy_(pinned["col%d" % i], non_blocking=True)
            h2d += 4 << MERKLE_LOG
        for i in range(4):
            self.fold_in[i].copy_(pinned["fold%d" % i], non_blocking=True)
            h2d += 4 << FOLD_LOG
        self.step(record=False)
        for n in FFT_LOGS:
            pinned["out%d" % n].copy_(self.fft_buf[n], non_blocking=True)
            d2h += 4 << n
        pinned["root"].copy_(self.layers[0], non_blocking=True)
        d2h += 32
        return h2d, d2h


def cpu_sweep_sample(threads):
    """Oracle (CPU restatement) on a bounded sample of the sweep: FFT log 20,
    Merkle 64 x 2^16, fold 2^20. Returns (GB/s, seconds, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.set_threads(threads)
    rng = np.random.default_rng(5)
    n = 20
    c = rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32)
    cols = [rng.integers(0, P, 1 << 16, dtype=np.int64).astype(np.uint32) for _ in range(64)]
    ev = rng.integers(0, P, (1 << 20, 4), dtype=np.int64).astype(np.uint32)
    alpha = [1, 2, 3, 4]
    t0 = time.perf_counter()
    reps = 0
    total = 0
    while True:
        e = O.evaluate(c, n, root_log=n)
        O.interpolate(e, n, root_log=n)
        total += 16 * (1 << n)
        O.merkle_root(cols)
        total += (4 * 64 + 32) * (1 << 16) + 96 * (1 << 16)
        O.fold_line(ev, 20, alpha)
        total += 24 * (1 << 20)
        reps += 1
        if time.perf_counter() - t0 > 10 or reps >= 20:
            break
    dt = time.perf_counter() - t0
    return total / dt / 1e9, dt, "oracle: FFT 2^20 eval+interp, Merkle 64x2^16, fold_line 2^20; %d reps" % reps


def fft_autotune(args, hi):
    """Installs the FFT pass splits the library's autotuner picks for log
    sizes 8..hi and LDE extensions 0..2 (set-up, outside every timed region);
    returns the picks that differ from the default 13/4 as
    {"log+extension": "tile_log/coalesce_bits"}."""
    if args.fft_autotune == "off":
        return "off"
    from gpustark.backend import GpuBackend
    picks = GpuBackend.fft_autotune(8, min(hi, 27), 2)
    return {"%d+%d" % k: "%d/%d" % v for k, v in picks.items() if v != (13, 4)}


def run_kernels(args, world, rank, local):
    import torch
    from gpustark import lib as gslib
    torch.cuda.set_device(local)
    tuning = fft_autotune(args, max(FFT_LOGS))
    hbm_peak, peak_kind = load_peaks()
    sw = KernelSweep(seed=1234 + rank)
    fft_b, leaf_b, node_b, fold_b = sweep_bytes()
    bytes_per_step = sum(fft_b.values()) + leaf_b + node_b + fold_b
    for _ in range(args.warmup):
        sw.step(record=False)
        sw.flush_l2()
    torch.cuda.synchronize()
    for g in sw.groups:
        sw.times[g].clear()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = gslib().gs_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = []
    for _ in range(args.steps):
        sw.flush_l2()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(sw.stream)
        sw.step(record=False)
        ev1.record(sw.stream)
        sw.stream.synchronize()
        step_ms.append(ev0.elapsed_time(ev1))
    torch.cuda.synchronize()
    barrier(world)
    launches = gslib().gs_launch_count() - l0
    clk = clocks.stop()
    # per-group timing pass (separate, with events between groups)
    for _ in range(max(2, min(args.steps, 5))):
        sw.flush_l2()
        sw.step(record=True)
    total_ms = max_over_ranks(sum(step_ms), world, "cuda")
    ms_per_step = total_ms / args.steps
    value = world * bytes_per_step * args.steps / (total_ms / 1e3) / 1e9
    # dominant kernel (op) and its roofline
    avg = {g: statistics.mean(sw.times[g]) for g in sw.groups}
    dom = max(avg, key=avg.get)
    alg = {**{"fft%d" % n: fft_b[n] for n in FFT_LOGS}, "merkle_leaf": leaf_b, "merkle_nodes": node_b, "fold_line": fold_b}
    achieved = alg[dom] / (avg[dom] / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(dom)
        except Exception:
            traffic = None
    # end-to-end through the C ABI with host buffers
    pinned = {}
    for n in FFT_LOGS:
        pinned["fft%d" % n] = torch.from_numpy(sw.host_fft[n].view(np.int32)).pin_memory()
        pinned["out%d" % n] = torch.empty(1 << n, dtype=torch.int32).pin_memory()
    for i, c in enumerate(sw.host_cols):
        pinned["col%d" % i] = torch.from_numpy(c.view(np.int32)).pin_memory()
    for i in range(4):
        pinned["fold%d" % i] = torch.from_numpy(sw.host_fold[:, i].copy().view(np.int32)).pin_memory()
    pinned["root"] = torch.empty(8, dtype=torch.int32).pin_memory()
    e2e_steps = max(1, args.steps)
    sw.e2e_step(pinned)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(sw.stream)
    for _ in range(e2e_steps):
        h2d, d2h = sw.e2e_step(pinned)
    e1.record(sw.stream)
    sw.stream.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    e2e_value = world * bytes_per_step * e2e_steps / (e2e_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        gbs, secs, desc = cpu_sweep_sample(threads)
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": desc,
               "seconds": round(secs, 2)}
    out = {
        "metric": "FFT/Merkle HBM GB/s (kernel sweep: circle FFT 2^16..2^26, Merkle 64x2^20, fold 2^22)",
        "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (M31)", "data": "synthetic: seeded uniform M31",
        "config": {"workload": "kernel sweep: circle-FFT evaluate+interpolate log 16..26, "
                               "Blake2s Merkle commit 64 cols x 2^20, QM31 fold_line 2^22",
                   "l2": "flushed between timed steps (write of 2x L2)",
                   "parallelism": "replicas x%d" % world, "fft_tuning": tuning},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                     "traffic": traffic, "algorithmic_bytes": alg[dom], "avg_ms": round(avg[dom], 4)},
        "per_op_ms": {g: round(v, 4) for g, v in avg.items()},
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if cpu:
        out["cpu_baseline"] = cpu
    return out


# ------------------------------------------------------------ full proofs
PROOF_SIZES = {"poseidon": 18, "wide_fibonacci": 16}


def proof_metric(workload, channel="blake2s"):
    suffix = "" if channel == "blake2s" else ", Poseidon252 channel"
    if workload == "poseidon":
        return "Poseidon2 2^18 proof ms" + suffix
    return "Wide-Fibonacci 2^16x100 proof ms" + suffix


def proof_config(workload, log_n, channel="blake2s"):
    base = {"pcs": "pow_bits=10, FriConfig(log_last_layer=0, log_blowup=1, n_queries=70, fold_step=1)",
            "channel": "Blake2s" if channel == "blake2s" else "Poseidon252 (Poseidon252MerkleChannel)",
            "inputs": "seeded uniform M31 states (mode 1)",
            "l2": "each proof streams >1 GB through HBM (inputs larger than L2)"}
    if workload == "poseidon":
        base.update({"workload": "Poseidon2 AIR full proof, 2^%d instances (one per row), width 16, 8 full + 14 "
                                 "partial rounds, logup interaction, composition split 4" % log_n})
    else:
        base.update({"workload": "Wide-Fibonacci AIR full proof, 2^%d rows x 100 columns" % log_n})
    return base


def cpu_proof_sample(workload, threads, log_target, channel="blake2s"):
    """Oracle (C++ restatement of the reference's CPU prover, all host
    threads): one proof of the full-size workload (about 2 s for Poseidon2
    2^18 on 16 threads). Returns (ms, desc)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.set_threads(threads)
    air = "poseidon" if workload == "poseidon" else "wide_fibonacci"
    t0 = time.perf_counter()
    O.prove(air, log_target, n_cols=100, seed=0, input_mode=1, merkle_channel=channel)
    dt = time.perf_counter() - t0
    return 1e3 * dt, "oracle %s proof at 2^%d (%s channel), full size (%.2f s)" % (air, log_target, channel, dt)


def cpu_mix_sample(jobs, threads, budget_s=20.0):
    """Oracle proofs of the job mix, in order, one at a time on all host
    threads, until the budget is spent. Returns (proofs/s, desc)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as O
    O.set_threads(threads)
    t0 = time.perf_counter()
    done = 0
    for a, n, c, sd in jobs:
        O.prove("poseidon" if a == 1 else "wide_fibonacci", n, n_cols=c or 100, seed=sd, input_mode=1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return done / dt, "oracle, first %d of %d jobs of the mix in order (%.1f s)" % (done, len(jobs), dt)


def run_proof(args, world, rank, local):
    import torch
    from gpustark import lib as gslib
    from gpustark import prove as G
    from gpustark.backend import Context
    torch.cuda.set_device(local)
    wl = args.workload
    log_n = args.log_n or PROOF_SIZES[wl]
    ctx = Context(torch.cuda.current_stream())
    stream = torch.cuda.current_stream()
    tuning = fft_autotune(args, 22)

    mc = args.merkle_channel

    def one(mode=G.INPUT_SEEDED, host=None):
        if wl == "poseidon":
            return G.prove_poseidon(log_n, seed=rank, input_mode=mode, host_inputs=host, ctx=ctx, merkle_channel=mc)
        return G.prove_wide_fibonacci(log_n, 100, seed=rank, input_mode=mode, host_inputs=host, ctx=ctx,
                                      merkle_channel=mc)

    for _ in range(args.warmup):
        proof = one()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = gslib().gs_launch_count()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    lat = []
    for _ in range(args.steps):
        t = time.perf_counter()
        proof = one()
        lat.append(1e3 * (time.perf_counter() - t))
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    launches = (gslib().gs_launch_count() - l0) // max(args.steps, 1)
    clk = clocks.stop()
    total_ms = max_over_ranks(ev0.elapsed_time(ev1), world, "cuda")
    ms_per_step = total_ms / args.steps
    value = total_ms / (args.steps * world)     # whole-job ms per proof
    # end to end through the C ABI with host inputs: H2D of the input columns
    # and D2H of the proof bytes inside the timed region
    n = 1 << log_n
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    rng = np.random.default_rng(rank)
    host_cols = 16 if wl == "poseidon" else 2
    host = rng.integers(0, P, (host_cols, n), dtype=np.int64).astype(np.uint32)
    host_t = torch.from_numpy(host.view(np.int32)).pin_memory()
    host_np = host_t.numpy().view(np.uint32)
    one(G.INPUT_HOST, host_np)
    torch.cuda.synchronize()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, args.steps)
    e0.record(stream)
    for _ in range(e2e_steps):
        p2 = one(G.INPUT_HOST, host_np)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda") / (e2e_steps * world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        ms, desc = cpu_proof_sample(wl, threads, log_n, mc)
        cpu = {"value": round(ms, 1), "unit": "ms", "cores": threads, "kind": "port", "sample": desc}
    out = {
        "metric": proof_metric(wl, mc) if log_n == PROOF_SIZES[wl] else proof_metric(wl, mc).replace(
            str(PROOF_SIZES[wl]), str(log_n)),
        "value": round(value, 3), "unit": "ms", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms_per_step, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (M31/QM31 integer arithmetic)", "data": "synthetic: seeded uniform M31",
        "config": dict(proof_config(wl, log_n, mc), parallelism="independent proofs x%d" % world,
                       fft_tuning=tuning),
        "proofs_per_s": round(1e3 / value, 2), "proof_bytes": len(proof),
        "latency_ms": {"p50": round(statistics.median(lat), 3), "max": round(max(lat), 3)},
        "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": int(host.nbytes),
                "d2h_bytes_per_step": len(p2)},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if cpu:
        out["cpu_baseline"] = cpu
    rl = proof_roofline(args, log_n, wl, ctx, clk) if mc == "blake2s" else None
    if rl:
        out["roofline"] = rl
    return out


def int_roof(counts, ms, clk):
    """The integer-instruction ceiling of a kernel whose instruction counts ncu
    measured: each SM issues at most one warp instruction per cycle on each of
    its 4 schedulers and two per cycle on the integer ALU pipe, so the launch
    cannot end before max(inst / 4, alu / 2) / n_SM cycles. Taken at the SM
    clock sampled during the timed region; frac = that time / measured time."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965
    issue = counts["warp_inst"] / (4.0 * sms)
    alu = counts["alu_warp_inst"] / (2.0 * sms)
    roof_ms = max(issue, alu) / (mhz * 1e3)
    return {"bound": "issue" if issue >= alu else "int_alu", "roof_ms": round(roof_ms, 4),
            "frac": round(roof_ms / ms, 4), "sm_mhz": mhz, "warp_inst": counts["warp_inst"],
            "alu_warp_inst": counts["alu_warp_inst"], "n_sm": sms}


def proof_roofline(args, log_n, wl, ctx, clk=None):
    """Roofline of the proof's dominant kernel, timed live on the proof's shape:
    the low-degree extension of the committed trace (evaluate_polynomials,
    CanonicCoset(log_n) coefficients -> 2^(log_n + 2) for Poseidon's constraint
    domain, 2^(log_n + 1) for Wide-Fibonacci). Beside the HBM line it reports
    the integer-issue ceiling (int_roof), the bound the kernel actually meets."""
    import torch
    from gpustark.backend import GpuBackend as B
    hbm_peak, peak_kind = load_peaks()
    cols = 162 if wl == "poseidon" else 100
    ext = 2 if wl == "poseidon" else 1
    target = log_n + ext
    tw = B.precompute_twiddles(target - 1, ctx=ctx)
    src = torch.randint(0, P, (cols, 1 << log_n), dtype=torch.int32, device="cuda")
    dst = torch.empty((cols, 1 << target), dtype=torch.int32, device="cuda")
    srcs = [src[i] for i in range(cols)]
    dsts = [dst[i] for i in range(cols)]
    for _ in range(3):
        B.evaluate_polynomials(srcs, target, tw, out=dsts, ctx=ctx)
    st = torch.cuda.current_stream()
    times = []
    for _ in range(5):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        B.evaluate_polynomials(srcs, target, tw, out=dsts, ctx=ctx)
        b.record(st)
        b.synchronize()
        times.append(a.elapsed_time(b))
    ms = statistics.mean(times)
    alg = 4 * cols * ((1 << log_n) + (1 << target))   # LDE n -> n+b: 4(2^n + 2^(n+b)) bytes per column
    achieved = alg / (ms / 1e3) / 1e9
    traffic = inst = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        try:
            recs = json.load(open(tpath))
            traffic = recs.get("lde_%s_%d" % (wl, log_n))
            inst = recs.get("inst_lde_%s_%d" % (wl, log_n))
        except Exception:
            traffic = inst = None
    out = {"kernel": "fft_tile_kernel (LDE %d cols 2^%d -> 2^%d, 2 launches)" % (cols, log_n, target), "bound": "hbm",
           "achieved": round(achieved, 1), "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
           "frac": round(achieved / hbm_peak, 4), "traffic": traffic, "algorithmic_bytes": alg,
           "avg_ms": round(ms, 4)}
    if inst:
        out["int_roof"] = int_roof(inst, ms, clk)
    return out


# ------------------------------------------------------------ batched / served
def job_mix(kind, seed):
    """configs 4/5 job lists: (air, log_n, n_cols, seed)."""
    rng = np.random.default_rng(seed)
    if kind == "batched":   # 64 independent Wide-Fibonacci proofs, rows 2^10..2^16, 16..100 columns
        return [(0, int(rng.integers(10, 17)), int(rng.integers(16, 101)), i) for i in range(64)]
    jobs = []               # served: Poseidon2 2^12..2^18 and Wide-Fibonacci 2^12..2^20 (100 columns)
    for i in range(48):
        if rng.random() < 0.5:
            jobs.append((1, int(rng.integers(12, 19)), 0, i))
        else:
            jobs.append((0, int(rng.integers(12, 21)), 100, i))
    return jobs


def serving_metric(kind, channel="blake2s"):
    suffix = "" if channel == "blake2s" else ", Poseidon252 channel"
    if kind == "batched":
        return "batched vs sequential proofs/s (64 Wide-Fibonacci proofs, 2^10..2^16 rows)" + suffix
    return "served proofs/s with p50/p99 latency (Poisson mix of Poseidon2 2^12..2^18, WF 2^12..2^20)" + suffix


def gpu_busy_fraction(fn):
    """Fraction of fn's wall time during which at least one kernel ran on
    the device (kernel intervals from a CUPTI trace via torch.profiler,
    merged); fn runs once, outside any timed region."""
    import torch
    from torch.profiler import profile, ProfilerActivity
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    iv = []
    for e in prof.events():
        if e.device_type == torch.autograd.DeviceType.CUDA and "Memcpy" not in e.name and "Memset" not in e.name:
            iv.append((e.time_range.start, e.time_range.end))
    if not iv:
        return None
    iv.sort()
    busy, cur_s, cur_e = 0.0, iv[0][0], iv[0][1]
    for a, b in iv[1:]:
        if a > cur_e:
            busy += cur_e - cur_s
            cur_s, cur_e = a, b
        else:
            cur_e = max(cur_e, b)
    busy += cur_e - cur_s
    span = max(b for _, b in iv) - iv[0][0]
    return round(busy / span, 3) if span > 0 else None


def run_serving(args, world, rank, local):
    import torch
    from gpustark import prove as G
    from gpustark import serve as S
    from gpustark.backend import Context
    torch.cuda.set_device(local)
    ctx = Context(torch.cuda.current_stream())
    tuning = fft_autotune(args, 23)
    jobs = job_mix(args.workload, 1 + rank)
    mc = args.merkle_channel
    steps, warmup = max(1, args.steps), max(0, args.warmup)

    def single(a, n, c, sd):
        if a == 0:
            return G.prove_wide_fibonacci(n, c, seed=sd, input_mode=G.INPUT_SEEDED, ctx=ctx, merkle_channel=mc)
        return G.prove_poseidon(n, seed=sd, input_mode=G.INPUT_SEEDED, ctx=ctx, merkle_channel=mc)

    # warm-up: every distinct shape once (pool growth, twiddle trees, pinned buffers)
    for shape in sorted({(a, n, c) for a, n, c, _ in jobs}):
        single(*shape, 0)
    torch.cuda.synchronize()
    # sequential: one proof at a time on one stream, the same job list `steps` times
    barrier(world)
    seq_lat, seq_proofs = [], None
    t0 = time.perf_counter()
    for _ in range(steps):
        proofs = []
        for j in jobs:
            ts = time.perf_counter()
            proofs.append(single(*j))
            seq_lat.append(1e3 * (time.perf_counter() - ts))
        seq_proofs = seq_proofs or proofs
    seq_s = (time.perf_counter() - t0) / steps
    workers, fibers = args.workers, args.fibers
    arrivals = None
    lat, identical, busy = [], True, None
    with S.ProofServer(workers, 96 << 30, fibers_per_worker=fibers) as sv:
        # warm every context on every shape (twiddle trees, domain tables and
        # pool growth happen once per context): `workers * fibers` copies of
        # each shape in flight at once, then `warmup` whole batches
        conc = workers * fibers
        for a, n, c in sorted({(a, n, c) for a, n, c, _ in jobs}):
            for i in [sv.submit(a, n, c or 100, 0, merkle_channel=mc) for _ in range(conc)]:
                sv.wait(i)

        def batch(record):
            t_start = time.perf_counter()
            if args.workload == "batched":
                ids = [sv.submit(a, n, c or 100, sd, merkle_channel=mc) for a, n, c, sd in jobs]
            else:
                ids = []
                for (a, n, c, sd), at in zip(jobs, arrivals):
                    now = time.perf_counter() - t_start
                    if at > now:
                        time.sleep(at - now)
                    ids.append(sv.submit(a, n, c or 100, sd, merkle_channel=mc))
            res = [sv.wait(i) for i in ids]
            if record:
                lat.extend(l for _, l in res)
            return res

        if args.workload == "served":
            # Poisson arrivals at `load` x the sequential proof rate (seeded)
            rate = args.load * len(jobs) / seq_s
            gaps = np.random.default_rng(7 + rank).exponential(1.0 / rate, len(jobs))
            arrivals = np.cumsum(gaps)
        for _ in range(warmup):
            batch(False)
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(steps):
            res = batch(True)
            identical = identical and all(p == q for (p, _), q in zip(res, seq_proofs))
        srv_s = (time.perf_counter() - t0) / steps
        busy = gpu_busy_fraction(lambda: batch(False))
    lat = sorted(lat)
    srv_s = max_over_ranks(srv_s, world, "cuda")
    seq_s = max_over_ranks(seq_s, world, "cuda")
    pps = world * len(jobs) / srv_s
    seq_pps = world * len(jobs) / seq_s
    q = lambda v, f: float(np.percentile(np.asarray(v), f))
    mode = ("%d host threads x %d proof fibers (one CUDA stream each)" % (workers, fibers) if fibers > 1
            else "%d workers (one CUDA stream each)" % workers)
    out = {
        "metric": serving_metric(args.workload, mc),
        "value": round(pps, 2), "unit": "proofs/s", "n_gpus": world, "steps": steps, "warmup": warmup,
        "ms_per_step": round(1e3 * srv_s, 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (M31/QM31 integer arithmetic)", "data": "synthetic: seeded uniform M31",
        "config": {"workload": "%s: %d jobs per step, %s, admission by HBM footprint"
                               % (args.workload, len(jobs), mode),
                   "parallelism": "replicas x%d" % world, "fft_tuning": tuning},
        "sequential_proofs_per_s": round(seq_pps, 2), "speedup_vs_sequential": round(pps / seq_pps, 2),
        "latency_ms": {"p50": round(q(lat, 50), 2), "p99": round(q(lat, 99), 2)},
        "sequential_latency_ms": {"p50": round(q(seq_lat, 50), 2), "p99": round(q(seq_lat, 99), 2)},
        "proofs_identical_to_sequential": identical,
        "gpu_busy_fraction": busy,
        "e2e": {"value": round(pps, 2), "unit": "proofs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(len(p) for p in seq_proofs))},
    }
    if arrivals is not None:
        out["arrival_rate_per_s"] = round(args.load * len(jobs) / seq_s, 2)
    if args.workload == "batched" and mc == "blake2s":
        out["commit"] = run_batched_commit(ctx, 1 + rank)
    return out


def run_batched_commit(ctx, seed, n_cols=256, lo=12, hi=24, blowup=1, reps=5):
    """Mixed-size commitment: 256 columns with log sizes uniform in
    12..24, extended by 2^blowup and committed in one Merkle tree. Times the
    batched plan eagerly and replayed from a CUDA graph (same inputs, same
    root), and the FFT part issued one column per launch for comparison."""
    import torch
    from gpustark.backend import CommitPlan, GpuBackend as B
    rng = np.random.default_rng(seed)
    logs = [int(v) for v in rng.integers(lo, hi + 1, n_cols)]
    cols = [torch.randint(0, P, (1 << lg,), dtype=torch.int32, device="cuda") for lg in logs]
    st = torch.cuda.current_stream()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            r = fn()
            b.record(st)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts), r

    eager = CommitPlan(logs, blowup, use_graph=False, ctx=ctx)
    graph = CommitPlan(logs, blowup, use_graph=True, ctx=ctx)
    e_ms, e_root = timed(lambda: eager.run(cols))
    g_ms, g_root = timed(lambda: graph.run(cols))
    eager.close()
    graph.close()
    # FFT part, one column per launch (interpolate in place on a copy, extend)
    tw = B.precompute_twiddles(hi + blowup - 1, ctx=ctx)
    work = [c.clone() for c in cols]
    outs = [torch.empty(1 << (lg + blowup), dtype=torch.int32, device="cuda") for lg in logs]

    def per_column():
        for c, o, lg in zip(work, outs, logs):
            B.interpolate_columns([c], lg, tw, ctx=ctx)
            B.evaluate_polynomials([c], lg + blowup, tw, out=[o], ctx=ctx)
    pc_ms, _ = timed(per_column)
    alg = sum(4 * ((1 << lg) + (1 << (lg + blowup))) for lg in logs)  # read evals, write extension
    alg += sum(4 * (1 << (lg + blowup)) for lg in logs) + 32 * (1 << (hi + blowup + 1))  # leaves + hashes
    return {"columns": n_cols, "log_sizes": "uniform %d..%d (seed %d)" % (lo, hi, seed), "log_blowup": blowup,
            "eager_ms": round(e_ms, 3), "graph_ms": round(g_ms, 3), "graph_root_equals_eager": e_root == g_root,
            "fft_one_column_per_launch_ms": round(pc_ms, 3),
            "algorithmic_gbs_graph": round(alg / (g_ms / 1e3) / 1e9, 1)}


def run_reference(args, world, rank):
    """The reference arm: the CPU implementation of the path on the host cores.
    The reference's Rust prover cannot be built here (no Rust toolchain), so
    this times the oracle port (a C++ restatement of the reference CPU
    backend and prover) with all host threads, on the same metric."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    if args.workload == "kernels":
        vals, t_all, desc = [], 0.0, ""
        for _ in range(args.warmup):
            cpu_sweep_sample(threads)
        for _ in range(args.steps):
            gbs, secs, desc = cpu_sweep_sample(threads)
            vals.append(gbs)
            t_all += secs
        v = statistics.mean(vals)
        return {
            "impl": "reference",
            "metric": "FFT/Merkle HBM GB/s (kernel sweep: circle FFT 2^16..2^26, Merkle 64x2^20, fold 2^22)",
            "value": round(v, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * t_all / max(args.steps, 1), 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31)", "data": "synthetic: seeded uniform M31",
            "config": {"workload": "kernel sweep, bounded CPU sample", "parallelism": "cpu threads"},
            "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    if args.workload in ("batched", "served"):
        jobs = job_mix(args.workload, 1)
        v, desc = cpu_mix_sample(jobs, threads)
        return {
            "impl": "reference", "metric": serving_metric(args.workload), "value": round(v, 3), "unit": "proofs/s",
            "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": round(1e3 / v, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 (M31/QM31 integer arithmetic)",
            "data": "synthetic: seeded uniform M31",
            "config": {"workload": "%s job mix, proved one at a time on the host cores" % args.workload,
                       "parallelism": "cpu threads"},
            "cpu_baseline": {"value": round(v, 3), "unit": "proofs/s", "cores": threads, "kind": "port",
                             "sample": desc},
            "e2e": {"value": round(v, 3), "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    log_n = args.log_n or PROOF_SIZES[args.workload]
    mc = args.merkle_channel
    # the same step count as the GPU arm, unless that would run past about
    # 150 s of CPU proving (sized from the one warm-up proof)
    warm = min(args.warmup, 1)
    est = None
    for _ in range(warm):
        t0 = time.perf_counter()
        cpu_proof_sample(args.workload, threads, log_n, mc)
        est = time.perf_counter() - t0
    vals, desc = [], ""
    steps = max(1, args.steps if est is None or est * args.steps <= 150 else int(150 / est))
    for _ in range(steps):
        ms, desc = cpu_proof_sample(args.workload, threads, log_n, mc)
        vals.append(ms)
    v = statistics.mean(vals)
    return {
        "impl": "reference", "metric": proof_metric(args.workload, mc), "value": round(v, 1), "unit": "ms",
        "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": round(v, 1),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (M31/QM31 integer arithmetic)", "data": "synthetic: seeded uniform M31",
        "config": dict(proof_config(args.workload, log_n, mc), parallelism="cpu threads"),
        "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def proof_timeline(air, log_n, reps):
    """Device timeline of `reps` proofs after warm-up, from a CUPTI activity trace
    (torch.profiler, CUDA activities only): per proof the span from the first to
    the last device event, the time at least one kernel or copy runs (the union
    of their intervals: kernels of the work and side streams overlap), and the
    idle time split by what borders each gap (kernel or copy on either side)."""
    import json as js
    import tempfile
    import torch
    from torch.profiler import profile, ProfilerActivity
    from gpustark import prove as G
    fn = ((lambda: G.prove_poseidon(log_n, seed=7, input_mode=G.INPUT_SEEDED)) if air == "poseidon" else
          (lambda: G.prove_wide_fibonacci(log_n, 100, seed=7, input_mode=G.INPUT_SEEDED)))
    for _ in range(4):
        fn()
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(reps):
            fn()
            torch.cuda.synchronize()
    path = os.path.join(tempfile.mkdtemp(), "trace.json")
    prof.export_chrome_trace(path)
    ev = [e for e in js.load(open(path))["traceEvents"]
          if e.get("ph") == "X" and e.get("cat") in ("kernel", "gpu_memcpy", "gpu_memset")]
    ev.sort(key=lambda e: e["ts"])
    # split into proofs at the host-side gaps between them (the largest reps - 1 gaps)
    ends, end = [], ev[0]["ts"]
    for i, e in enumerate(ev):
        if i and e["ts"] > end:
            ends.append((e["ts"] - end, i))
        end = max(end, e["ts"] + e["dur"])
    cuts = sorted(i for _, i in sorted(ends, reverse=True)[:reps - 1])
    rows, lo = [], 0
    for hi in cuts + [len(ev)]:
        part = ev[lo:hi]
        lo = hi
        t0 = part[0]["ts"]
        end, busy, prev = t0, 0.0, None
        idle = {"kernel->kernel": 0.0, "kernel->copy": 0.0, "copy->kernel": 0.0, "copy->copy": 0.0}
        for e in part:
            s, d = e["ts"], e["dur"]
            if s > end and prev is not None:
                k = ("kernel" if prev["cat"] == "kernel" else "copy") + "->" + ("kernel" if e["cat"] == "kernel" else "copy")
                idle[k] += s - end
            busy += max(0.0, s + d - max(s, end))
            if s + d > end:
                end, prev = s + d, e
        rows.append((end - t0, busy, idle, sum(1 for e in part if e["cat"] == "kernel")))
    n = len(rows)
    span = sum(r[0] for r in rows) / n
    busy = sum(r[1] for r in rows) / n
    idle = {k: round(sum(r[2][k] for r in rows) / n, 1) for k in rows[0][2]}
    print(js.dumps({"air": air, "log_n": log_n, "proofs": n, "span_us": round(span, 1), "busy_us": round(busy, 1),
                    "busy_frac": round(busy / span, 3), "idle_us": idle,
                    "kernels_per_proof": round(sum(r[3] for r in rows) / n, 1)}))


def fft_worklist_case(n_items, min_log, max_log, args):
    """Many FFTs of uneven sizes: n_items columns of log sizes uniform in
    [min_log, max_log], half interpolated in place, half evaluated with blowup
    1 (coefficients of log - 1), timed three ways on one stream with CUDA
    events (device time of the whole sequence, host launch costs included):
    one gs_fft_worklist call; one gs_interpolate_columns / gs_evaluate_columns
    call per size group; one call per column. Prints one JSON line."""
    import torch
    from gpustark import lib as gslib
    from gpustark.backend import GpuBackend as B, Context
    rng = np.random.default_rng(11)
    ctx = Context(torch.cuda.current_stream())
    tw = B.precompute_twiddles(max_log, ctx=ctx)
    items = []
    for k in range(n_items):
        log = int(rng.integers(min_log, max_log + 1))
        if k % 2 == 0:
            x = torch.from_numpy(rng.integers(0, P, 1 << log, dtype=np.int64).astype(np.int32)).cuda()
            items.append(("interpolate", x, x))
        else:
            c = torch.from_numpy(rng.integers(0, P, 1 << (log - 1), dtype=np.int64).astype(np.int32)).cuda()
            items.append(("evaluate", c, torch.empty(1 << log, dtype=torch.int32, device="cuda")))
    groups = {}
    for kind, s, d in items:
        groups.setdefault((kind, s.numel(), d.numel()), []).append((s, d))
    # every argument array is built once, outside the timed loops: the three
    # forms differ in their launches, not in Python-side preparation
    import ctypes as C
    from gpustark import _lib as L
    lib = gslib()
    arr = (L.FftItem * n_items)()
    for k, (kind, s, d) in enumerate(items):
        arr[k].src, arr[k].dst = s.data_ptr(), d.data_ptr()
        arr[k].log_size = d.numel().bit_length() - 1
        arr[k].coeffs_log_size = s.numel().bit_length() - 1
        arr[k].inverse = 1 if kind == "interpolate" else 0
    twp, itwp = C.c_void_p(tw.twiddles.data_ptr()), C.c_void_p(tw.itwiddles.data_ptr())
    calls_group = []
    for (kind, ns, nd), cols in groups.items():
        dp, kd = L.ptr_array([d.data_ptr() for _, d in cols])
        if kind == "interpolate":
            calls_group.append((lib.gs_interpolate_columns, (ctx.handle, dp, len(cols), nd.bit_length() - 1, itwp,
                                                             tw.root_log), kd))
        else:
            sp, ks = L.ptr_array([s.data_ptr() for s, _ in cols])
            calls_group.append((lib.gs_evaluate_columns, (ctx.handle, sp, ns.bit_length() - 1, dp, len(cols),
                                                          nd.bit_length() - 1, twp, tw.root_log), (kd, ks)))
    calls_col = []
    for kind, s, d in items:
        dp, kd = L.ptr_array([d.data_ptr()])
        if kind == "interpolate":
            calls_col.append((lib.gs_interpolate_columns, (ctx.handle, dp, 1, d.numel().bit_length() - 1, itwp,
                                                           tw.root_log), kd))
        else:
            sp, ks = L.ptr_array([s.data_ptr()])
            calls_col.append((lib.gs_evaluate_columns, (ctx.handle, sp, s.numel().bit_length() - 1, dp, 1,
                                                        d.numel().bit_length() - 1, twp, tw.root_log), (kd, ks)))

    def worklist():
        L.check(lib.gs_fft_worklist(ctx.handle, arr, n_items, twp, itwp, tw.root_log), "fft_worklist")

    def per_size():
        for f, a, _ in calls_group:
            L.check(f(*a), "fft")

    def per_column():
        for f, a, _ in calls_col:
            L.check(f(*a), "fft")

    res = {}
    for name, fn in (("worklist", worklist), ("per_size_group", per_size), ("per_column", per_column)):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        l0 = gslib().gs_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        e1.synchronize()
        res[name] = {"us": round(1e3 * e0.elapsed_time(e1) / args.steps, 1),
                     "launches": (gslib().gs_launch_count() - l0) // args.steps}
    words = sum(d.numel() for _, _, d in items)
    print(json.dumps({"case": "fft_worklist", "items": n_items, "logs": [min_log, max_log],
                      "size_groups": len(groups), "output_words": words, **res}))


def merkle_worklist_case(n_trees, min_log, max_log, n_cols, args):
    """Many small Merkle trees: n_trees trees of n_cols columns, log sizes
    uniform in [min_log, max_log], built (leaves and every node layer) by one
    gs_merkle_worklist call, against one gs_commit_on_layer +
    gs_commit_node_layers pair per tree (the per-tree path). CUDA events
    around the whole sequence, argument arrays built outside the timed loop;
    one JSON line."""
    import ctypes as C
    import torch
    from gpustark import lib as gslib
    from gpustark import _lib as L
    from gpustark.backend import Context
    rng = np.random.default_rng(13)
    ctx = Context(torch.cuda.current_stream())
    lib = gslib()
    arr = (L.MerkleItem * n_trees)()
    keep, per_tree = [], []
    for k in range(n_trees):
        log = int(rng.integers(min_log, max_log + 1))
        cols = torch.from_numpy(rng.integers(0, P, (n_cols, 1 << log), dtype=np.int64).astype(np.int32)).cuda()
        layers = [torch.empty((1 << lg) * 8, dtype=torch.int32, device="cuda") for lg in range(log + 1)]
        cp, kc = L.ptr_array([cols[i].data_ptr() for i in range(n_cols)])
        lp, kl = L.ptr_array([t.data_ptr() for t in layers])
        keep += [cols, layers, kc, kl]
        arr[k].cols, arr[k].n_cols, arr[k].log_size, arr[k].layers = cp, n_cols, log, lp
        per_tree.append((log, cp, C.c_void_p(layers[log].data_ptr()), lp))

    def worklist():
        L.check(lib.gs_merkle_worklist(ctx.handle, arr, n_trees), "merkle_worklist")

    def per_tree_calls():
        for log, cp, leaf, lp in per_tree:
            L.check(lib.gs_commit_on_layer(ctx.handle, log, None, n_cols, cp, leaf), "commit_on_layer")
            if log:
                L.check(lib.gs_commit_node_layers(ctx.handle, log, lp), "commit_node_layers")

    res = {}
    for name, fn in (("worklist", worklist), ("per_tree", per_tree_calls)):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        l0 = lib.gs_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        e1.synchronize()
        res[name] = {"us": round(1e3 * e0.elapsed_time(e1) / args.steps, 1),
                     "launches": (lib.gs_launch_count() - l0) // args.steps}
    print(json.dumps({"case": "merkle_worklist", "trees": n_trees, "logs": [min_log, max_log], "columns": n_cols,
                      **res}))


def run_case(args):
    """One op on a small case, for ncu captures: `--case fft:26`, `--case lde:18:162:2` (extension
    of 162 columns from 2^18 to 2^20), `--case merkle:20:64`, `--case fold:22`, `--case p252:18:8`
    (Poseidon252 Merkle leaves of 8 columns x 2^18 rows, then the node layer above them);
    `--case timeline:poseidon:18` prints the device timeline of proofs (busy and idle time)."""
    import torch
    from gpustark.backend import GpuBackend as B, to_device, Context
    kind, *params = args.case.split(":")
    if kind == "timeline":
        proof_timeline(params[0], int(params[1]), max(2, args.steps))
        return
    if kind == "fftwl":
        fft_worklist_case(int(params[0]), int(params[1]), int(params[2]), args)
        return
    if kind == "merklewl":
        merkle_worklist_case(int(params[0]), int(params[1]), int(params[2]), int(params[3]), args)
        return
    rng = np.random.default_rng(7)
    ctx = Context(torch.cuda.current_stream())
    if kind == "fft":
        n = int(params[0])
        tw = B.precompute_twiddles(n, ctx=ctx)
        x = to_device(rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32))
        y = torch.empty_like(x)
        work = lambda: (B.evaluate_polynomials([x], n, tw, out=[y], ctx=ctx), B.interpolate_columns([y], n, tw, ctx=ctx))
    elif kind == "lde":
        n, k = int(params[0]), int(params[1])
        b = int(params[2]) if len(params) > 2 else 1
        tw = B.precompute_twiddles(n + b - 1, ctx=ctx)
        src = torch.from_numpy(rng.integers(0, P, (k, 1 << n), dtype=np.int64).astype(np.int32)).cuda()
        dst = torch.empty((k, 1 << (n + b)), dtype=torch.int32, device="cuda")
        cs = [src[i] for i in range(k)]
        ev = [dst[i] for i in range(k)]
        work = lambda: B.evaluate_polynomials(cs, n + b, tw, out=ev, ctx=ctx)
    elif kind == "merkle":
        n, k = int(params[0]), int(params[1])
        cols = [to_device(rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32)) for _ in range(k)]
        out = torch.empty((1 << n) * 8, dtype=torch.int32, device="cuda")
        work = lambda: B.commit_on_layer(n, None, cols, ctx=ctx, out=out)
    elif kind == "p252":
        n, k = int(params[0]), int(params[1])
        cols = [to_device(rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32)) for _ in range(k)]
        leaves = torch.empty((1 << n) * 32, dtype=torch.uint8, device="cuda")
        nodes = torch.empty((1 << (n - 1)) * 32, dtype=torch.uint8, device="cuda")
        work = lambda: (B.poseidon252_commit_on_layer(n, None, cols, ctx=ctx, out=leaves),
                        B.poseidon252_commit_on_layer(n - 1, leaves, [], ctx=ctx, out=nodes))
    elif kind == "fold":
        n = int(params[0])
        tw = B.precompute_twiddles(n + 1, ctx=ctx)
        ev = [to_device(rng.integers(0, P, 1 << n, dtype=np.int64).astype(np.uint32)) for _ in range(4)]
        work = lambda: B.fold_line(ev, n, [1, 2, 3, 4], tw, ctx=ctx)
    else:
        raise SystemExit("unknown case " + args.case)
    for _ in range(args.warmup + args.steps):
        work()
    torch.cuda.synchronize()
    print("case done:", args.case)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpustark", choices=["gpustark", "reference"])
    ap.add_argument("--workload", default="poseidon",
                    choices=["poseidon", "wide_fibonacci", "kernels", "batched", "served"])
    ap.add_argument("--workers", type=int, default=4, help="server host threads (batched / served)")
    ap.add_argument("--fibers", type=int, default=6,
                    help="batched / served: proofs per server thread as cooperative fibers (1 = one proof per thread)")
    ap.add_argument("--load", type=float, default=2.0, help="served: arrival rate / sequential proof rate")
    ap.add_argument("--merkle-channel", default="blake2s", choices=["blake2s", "poseidon252"],
                    help="proof workloads: Blake2sMerkleChannel or Poseidon252MerkleChannel")
    ap.add_argument("--log-n", type=int, default=0, help="override the proof size (log instances / rows)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fft-autotune", default="on", choices=["on", "off"],
                    help="time the FFT pass splits per log size before warm-up and install the fastest")
    ap.add_argument("--case", default=None,
                    help="profiling case: fft:<log>, lde:<log>:<cols>[:<ext>], merkle:<log>:<cols>, fold:<log> (one op, "
                         "no JSON contract); fftwl:<items>:<min_log>:<max_log> times the FFT work-list against "
                         "per-size and per-column calls; merklewl:<trees>:<min_log>:<max_log>:<cols> the Merkle "
                         "work-list against per-tree calls")
    args = ap.parse_args()
    if args.case:
        run_case(args)
        return
    if args.impl == "reference":
        world, rank, _ = dist_setup(args, "gloo")
        out = run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup(args, "nccl")
        if args.workload == "kernels":
            out = run_kernels(args, world, rank, local)
        elif args.workload in ("batched", "served"):
            out = run_serving(args, world, rank, local)
        else:
            out = run_proof(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
