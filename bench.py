#!/usr/bin/env python
"""Benchmark of the B200 transform path (one JSON line on rank 0).

Default workload: the fused real pipeline rfft(4096) -> raised-cosine notch
(mul-spectrum, bins 400-420 with 32-bin ramps) -> irfft, FP32, batch 8192
signals of N(0,1) noise + a 5-amplitude tone at bin 410 (seed 1).  One step
is one pass of the fused pipeline kernel over the whole batch, inputs
resident in HBM; the metric is algorithmic HBM GB/s (each input sample read
once, each output sample written once: 8 bytes per sample) and its fraction
of the measured HBM copy bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload pipeline|r2c|c2c1024|c2c4096|c2c16384|c2c16384tc|c2c4096fp64|
                                stft|istft|cwt|icwt|uneven|serve]

--workload serve replays a Poisson request trace (20k requests/s: 40% rfft
of log-uniform sizes 256..65536 rounded to the recommended size, 30% the
notch pipeline, 30% STFT of log-uniform 2^16..2^20 samples) through the
continuous-batching server and reports p50 / p99 latency and throughput,
next to the same trace served one request at a time (no merging, one
stream).

--impl reference times the reference library's own CPU path (compiled from
its sources into oracle/_ref) on all host cores over a bounded sample of the
same workload.  Under torchrun (N > 1) every rank runs its own batch (weak
scaling, no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

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

FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 1024 * 1024


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def notch_mask(n=4096, lo=400, hi=420, ramp=32):
    nb = n // 2 + 1
    k = np.arange(nb)
    m = np.ones(nb)
    m[(k >= lo) & (k <= hi)] = 0.0
    left = (k >= lo - ramp) & (k < lo)
    m[left] = 0.5 * (1 + np.cos(np.pi * (k[left] - (lo - ramp)) / ramp))
    right = (k > hi) & (k <= hi + ramp)
    m[right] = 0.5 * (1 - np.cos(np.pi * (k[right] - hi) / ramp))
    return m.astype(np.float32)


WORKLOADS = {
    # name: (description, n, batch, bytes per transform, flops per transform)
    "pipeline": ("fused rfft(4096)->notch mul-spectrum->irfft, batch 8192, seed 1",
                 4096, 8192, 8 * 4096, 2 * 2.5 * 4096 * 12),
    "r2c": ("R2C n=4096 batch 8192, seed 1", 4096, 8192, 4 * 4096 + 8 * 2049, 2.5 * 4096 * 12),
    "c2c1024": ("C2C n=1024 batch 256 forward (split planes), seed 0", 1024, 256,
                16 * 1024, 5 * 1024 * 10),
    "c2c16384": ("C2C n=16384 batch 2048 forward (split planes), seed 3", 16384, 2048,
                 16 * 16384, 5 * 16384 * 14),
    "c2c4096": ("C2C n=4096 batch 8192 forward (split planes, inputs landed by bulk copy), seed 3",
                4096, 8192, 16 * 4096, 5 * 4096 * 12),
    "c2c16384tc": ("C2C n=16384 batch 2048 forward, tensor-core form (64-point DFTs as FP16 "
                   "hi+lo tcgen05 MMAs in two passes, radix-4 on CUDA cores, FP32 accumulation), "
                   "seed 3, 1% of entries x1e3",
                   16384, 2048, 16 * 16384, 5 * 16384 * 14),
    "stft": ("STFT Hann 1024 hop 256, 64 signals x 2^18 samples, seed 4", 1024, 64,
             None, None),
    "uneven": ("uneven batch: 4096 C2C, lengths uniform over {12,17,31,60,240,1000,3072,6000,"
               "16384,65536} (sorted by length), U[-1,1), seed 2, one persistent launch",
               None, 4096, None, None),
}

WORKLOADS["c2c4096fp64"] = ("C2C n=4096 batch 4096 forward in FP64 (split planes, FAF_PREC_FP64), "
                            "U[-1,1), seed 0", 4096, 4096, 32 * 4096, 5 * 4096 * 12)
WORKLOADS["istft"] = ("inverse STFT Hann 1024 hop 256: 64 signals x 1021 frames x 513 bins -> "
                      "2^18 samples, N(0,1) frames, seed 4", 1024, 64, None, None)

# 60 rows: the row count of the reference's default bank (Morse 20/3, 10
# voices, lowpass) at n = 4096; the rows themselves are synthetic here.
CWT_ROWS = 60
WORKLOADS["cwt"] = ("CWT filter bank n=4096: 256 signals x 60 rows (synthetic Gaussian bandpass "
                    "bank, seed 6; the reference's default bank has 60 rows at this n), N(0,1) "
                    "signals, seed 5", 4096, 256, 4 * 4096 * (1 + CWT_ROWS), None)


def cwt_bank(rows=CWT_ROWS, n=4096, seed=6):
    """Seeded Gaussian bandpass rows on geometric centres (an analytic
    wavelet bank's shape: positive, one octave per 10 rows)."""
    nb = n // 2 + 1
    k = np.arange(nb)[None, :]
    c = np.geomspace(2.0, 0.8 * nb, rows)[:, None]
    g = np.random.default_rng(seed).uniform(0.8, 1.2, (rows, 1))
    return (g * np.exp(-0.5 * ((k - c) / (0.2 * c + 1.0)) ** 2)).astype(np.float32)


WORKLOADS["icwt"] = ("inverse CWT (dual frame) n=4096: 256 coefficient sets x 60 rows -> 256 "
                     "signals (dual rows of the synthetic bank, seed 6), N(0,1) coefficients, "
                     "seed 7", 4096, 256, 4 * 4096 * (1 + CWT_ROWS), None)

WORKLOADS["serve"] = ("serving trace: 4000 requests, Poisson 20k req/s (seed 4); 40% rfft "
                      "N log-uniform [256, 65536] -> recommended size, 30% notch pipeline "
                      "4096, 30% STFT Hann 1024 hop 256 over L log-uniform [2^16, 2^20]; "
                      "inputs N(0,1) generated on the device", None, 4000, None, None)

UNEVEN_SET = [12, 17, 31, 60, 240, 1000, 3072, 6000, 16384, 65536]


def uneven_lengths(batch=4096):
    rng = np.random.default_rng(2)
    return sorted(int(v) for v in rng.choice(UNEVEN_SET, batch))


def make_inputs(workload, batch):
    n = WORKLOADS[workload][1]
    if workload in ("pipeline", "r2c"):
        rng = np.random.default_rng(1)
        k = np.arange(n)
        x = rng.standard_normal((batch, n), dtype=np.float32)
        x += (5 * np.cos(2 * np.pi * 410 * k / n)).astype(np.float32)
        return [x]
    if workload == "c2c4096fp64":
        rng = np.random.default_rng(0)
        return [rng.uniform(-1, 1, (batch, n)), rng.uniform(-1, 1, (batch, n))]
    if workload == "istft":
        rng = np.random.default_rng(4)
        F_ = stft_geometry(1 << 18)[0]
        return [rng.standard_normal((batch, F_, 513), dtype=np.float32),
                rng.standard_normal((batch, F_, 513), dtype=np.float32)]
    if workload.startswith("c2c"):
        seed = 0 if workload == "c2c1024" else 3
        rng = np.random.default_rng(seed)
        re = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
        im = rng.uniform(-1, 1, (batch, n)).astype(np.float32)
        if workload.startswith("c2c16384"):
            for a in (re, im):
                a[rng.random(a.shape) < 0.01] *= 1e3
        return [re, im]
    if workload == "stft":
        rng = np.random.default_rng(4)
        return [rng.standard_normal((batch, 1 << 18), dtype=np.float32)]
    if workload == "cwt":
        return [np.random.default_rng(5).standard_normal((batch, n), dtype=np.float32)]
    if workload == "icwt":
        return [np.random.default_rng(7).standard_normal((batch, CWT_ROWS, n), dtype=np.float32)]
    if workload == "uneven":
        total = sum(uneven_lengths(batch))
        rng = np.random.default_rng(2)
        return [rng.uniform(-1, 1, total).astype(np.float32),
                rng.uniform(-1, 1, total).astype(np.float32)]
    raise ValueError(workload)


def stft_geometry(L, n=1024, win=1024, hop=256):
    F = 1 + (L - win) // hop
    return F, F * (n // 2 + 1)


def algorithmic_bytes(workload, batch):
    if workload == "uneven":
        return 16 * sum(uneven_lengths(batch))
    if workload in ("stft", "istft"):
        L = 1 << 18
        F, bins = stft_geometry(L)
        return batch * (4 * L + 8 * bins)
    return batch * WORKLOADS[workload][3]


# ---------------------------------------------------------------------------
# clocks (NVML, sampled during the timed region)
# ---------------------------------------------------------------------------

class ClockSampler:
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def result(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "measured"
    except Exception:
        pass
    return FALLBACK_HBM_GBS, "fallback"


# committed ncu summary of each workload's dominant kernel
PROFILES = {"uneven": "uneven_config3", "c2c16384tc": "c2c_tc_16384"}


def ncu_traffic(workload):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/<name>.md, line `traffic_per_launch_bytes: X`)."""
    p = os.path.join(ROOT, "profiles", f"{PROFILES.get(workload, workload)}.md")
    try:
        with open(p) as f:
            for line in f:
                if line.strip().startswith("traffic_per_launch_bytes:"):
                    return float(line.split(":", 1)[1].strip().split()[0])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def build_transform(F, workload, torch):
    n = WORKLOADS[workload][1]
    if workload == "pipeline":
        t = F.Transform.chirp(f"(pipeline (rfft :size {n}) (mul-spectrum) (irfft))")
        m = torch.from_numpy(notch_mask(n)).cuda()
        z = torch.zeros_like(m)
        t.bind(m, z, n // 2 + 1)
        return t
    if workload == "r2c":
        return F.Transform.rfft(n)
    if workload == "c2c16384tc":
        return F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
    if workload == "c2c4096fp64":
        return F.Transform.fft(n, precision=F.PREC_FP64)
    if workload == "istft":
        return F.Transform.istft(1024, win=1024, hop=256)
    if workload == "cwt":
        return F.Transform.cwt(4096, cwt_bank())
    if workload == "icwt":
        return F.Transform.icwt_dual(4096, F.Transform.cwt_dual_rows(cwt_bank()))
    if workload.startswith("c2c"):
        return F.Transform.fft(n)
    if workload == "stft":
        return F.Transform.stft(1024, win=1024, hop=256)
    if workload == "uneven":
        return F.Uneven(uneven_lengths(WORKLOADS["uneven"][2]), measure=True)
    raise ValueError(workload)


def run_step(F, t, workload, ins, outs, plain=False):
    if workload == "pipeline":
        t.pipeline(ins[0], out=outs[0])
    elif workload == "r2c":
        t.r2c(ins[0], out_re=outs[0], out_im=outs[1])
    elif workload.startswith("c2c"):
        t.c2c(ins[0], ins[1], out_re=outs[0], out_im=outs[1])
    elif workload == "stft":
        t.stft_frames(ins[0], out_re=outs[0], out_im=outs[1])
    elif workload == "istft":
        t.istft_frames(ins[0], ins[1], out=outs[0])
    elif workload == "cwt":
        t.analyze(ins[0], out=outs[0])
    elif workload == "icwt":
        t.synthesize(ins[0], out=outs[0])
    elif workload == "uneven":
        if hasattr(ins[0], "data_ptr"):
            t.execute(ins[0], ins[1], outs[0], outs[1], plain=plain)
        else:
            # the uneven API takes device buffers: pinned host -> device copies
            # into buffers kept across steps (so the captured graph replays),
            # then device -> pinned host copies of both output planes
            import torch
            if getattr(t, "_stage", None) is None:
                t._stage = [torch.empty(a.shape, dtype=torch.float32, device="cuda")
                            for a in list(ins) + list(outs)]
            d = t._stage
            for dev, host in zip(d[:2], ins):
                dev.copy_(torch.from_numpy(host), non_blocking=True)
            t.execute(d[0], d[1], d[2], d[3], plain=plain)
            for dev, host in zip(d[2:], outs):
                torch.from_numpy(host).copy_(dev, non_blocking=True)
            torch.cuda.current_stream().synchronize()


def alloc_outputs(workload, batch, like, torch):
    n = WORKLOADS[workload][1]
    # torch tensors -> device outputs; numpy inputs -> pinned host numpy outputs
    dt = torch.float64 if workload == "c2c4096fp64" else torch.float32
    if hasattr(like, "data_ptr"):
        mk = lambda shp: torch.empty(shp, dtype=dt, device=like.device)  # noqa: E731
    else:
        mk = lambda shp: torch.empty(shp, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    if workload == "pipeline":
        return [mk((batch, n))]
    if workload == "r2c":
        return [mk((batch, n // 2 + 1)), mk((batch, n // 2 + 1))]
    if workload.startswith("c2c"):
        return [mk((batch, n)), mk((batch, n))]
    if workload == "stft":
        F_, bins = stft_geometry(1 << 18)
        return [mk((batch, F_, 513)), mk((batch, F_, 513))]
    if workload == "istft":
        return [mk((batch, 1 << 18))]
    if workload == "cwt":
        return [mk((batch, CWT_ROWS, n))]
    if workload == "icwt":
        return [mk((batch, n))]
    if workload == "uneven":
        total = sum(uneven_lengths(batch))
        return [mk((total,)), mk((total,))]


def max_over_ranks(x, dist, device):
    """Max of a per-rank float over all ranks (identity without a process
    group); every rank calls it at the same point."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def buffer_sets(workload, nbytes):
    """Input/output buffer sets the timed loop rotates over: enough that
    consecutive steps never share a set and the sets together exceed twice
    the L2, so no step reads data the step before left in L2.  Working sets
    under 16 MB (the launch-bound C2C of 256 x 1024) stay L2-resident: one."""
    if nbytes < (16 << 20):
        return 1
    return max(2, -(-2 * L2_BYTES // nbytes))


def fp64_check(workload, host_in, outs, batch, sample=8):
    """rel L2 of the first and last `sample` transforms of a timed output
    against FP64 numpy (the reference semantics: NumPy-style norm)."""
    n = WORKLOADS[workload][1]
    idx = sorted(set(list(range(min(sample, batch))) + list(range(max(0, batch - sample), batch))))
    get = lambda a: a[idx].cpu().numpy().astype(np.float64)  # noqa: E731
    if workload == "pipeline":
        x = host_in[0][idx].astype(np.float64)
        want = np.fft.irfft(np.fft.rfft(x, axis=-1) * notch_mask(n), n=n, axis=-1)
        got = get(outs[0])
    elif workload == "r2c":
        want = np.fft.rfft(host_in[0][idx].astype(np.float64), axis=-1)
        got = get(outs[0]) + 1j * get(outs[1])
    elif workload.startswith("c2c"):
        want = np.fft.fft(host_in[0][idx].astype(np.float64) + 1j * host_in[1][idx], axis=-1)
        got = get(outs[0]) + 1j * get(outs[1])
    else:
        return None
    return {"rel_l2_vs_fp64": float(np.linalg.norm(got - want) / np.linalg.norm(want)),
            "sample": f"transforms {idx[0]}..{idx[min(sample, len(idx)) - 1]} and the last "
                      f"{min(sample, batch)} of the last timed step"}


def gpu_lead(torch, stream):
    """Keep `stream` busy for about 0.5 ms (a GPU-side spin), so that the
    timed region opened after it starts with work already queued behind it:
    the host's call for the first timed step then runs while the GPU spins,
    not inside the timed region.  Nothing of a timed step is skipped."""
    sleep = getattr(torch.cuda, "_sleep", None)
    if sleep is None:  # no spin available: the timed region opens on an idle GPU
        return
    with torch.cuda.stream(stream):
        sleep(1_000_000)


def time_steps(torch, stream, steps, fn):
    """CUDA-event time of `steps` calls fn(i) on `stream` (ms per step)."""
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    gpu_lead(torch, stream)
    ev0.record(stream)
    for i in range(steps):
        fn(i)
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / steps


def step_latencies(torch, stream, steps, fn):
    """p50 / p99 / max of `steps` individually timed calls fn(i) (CUDA events
    around each call on `stream`), in ms."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(evs):
        a.record(stream)
        fn(i)
        b.record(stream)
    torch.cuda.synchronize()
    ms = np.array([a.elapsed_time(b) for a, b in evs])
    return {"p50_ms": round(float(np.percentile(ms, 50)), 4),
            "p99_ms": round(float(np.percentile(ms, 99)), 4),
            "max_ms": round(float(ms.max()), 4), "steps": steps}


def r2c_subrecord(F, torch, stream, sets, host_in, steps, peak):
    """Kernel-only R2C n=4096 on the headline's seed-1 signals (batch 8192),
    rotating over the same input sets: the >= 70 % of HBM target's line."""
    n, batch = 4096, WORKLOADS["r2c"][2]
    t = F.Transform.rfft(n)
    t.set_stream(stream)
    outs = [alloc_outputs("r2c", batch, ins[0], torch) for ins, _ in sets]
    step = lambda i: run_step(F, t, "r2c", sets[i % len(sets)][0], outs[i % len(sets)])  # noqa
    for i in range(3):
        step(i)
    ms = time_steps(torch, stream, steps, step)
    nbytes = algorithmic_bytes("r2c", batch)
    gbs = nbytes / (ms * 1e-3) / 1e9
    chk = fp64_check("r2c", host_in, outs[(steps - 1) % len(sets)], batch)
    rec = {"kernel": "k2_r2c", "workload": WORKLOADS["r2c"][0], "value": round(gbs, 1),
           "unit": "GB/s", "ms_per_step": round(ms, 5), "frac": round(gbs / peak, 4),
           "algorithmic_bytes_per_launch": nbytes, "traffic": ncu_traffic("r2c"),
           "output_check": chk, "wait_status": t.wait_status(),
           "gpu_launches": steps * F.lib().faf_cuda_last_launches()}
    t.close()
    return rec


def run_ours(args, rank, world, local_rank):
    import torch
    import fastandfourier_b200 as F

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    workload = args.workload
    desc, n, batch, _, flops_per = WORKLOADS[workload]
    host_in = make_inputs(workload, batch)
    nbytes = algorithmic_bytes(workload, batch)
    nsets = buffer_sets(workload, nbytes)
    sets = []
    for _ in range(nsets):
        ins = [torch.from_numpy(a).cuda() for a in host_in]
        sets.append((ins, alloc_outputs(workload, batch, ins[0], torch)))
    stream = torch.cuda.current_stream()
    # the uneven plan replays a CUDA graph captured on fixed buffers: one plan
    # per buffer set
    plans = [build_transform(F, workload, torch)
             for _ in range(nsets if workload == "uneven" else 1)]
    for p in plans:
        p.set_stream(stream)
    t = plans[0]

    def step(i, plain=False, pl=None):
        k = i % nsets
        run_step(F, (pl or plans)[k % len(pl or plans)], workload, sets[k][0], sets[k][1],
                 plain=plain)

    for i in range(max(args.warmup, 3)):
        step(i)
    sampler = ClockSampler(local_rank)
    with sampler:  # sampling starts before the barrier, so its start-up is not timed
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gpu_lead(torch, stream)
        ev0.record(stream)
        for i in range(args.steps):
            step(i)
        ev1.record(stream)
        torch.cuda.synchronize()
    # every step is the same call: the last one's launch count, times the steps
    launches = args.steps * F.lib().faf_cuda_last_launches()
    ms = ev0.elapsed_time(ev1)
    if dist:
        dist.barrier()
    ms = max_over_ranks(ms, dist, "cuda")
    ms_per_step = ms / args.steps
    value = world * nbytes / (ms_per_step * 1e-3) / 1e9
    last_outs = sets[(args.steps - 1) % nsets][1]
    check = fp64_check(workload, host_in, last_outs, batch)
    wait = t.wait_status() if hasattr(t, "wait_status") else None
    plain = None
    if workload == "uneven":
        # the plain GPU method on the same data: one batched launch per length
        for i in range(3):
            step(i, plain=True)
        pms = time_steps(torch, stream, args.steps, lambda i: step(i, plain=True))
        plain = {"value": round(nbytes / (pms * 1e-3) / 1e9, 1), "ms_per_step": round(pms, 4),
                 "launches_per_step": len(set(uneven_lengths(batch))),
                 "speedup_of_persistent": round(pms / ms_per_step, 3)}
        # the tensor-core form of the same graph, with its error vs FP64
        ttc = [F.Uneven(uneven_lengths(batch), measure=True, tensor_core=True)
               for _ in range(nsets)]
        for p in ttc:
            p.set_stream(stream)
        for i in range(3):
            step(i, pl=ttc)
        tms = time_steps(torch, stream, args.steps, lambda i: step(i, pl=ttc))
        ls = uneven_lengths(batch)
        offs = np.concatenate([[0], np.cumsum(ls)])
        errs = []
        o = sets[(args.steps - 1) % nsets][1]
        yr, yi = o[0].cpu().numpy(), o[1].cpu().numpy()
        for j in range(0, len(ls), max(1, len(ls) // 16)):  # every size class
            a, b = offs[j], offs[j + 1]
            want = np.fft.fft(host_in[0][a:b].astype(np.float64) + 1j * host_in[1][a:b])
            got = yr[a:b] + 1j * yi[a:b]
            errs.append(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
        plain["tensor_core_form"] = {"value": round(nbytes / (tms * 1e-3) / 1e9, 1),
                                     "ms_per_step": round(tms, 4),
                                     "speedup_over_plain": round(pms / tms, 3),
                                     "max_rel_l2_vs_fp64": max(errs),
                                     "sample": f"{len(errs)} transforms across the lengths"}
        # latency of one whole uneven batch, step by step, for the three methods
        nlat = max(args.steps, 100)
        plain["latency_per_batch"] = {
            "persistent_graph": step_latencies(torch, stream, nlat, lambda i: step(i)),
            "tensor_core_graph": step_latencies(torch, stream, nlat, lambda i: step(i, pl=ttc)),
            "plain_one_launch_per_length": step_latencies(torch, stream, nlat,
                                                           lambda i: step(i, plain=True))}
        for p in ttc:
            p.close()

    if workload == "c2c16384tc":
        # accuracy of the tensor-core form on a sample, and the plain CUDA-core
        # path on the same data
        acc = dict(check or {})
        acc["tc_status"] = t.tc_status()
        tp = F.Transform.fft(n)
        tp.set_stream(stream)
        for i in range(3):
            step(i, pl=[tp])
        pms = time_steps(torch, stream, args.steps, lambda i: step(i, pl=[tp]))
        plain = {"value": round(nbytes / (pms * 1e-3) / 1e9, 1), "ms_per_step": round(pms, 4),
                 "speedup_of_tensor_core_form": round(pms / ms_per_step, 3)}
        # the radix-16 tensor-core kernels on the same data
        os.environ["FAF_CUDA_TC_RADIX"] = "16"
        try:
            t16 = F.Transform.fft(n, flags=F.FLAG_TENSOR_CORE)
        finally:
            del os.environ["FAF_CUDA_TC_RADIX"]
        t16.set_stream(stream)
        for i in range(3):
            step(i, pl=[t16])
        ms16 = time_steps(torch, stream, args.steps, lambda i: step(i, pl=[t16]))
        plain["radix16_tensor_core_form"] = {
            "value": round(nbytes / (ms16 * 1e-3) / 1e9, 1), "ms_per_step": round(ms16, 4),
            "kernel": "k2_c2c_tc", "tc_status": t16.tc_status()}
        t16.close()
        # two stages x two M=128 tiles x 8 K steps x 3 products of 128x128x16
        tflops = batch * 2 * 2 * 8 * 3 * 2 * 128 * 128 * 16 / (ms_per_step * 1e-3) / 1e12
        acc["tensor_tflops"] = round(tflops, 1)
        acc["plan_kind"] = t.kind
        tp.close()

    peak, peak_kind = measured_hbm_peak()
    r2c = None
    if workload == "pipeline" and not args.no_r2c:
        r2c = r2c_subrecord(F, torch, stream, sets, host_in, args.steps, peak)

    # end to end through the public API with pinned host buffers
    host_pinned = [torch.from_numpy(a).pin_memory().numpy() for a in host_in]
    host_out = alloc_outputs(workload, batch, host_pinned[0], torch)
    t_e2e = build_transform(F, workload, torch)
    for _ in range(2):
        run_step(F, t_e2e, workload, host_pinned, host_out)
    e2e_steps = max(2, min(args.steps, 10))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run_step(F, t_e2e, workload, host_pinned, host_out)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, dist, "cuda")
    h2d = sum(a.nbytes for a in host_pinned)
    d2h = sum(a.nbytes for a in host_out)
    e2e_value = world * nbytes / e2e_s / 1e9

    achieved = nbytes / (ms_per_step * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": ncu_traffic(workload),
                "algorithmic_bytes_per_launch": nbytes,
                "kernel": {"pipeline": "k2_pipeline", "r2c": "k2_r2c", "stft": "k2_stft",
                           "uneven": "k4p_col (65536-point class, column pass; traffic of one "
                                     "128-transform chunk)",
                           "c2c16384": "k2_c2c_land", "c2c4096": "k2_c2c_land",
                           "c2c16384tc": "k2_c2c_tc64",
                           "c2c4096fp64": "k64_c2c", "istft": "k2_c2r + k_ola",
                           "cwt": "k2_c2r (bank rows) + k2_r2c",
                           "icwt": "k2_r2c (rows) + k_icwt_acc + k2_c2r"}.get(
                               workload, "k2_c2c")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(workload, host_in, seconds=args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": "FFT GB/s (%HBM peak)",
            "value": round(value, 1),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": round(ms_per_step, 5),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if workload == "c2c4096fp64" else "f32",
            "data": "synthetic (seeded numpy PCG64)",
            "config": {"workload": desc, "n": n, "batch_per_gpu": batch,
                       "parallelism": f"replicas{world}",
                       "l2": (f"rotates over {nsets} input/output buffer sets of "
                              f"{nbytes / 2**20:.0f} MiB (together > 2 x the 126 MB L2): no step "
                              "reads data the previous step left in L2")
                       if nsets > 1 else "L2-resident working set (launch-bound)"},
            "pct_hbm_peak": round(100 * achieved / peak, 2),
            "gflops_5nlog2n": round(world * batch * flops_per / (ms_per_step * 1e-3) / 1e9, 1)
            if flops_per else None,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_s * 1e3, 3),
                    "api": "faf_execute_batched with pinned host buffers"},
            "gpu_launches": launches,
            "clocks": sampler.result(),
            "output_check": check,
            "wait_status": wait,
        }
        if r2c is not None:
            line["r2c"] = r2c
        if plain is not None and workload == "uneven":
            line["plain_one_launch_per_length"] = plain
        elif plain is not None:
            line["plain_cuda_core_path"] = plain
            line["accuracy"] = acc
        print(json.dumps(line), flush=True)
    for p in plans:
        p.close()
    t_e2e.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# reference (CPU) arm
# ---------------------------------------------------------------------------

def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class RefRunner:
    """The reference library's CPU path for one workload, planned once:
    persistent worker threads, each with its own transform created and
    warmed (the pipeline JIT compiled) at construction, so run() times only
    faf_execute calls over the whole batch (the reference's own benchmarks
    plan once and execute in a loop, benchmarks/benchmark_throughput.cpp:34-39).
    The inverse STFT has no reference counterpart: the oracle's FP64 numpy
    restatement stands in for it, on one core."""

    def __init__(self, refimpl, workload, host_in, threads):
        self.workload, self.host_in = workload, host_in
        n = WORKLOADS[workload][1]
        self.sessions = []
        S = refimpl.Session
        if workload == "pipeline":
            m = notch_mask(n)
            self.sessions = [S("pipeline", n, threads,
                               src=f"(pipeline (rfft :size {n}) (mul-spectrum) (irfft))",
                               h=(m, np.zeros_like(m)))]
        elif workload == "r2c":
            self.sessions = [S("r2c", n, threads)]
        elif workload == "c2c4096fp64":
            self.sessions = [S("c2c64", n, threads)]
        elif workload.startswith("c2c"):
            self.sessions = [S("c2c", n, threads)]
        elif workload == "stft":
            self.sessions = [S("stft", 1024, threads, win=1024, hop=256,
                               sig_len=host_in[0].shape[-1])]
        elif workload == "cwt":
            self.sessions = [S("cwt", n, threads)]
        elif workload == "icwt":
            self.sessions = [S("icwt_dual", n, threads)]
        elif workload == "uneven":
            ls = uneven_lengths(WORKLOADS["uneven"][2])
            self.runs = []  # (session, offset, count) per run of equal lengths
            off, i = 0, 0
            while i < len(ls):
                j = i
                while j < len(ls) and ls[j] == ls[i]:
                    j += 1
                sess = S("c2c", ls[i], threads)
                self.sessions.append(sess)
                self.runs.append((sess, off, j - i))
                off += ls[i] * (j - i)
                i = j
        elif workload != "istft":
            raise ValueError(workload)
        self.threads = self.sessions[0].threads if self.sessions else 1
        self.outs = self._outputs(host_in)

    def _outputs(self, host_in):
        w = self.workload
        if w == "pipeline":
            return [np.empty_like(host_in[0])]
        if w == "r2c":
            shp = host_in[0].shape[:-1] + (host_in[0].shape[-1] // 2 + 1,)
            return [np.empty(shp, np.float32), np.empty(shp, np.float32)]
        if w.startswith("c2c") or w == "uneven":
            return [np.empty_like(host_in[0]), np.empty_like(host_in[1])]
        if w == "stft":
            F_, bins = stft_geometry(host_in[0].shape[-1])
            return [np.empty((host_in[0].shape[0], F_, 513), np.float32) for _ in range(2)]
        if w == "cwt":
            from oracle import refimpl
            r = refimpl.cwt_bank(WORKLOADS[w][1])[0].shape[0]
            return [np.empty(host_in[0].shape[:-1] + (r, host_in[0].shape[-1]), np.float32)]
        if w == "icwt":
            return [np.empty(host_in[0].shape[:-2] + (host_in[0].shape[-1],), np.float32)]
        return []

    def run(self, count=None):
        """One pass over the first `count` transforms (signals) of the
        workload (the whole batch by default)."""
        w, x, o = self.workload, self.host_in, self.outs
        if w == "istft":
            from oracle import orc
            c = count or 2
            orc.istft(x[0][:c], x[1][:c], 1024, 1024, 256)
            return
        if w == "uneven":
            for sess, off, cnt in self.runs:
                sess.run(cnt, x[0][off:], x[1][off:], o[0][off:], o[1][off:])
            return
        b = count or x[0].shape[0]
        s = self.sessions[0]
        if w in ("pipeline", "cwt", "icwt"):
            s.run(b, x[0], None, o[0], None)
        elif w in ("r2c", "stft"):
            s.run(b, x[0], None, o[0], o[1])
        else:
            s.run(b, x[0], x[1], o[0], o[1])

    def close(self):
        for s in self.sessions:
            s.close()


def _ref_open(workload, host_in, threads):
    from oracle import refimpl
    if not refimpl.available():
        refimpl.build()  # raises with the reason when the sources are absent
    return refimpl, RefRunner(refimpl, workload, host_in, threads)


def _bytes_of(workload, count):
    return algorithmic_bytes(workload, count) if workload != "uneven" else \
        algorithmic_bytes(workload, WORKLOADS["uneven"][2])


def cpu_baseline(workload, host_in, seconds=1.0, threads=None):
    """The reference library (oracle/_ref, built from its own sources) on the
    host cores, planned once: full-batch passes of the workload, repeated
    until `seconds` elapse, on all host threads; plus the same on one thread
    over one thread's share of the batch."""
    threads = threads or host_threads()
    try:
        refimpl, rr = _ref_open(workload, host_in, threads)
    except Exception as e:  # the prebuilt library did not travel
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": f"unavailable: {e}"}
    batch = WORKLOADS[workload][2]
    if workload == "istft":
        rr.run(2)
        reps, t0 = 0, time.perf_counter()
        while True:
            rr.run(2)
            reps += 1
            el = time.perf_counter() - t0
            if el >= seconds or reps >= 1000:
                break
        return {"value": round(reps * _bytes_of(workload, 2) / el / 1e9, 3), "unit": "GB/s",
                "cores": 1, "kind": "port",
                "sample": f"{reps} passes x 2 signals of the workload ({el:.1f} s, the oracle's "
                          "FP64 numpy restatement: the reference has no inverse STFT)"}
    for _ in range(5):  # warm-up passes, as the reference arm's default
        rr.run()
    reps, t0 = 0, time.perf_counter()
    while True:
        rr.run()
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds or reps >= 1000:
            break
    gbs = reps * _bytes_of(workload, batch) / el / 1e9
    rr.close()
    single = None
    if workload != "uneven":
        share = max(1, batch // threads)
        _, r1 = _ref_open(workload, host_in, 1)
        r1.run(share)
        reps1, t1 = 0, time.perf_counter()
        while True:
            r1.run(share)
            reps1 += 1
            el1 = time.perf_counter() - t1
            if el1 >= min(3.0, seconds / 3) or reps1 >= 1000:
                break
        r1.close()
        single = {"value": round(reps1 * _bytes_of(workload, share) / el1 / 1e9, 3),
                  "cores": 1, "sample": f"{reps1} passes x {share} transforms ({el1:.1f} s)"}
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "isa": refimpl.isa(),
            "sample": f"{reps} passes x the whole batch ({batch} transforms) of the workload "
                      f"({el:.1f} s); one faf_transform per thread, created and warmed "
                      "(pipeline JIT compiled) before timing",
            "single_core": single}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU path on the host cores over the
    same batch as our arm, each step one full pass, plans created and warmed
    before the timed steps.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    workload = args.workload
    desc, n, batch, _, _ = WORKLOADS[workload]
    host_in = make_inputs(workload, batch)
    threads = host_threads()
    try:
        refimpl, rr = _ref_open(workload, host_in, threads)
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference library missing: {e}"}))
        return
    count = 2 if workload == "istft" else None
    if workload == "istft":
        threads = 1
    for _ in range(max(args.warmup, 1)):
        rr.run(count)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rr.run(count)
        times.append(time.perf_counter() - t0)
    rr.close()
    s = sum(times) / len(times)
    nbytes = _bytes_of(workload, count or batch)
    gbs = nbytes / s / 1e9
    line = {
        "impl": "reference",
        "metric": "FFT GB/s (%HBM peak)",
        "value": round(gbs, 3),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(s * 1e3, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if workload == "c2c4096fp64" else "f32",
        "data": "synthetic (seeded numpy PCG64)",
        "config": {"workload": desc, "n": n, "batch_per_gpu": batch,
                   "parallelism": f"host cores ({threads} threads)"},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads,
                         "kind": "port" if workload == "istft" else "reference",
                         "isa": refimpl.isa(),
                         "sample": (f"{count or batch} of {batch} transforms per step, mean of "
                                    f"{args.steps} steps; plans created and warmed (pipeline JIT "
                                    "compiled) before the timed steps")},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving trace (continuous batching)
# ---------------------------------------------------------------------------

def serve_trace(F, n_req=4000, rate=20000.0, seed=4):
    """Request kinds, sizes and arrival times of the serving trace."""
    from fastandfourier_b200 import _lib as C
    rng = np.random.default_rng(seed)
    kinds = rng.choice(3, n_req, p=[0.4, 0.3, 0.3])
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    sizes = []
    for k in kinds:
        if k == 0:
            n = int(np.exp(rng.uniform(np.log(256), np.log(65536))))
            sizes.append(int(C.lib().faf_get_recommended_size(C.T_RFFT, n)))
        elif k == 1:
            sizes.append(4096)
        else:
            sizes.append(int(np.exp(rng.uniform(np.log(1 << 16), np.log(1 << 20)))))
    return kinds, sizes, arrivals


def build_serve_requests(F, torch, kinds, sizes, seed=4):
    """Device inputs (N(0,1) from a seeded device generator) and outputs."""
    nin = sum(sizes)
    nout = 0
    for k, n in zip(kinds, sizes):
        nout += 2 * (n // 2 + 1) if k == 0 else n if k == 1 else 2 * stft_geometry(n)[1]
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    xin = torch.randn(nin, device="cuda", generator=g)
    xout = torch.empty(nout, device="cuda")
    m = torch.from_numpy(notch_mask(4096)).cuda()
    z = torch.zeros_like(m)
    h = (m, z, 2049)
    reqs, algo = [], 0
    io = oo = 0
    pipe = "(pipeline (rfft :size 4096) (mul-spectrum) (irfft))"
    for k, n in zip(kinds, sizes):
        x = xin[io:io + n]
        io += n
        if k == 0:
            nb = n // 2 + 1
            o_re, o_im = xout[oo:oo + nb], xout[oo + nb:oo + 2 * nb]
            oo += 2 * nb
            reqs.append(F.Request(x, o_re, o_im, chirp=f"(rfft :size {n})"))
            algo += 4 * n + 8 * nb
        elif k == 1:
            o = xout[oo:oo + n]
            oo += n
            reqs.append(F.Request(x, o, chirp=pipe, h=h))
            algo += 8 * n
        else:
            bins = stft_geometry(n)[1]
            o_re, o_im = xout[oo:oo + bins], xout[oo + bins:oo + 2 * bins]
            oo += 2 * bins
            reqs.append(F.Request(x, o_re, o_im, stft=(1024, 1024, 256)))
            algo += 4 * n + 8 * bins
    return reqs, algo, (xin, xout, m, z)


def serve_once(F, reqs, arrivals, *, streams, max_merge, budget=16 << 30):
    srv = F.Server(hbm_budget=budget, streams=streams, max_merge=max_merge)
    seen = set()
    for r in reqs:  # plans (device tables) created ahead of the trace
        key = (r.struct.chirp, r.struct.stft_n)
        if key not in seen:
            seen.add(key)
            srv.prepare(r)
    srv.replay(reqs[:200], arrivals[:200] - arrivals[0])  # warm-up
    srv.reset_stats()
    lat = srv.replay(reqs, arrivals)
    st = srv.stats()
    srv.close()
    return st, lat


def run_serve(args, rank, world, local_rank):
    import torch
    import fastandfourier_b200 as F
    torch.cuda.set_device(local_rank)
    desc = WORKLOADS["serve"][0]
    kinds, sizes, arrivals = serve_trace(F, WORKLOADS["serve"][2])
    reqs, algo, keep = build_serve_requests(F, torch, kinds, sizes)
    torch.cuda.synchronize()
    sampler = ClockSampler(local_rank)
    with sampler:
        st, lat = serve_once(F, reqs, arrivals, streams=8, max_merge=64)
    plain, _ = serve_once(F, reqs, arrivals, streams=1, max_merge=1)

    def summary(s):
        return {"p50_ms": round(1e3 * s["p50_latency_s"], 3),
                "p99_ms": round(1e3 * s["p99_latency_s"], 3),
                "max_ms": round(1e3 * s["max_latency_s"], 3),
                "requests_per_s": round(s["requests_per_s"], 1),
                "GB_per_s": round(s["bytes_per_s"] / 1e9, 2),
                "launch_batches": s["batches"], "merged_requests": s["merged_requests"],
                "completed": s["completed"], "failed": s["failed"]}

    lat = np.asarray(lat)
    by_kind = {}
    for k, name in enumerate(("rfft", "pipeline", "stft")):
        v = lat[np.asarray(kinds) == k]
        if v.size:
            by_kind[name] = {"p50_ms": round(1e3 * float(np.percentile(v, 50)), 3),
                             "p99_ms": round(1e3 * float(np.percentile(v, 99)), 3)}
    if rank == 0:
        line = {
            "metric": "served GB/s at the trace's arrival rate",
            "value": round(st["bytes_per_s"] / 1e9, 2),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": 1,
            "warmup": 1,
            "ms_per_step": round(1e3 * st["wall_s"], 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded device N(0,1), Poisson arrivals)",
            "config": {"workload": desc, "requests": len(reqs), "algorithmic_bytes": algo,
                       "streams": 8, "max_merge": 64, "hbm_budget_bytes": 16 << 30},
            "latency": summary(st),
            "latency_by_kind": by_kind,
            "plain_one_request_at_a_time": summary(plain),
            "arena_peak_bytes": st["arena_peak_bytes"],
            "clocks": sampler.result(),
        }
        print(json.dumps(line), flush=True)
    del keep

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pipeline", choices=sorted(WORKLOADS))
    # about the reference arm's timed span (20 full-batch passes), so that the
    # two CPU figures see the same host clocks
    ap.add_argument("--cpu-seconds", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-r2c", action="store_true",
                    help="skip the R2C kernel-only sub-record of the pipeline line")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "WORLD_SIZE" not in os.environ:
        world = 1
    if args.workload == "serve":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no "
                                  "request loop; its CPU path is timed by the other workloads"}))
            return
        run_serve(args, rank, world, local_rank)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
