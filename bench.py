#!/usr/bin/env python
"""FX correlator throughput on B200: input Gsamp/s on one GPU and X-stage TFLOP/s.

Default workload (the geometry the headline metric is quoted on): 64 antennas x
1 polarisation x 8 subbands x 1024 channels (2048-point FFT), 0.5 s
subintegration = 31250 FFTs per subband at 128 MS/s, 2-bit real samples.
One step = one subintegration (all subbands) through the whole hot path:
delay table, fused unpack/shift/fringe/FFT/fractional-sample F stage, X stage.

  python bench.py [--gpus N --steps K --warmup W] [--xmode tc|plain] [--impl reference]

Under torchrun (N > 1) every rank correlates its own subintegration (weak
scaling, no data-path collective) and rank 0 prints one JSON line; time is the
max over ranks of CUDA-event time on the correlator's stream.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    "cfg2": dict(nant=64, npol=1, nchan=1024, nsb=8, numffts=31250, bw=64e6, lo=1.4e9, rho=0.1,
                 desc="64 ant x 1 pol x 8 subbands x 1024 ch, 0.5 s @ 128 MS/s (31250 FFTs/subband)"),
    "cfg1": dict(nant=16, npol=2, nchan=2048, nsb=4, numffts=31250, bw=64e6, lo=1.4e9, rho=0.05,
                 desc="16 ant x 2 pol x 4 subbands x 2048 ch, 1 s @ 128 MS/s (31250 FFTs/subband)"),
    "cfg0": dict(nant=4, npol=1, nchan=256, nsb=1, numffts=3125, bw=32e6, lo=1.4e9, rho=0.1,
                 desc="4 ant x 1 pol x 1 subband x 256 ch, 25 ms @ 64 MS/s (3125 FFTs)"),
    # profiling case: cfg2 geometry, 1 subband, 4096 FFTs (134 MB input > L2, ~1.2 GB on the device)
    "cfg2s": dict(nant=64, npol=1, nchan=1024, nsb=1, numffts=4096, bw=64e6, lo=1.4e9, rho=0.1,
                  desc="64 ant x 1 pol x 1 subband x 1024 ch, 4096 FFTs (profiling size)"),
}

METRIC = "input Gsamp/s on 1 GPU & X TFLOP/s: TC form vs FP32 plain at stated visibility error"
UNIT = "Gsamp/s"


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
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
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ data
def gen_device_data(torch, nsb, nant, npol, subint, pitch, rho, seed, device):
    """Seeded 2-bit data on the GPU: per subband a common N(0,1) signal (one per
    polarisation) with correlation rho plus independent N(0,1) noise, quantised at
    +-0.98 sigma and packed in the reference's bit order."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.zeros((nsb * nant, pitch), dtype=torch.uint8, device=device)
    nsamp = subint * 8 // (2 * npol)
    th = torch.tensor([-0.98, 0.0, 0.98], device=device)
    a, b = math.sqrt(rho), math.sqrt(1.0 - rho)
    for sb in range(nsb):
        common = torch.randn((npol, nsamp), generator=g, device=device)
        for ant in range(nant):
            x = a * common + b * torch.randn((npol, nsamp), generator=g, device=device)
            c = torch.bucketize(x, th).to(torch.uint8)
            if npol == 1:
                c = c[0].view(-1, 4)
                packed = c[:, 0] | (c[:, 1] << 2) | (c[:, 2] << 4) | (c[:, 3] << 6)
            else:
                c0 = c[0].view(-1, 2)
                c1 = c[1].view(-1, 2)
                packed = c0[:, 0] | (c1[:, 0] << 2) | (c0[:, 1] << 4) | (c1[:, 1] << 6)
            out[sb * nant + ant, : packed.numel()] = packed
    return out


def delay_model(nant, nchan, bw, seed):
    from difx_tests_b200 import synth
    rng = np.random.default_rng(seed)
    T_fft = 2 * nchan / (2 * bw)
    return synth.draw_delays(rng, nant, T_fft)


# ------------------------------------------------------------------ accuracy
def accuracy_sample(w, xmode):
    """max / RMS relative visibility error vs the FP64 oracle on a bounded sample
    of the workload's geometry (1 subband, 128 FFTs, full generator)."""
    import difx_tests_b200 as fx
    from difx_tests_b200 import synth
    from oracle import fxoracle as fo
    nf = 128
    job = synth.make_job(nant=w["nant"], npol=w["npol"], nchan=w["nchan"], numffts=nf, bw=w["bw"], lo=w["lo"],
                         rho=w["rho"], seed=1234)
    cfg = fx.make_config(job.nant, job.nchan, nf, job.bw, job.lo, npol=job.npol, xmode=xmode)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    ref, rc = fo.correlate(job.data[0], job.delays, job.fileoffsets, job.bw, job.lo, job.nchan, job.npol,
                           numffts=nf)
    mx, rms = fo.vis_error(vis[0], ref)
    return {"max_rel": float(mx.max()), "rms_rel": float(rms.max()), "vs": "FP64 oracle",
            "sample": f"1 subband x {nf} FFTs, {w['nant']} ant x {w['npol']} pol x {w['nchan']} ch",
            "counts_match": bool(np.array_equal(counts, rc))}


# ------------------------------------------------------------------ CPU reference
REF_GEOM = dict(nant=32, nchan=1024, bw=64e6, lo=1.4e9)   # 64 signals as 32 dual-pol antennas


def ref_workload_desc(nfft):
    return (f"reference kernel.c (+ IPP stand-in) on {REF_GEOM['nant']} ant x 2 pol (the reference's only input "
            f"format; 64 signals like the GPU workload) x {REF_GEOM['nchan']} ch, {nfft} FFTs")


def ref_run_shard(nfft, seed):
    """One bounded run of the reference CPU correlator; returns (seconds, samples)."""
    from difx_tests_b200 import synth
    from oracle import refcall
    g = REF_GEOM
    job = synth.random_job(nant=g["nant"], npol=2, nchan=g["nchan"], numffts=nfft, bw=g["bw"], lo=g["lo"],
                           seed=seed)
    t0 = time.perf_counter()
    refcall.run_reference(job.data[0], job.delays, job.fileoffsets, g["nchan"], nfft, g["bw"], g["lo"])
    dt = time.perf_counter() - t0
    return dt, g["nant"] * 2 * nfft * 2 * g["nchan"]


def _quiet_call(fn, *a):
    """Run fn with the C library's stdout (per-stage printf of kernel.c) discarded."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        return fn(*a)
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


def cpu_baseline_one_core(nfft=600):
    from oracle import refcall
    if not refcall.available():
        return None
    dt, samp = _quiet_call(ref_run_shard, nfft, 99)
    return {"value": samp / dt / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": ref_workload_desc(nfft) + f", 1 process, {dt:.1f} s"}


def ref_parallel_step(nproc, nfft_per_proc, seed):
    """All host cores: nproc forked processes over FFT shards (the reference's own
    split decomposition, main.c:398-408); each exits after its shard (kernel.c
    leaks ~75 KB per FFT x antenna)."""
    pipes = []
    t0 = time.perf_counter()
    for i in range(nproc):
        r, wfd = os.pipe()
        pid = os.fork()
        if pid == 0:
            os.close(r)
            try:
                dt, samp = _quiet_call(ref_run_shard, nfft_per_proc, seed + i)
                os.write(wfd, f"{dt} {samp}".encode())
            finally:
                os._exit(0)
        os.close(wfd)
        pipes.append((pid, r))
    total = 0
    for pid, r in pipes:
        data = b""
        while True:
            chunk = os.read(r, 256)
            if not chunk:
                break
            data += chunk
        os.close(r)
        os.waitpid(pid, 0)
        if data:
            total += int(float(data.split()[1]))
    return time.perf_counter() - t0, total


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import refcall
    w = WORKLOADS[args.workload]
    if not refcall.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfxref.so not built"}))
        return 0
    nproc = len(os.sched_getaffinity(0))
    # bound the leak: <= ~24 GB in flight over all processes
    per_call_kb = 75.0
    nfft = int(max(8, min(160, 24e6 / (nproc * REF_GEOM["nant"] * per_call_kb))))
    for _ in range(args.warmup):
        ref_parallel_step(nproc, nfft, 7)
    times, samples = [], []
    for k in range(args.steps):
        dt, s = ref_parallel_step(nproc, nfft, 1000 + 37 * k)
        times.append(dt)
        samples.append(s)
    tot = sum(times)
    val = sum(samples) / tot / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["desc"], "reference_sample": ref_workload_desc(nfft) + f" per process x {nproc}"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "reference",
                         "sample": f"{nproc} forked processes x {nfft} FFTs each per step"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU arm
def run_gpu_arm(args):
    import torch
    import torch.distributed as dist

    import difx_tests_b200 as fx

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    w = WORKLOADS[args.workload]
    xmode = fx.FXC_X_TC_FP16 if args.xmode == "tc" else fx.FXC_X_PLAIN_FP32
    F = 2 * w["nchan"]
    nsig = w["nant"] * w["npol"]
    cfg = fx.make_config(w["nant"], w["nchan"], w["numffts"], w["bw"], w["lo"], npol=w["npol"], nsubband=w["nsb"],
                         xmode=xmode)
    corr = fx.Correlator(cfg)
    subint = corr.subint_bytes
    dptr, pitch = corr.device_input()
    delays, offs = delay_model(w["nant"], w["nchan"], w["bw"], seed=42 + rank)
    data = gen_device_data(torch, w["nsb"], w["nant"], w["npol"], subint, pitch, w["rho"], seed=1000 + rank,
                           device=dev)
    # a dedicated (non-default) stream: the correlator's kernels and the timing
    # events are then ordered on the same stream
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    torch.cuda.synchronize()
    corr.set_stream(stream.cuda_stream)
    samples_per_step = w["nant"] * w["npol"] * w["nsb"] * w["numffts"] * F

    def step():
        corr.reset()
        corr.process_device(data.data_ptr(), pitch, delays, offs)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    corr.enable_stage_timing(True)
    corr.stage_times(reset=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    stage_ms, launches = corr.stage_times(reset=True)
    corr.enable_stage_timing(False)
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * samples_per_step * args.steps / (ms_max / 1e3) / 1e9

    # ---- roofline of the dominant kernel (per-launch averages over the timed region)
    hbm, tc_peak, peak_kind = peaks()
    f_launches = max(1, int(launches[1]))
    x_launches = max(1, int(launches[2]))
    f_ms = stage_ms[1] / f_launches
    x_ms = stage_ms[2] / x_launches
    T = corr_T = int(math.ceil(w["numffts"] / f_launches * args.steps))  # FFT slots per launch (approx.)
    ffts_per_launch = w["numffts"] * args.steps / f_launches
    in_bytes = nsig * w["nsb"] * ffts_per_launch * F / 4.0            # 2-bit packed input
    spec_bpc = 8 if xmode == fx.FXC_X_PLAIN_FP32 else 4                # bytes per complex spectrum value
    out_bytes = nsig * w["nsb"] * ffts_per_launch * w["nchan"] * spec_bpc
    f_gbs = (in_bytes + out_bytes) / (f_ms / 1e3) / 1e9
    x_flop = 8.0 * w["nchan"] * ffts_per_launch * w["nsb"] * nsig * (nsig + 1) / 2   # Hermitian incl. autos
    x_tflops = x_flop / (x_ms / 1e3) / 1e12
    if stage_ms[1] >= stage_ms[2] or xmode == fx.FXC_X_PLAIN_FP32:
        roof = {"kernel": "k_fstage (fused unpack/shift/fringe/FFT/frac)", "bound": "hbm", "achieved": f_gbs,
                "peak": hbm, "unit": "GB/s", "frac": f_gbs / hbm, "traffic": None,
                "peak_source": peak_kind, "share": stage_ms[1] / max(1e-9, stage_ms.sum())}
    else:
        roof = {"kernel": "k_xtc (tcgen05 X stage)", "bound": "tensor", "achieved": x_tflops, "peak": tc_peak,
                "unit": "TFLOP/s", "frac": x_tflops / tc_peak, "traffic": None, "peak_source": peak_kind,
                "share": stage_ms[2] / max(1e-9, stage_ms.sum())}
    del T, corr_T

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if xmode == fx.FXC_X_PLAIN_FP32 else "f32 F / f16 X",
        "data": "synthetic (seeded, on device)",
        "config": {"workload": w["desc"], "xmode": args.xmode, "parallelism": f"replicas x{world}",
                   "l2": "inputs (8.2 GB packed at cfg2) larger than L2; no flush",
                   "chunk_ffts": int(round(ffts_per_launch))},
        "stages_ms_per_step": {"delay+counts": stage_ms[0] / args.steps, "F": stage_ms[1] / args.steps,
                               "X": stage_ms[2] / args.steps},
        "x_stage": {"tflops": x_tflops, "flop_per_step": 8.0 * w["nchan"] * w["numffts"] * w["nsb"] * nsig *
                    (nsig + 1) / 2},
        "roofline": roof,
        "clocks": clk,
        "gpu_launches": int(launches.sum()),
    }

    # ---- end to end through the C ABI with pinned host buffers (rank-local)
    if not args.no_e2e:
        host = torch.empty((w["nsb"] * w["nant"], subint), dtype=torch.uint8, pin_memory=True)
        host.copy_(data[:, :subint])
        rows = host.numpy()
        vis_n = w["nsb"] * (w["nant"] * (w["nant"] - 1) // 2 + w["nant"]) * w["npol"] ** 2 * w["nchan"]
        e2e_steps = max(1, min(args.steps, 3))
        corr.process(rows.reshape(w["nsb"], w["nant"], subint), delays, offs)   # warm
        corr.visibilities()
        corr.reset()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            corr.reset()
            corr.process(rows.reshape(w["nsb"], w["nant"], subint), delays, offs)
            corr.visibilities()
        t = (time.perf_counter() - t0) / e2e_steps
        t_t = torch.tensor([t], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t_t, op=dist.ReduceOp.MAX)
        line["e2e"] = {"value": world * samples_per_step / float(t_t.item()) / 1e9, "unit": UNIT,
                       "h2d_bytes_per_step": int(w["nsb"] * w["nant"] * subint),
                       "d2h_bytes_per_step": int(vis_n * 8 + 4 * (w["nant"] * (w["nant"] + 1) // 2)),
                       "steps": e2e_steps, "ms_per_step": 1e3 * float(t_t.item())}

    if rank == 0 and not args.no_accuracy:
        line["accuracy"] = accuracy_sample(w, xmode)
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline_one_core()
        if cb is not None:
            line["cpu_baseline"] = cb
    corr.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS))
    ap.add_argument("--xmode", default="plain", choices=["plain", "tc"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
