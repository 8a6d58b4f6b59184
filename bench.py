#!/usr/bin/env python
"""FX correlator throughput on B200: input Gsamp/s on one GPU and X-stage TFLOP/s.

Default workload (the geometry the headline metric is quoted on): 64 antennas x
1 polarisation x 8 subbands x 1024 channels (2048-point FFT), 0.5 s
subintegration = 31250 FFTs per subband at 128 MS/s, 2-bit real samples.
One step = one subintegration (all subbands) through the whole hot path:
delay table, fused unpack/shift/fringe/FFT/fractional-sample F stage, X stage.

  python bench.py [--gpus N --steps K --warmup W] [--xmode all|both|tc|tc16f|fp8|plain] [--impl reference]

The headline `value` is the tensor-core form at FP32 F-stage accuracy: the FP32-grade
tensor-core F stage (k_ftc32: every operand an FP16 hi + lo pair, three products per GEMM,
FP32 accumulation; spectra held to the FP32 FFT's error bar), its spectra cast to FP16 for
the tcgen05 X stage with FP32 accumulation.  The same X form on the FP32 FFT F stage on the
CUDA cores ("tc"), on the FP16 tensor-core F stage ("tc16f"), the FP8-E4M3 tensor-core form
and the FP32 plain form run on the same input in the same invocation and are reported under
their names.  Geometries the tensor-core F stages do not cover (other than 1024 channels x
one polarisation) take "tc" as the headline.

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
    # profiling case: cfg1 geometry (4096-point FFTs, dual polarisation), 1 subband, 4096 FFTs
    "cfg1s": dict(nant=16, npol=2, nchan=2048, nsb=1, numffts=4096, bw=64e6, lo=1.4e9, rho=0.05,
                  desc="16 ant x 2 pol x 1 subband x 2048 ch, 4096 FFTs (profiling size)"),
    # profiling case: the cfg4 FFT (8192 points, dual polarisation) on 16 antennas, 1 subband, 2048 FFTs
    "cfg4s": dict(nant=16, npol=2, nchan=4096, nsb=1, numffts=2048, bw=64e6, lo=1.4e9, rho=0.05,
                  desc="16 ant x 2 pol x 1 subband x 4096 ch, 2048 FFTs (profiling size)"),
}

# Batched uneven workload: 12 independent jobs, antenna counts fixed, FFT length, subband count and
# subintegration length drawn (seed 3) from {256, 512, 1024, 4096, 8192} points, 1-8 subbands and
# 5-200 ms at 64 MS/s (32 MHz, single polarisation); per-job data seed 1000 + job.
BATCH_ANTS = [4, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 56]


def batch_jobs():
    rng = np.random.default_rng(3)
    jobs = []
    for j, a in enumerate(BATCH_ANTS):
        F = int(rng.choice([256, 512, 1024, 4096, 8192]))
        nsb = int(rng.integers(1, 9))
        dur = float(rng.uniform(5e-3, 200e-3))
        jobs.append(dict(nant=a, npol=1, nchan=F // 2, nsb=nsb, numffts=int(round(dur * 64e6 / F)), bw=32e6,
                         lo=1.4e9, rho=0.1, seed=1000 + j))
    return jobs


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
def accuracy_sample(w, xmode, fstage=0):
    """max / RMS relative visibility error vs the FP64 oracle on a bounded sample
    of the workload's geometry (1 subband, 128 FFTs, full generator)."""
    import difx_tests_b200 as fx
    from difx_tests_b200 import synth
    from oracle import fxoracle as fo
    nf = 128
    job = synth.make_job(nant=w["nant"], npol=w["npol"], nchan=w["nchan"], numffts=nf, bw=w["bw"], lo=w["lo"],
                         rho=w["rho"], seed=1234)
    cfg = fx.make_config(job.nant, job.nchan, nf, job.bw, job.lo, npol=job.npol, xmode=xmode, fstage=fstage)
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
# The reference reads only interleaved dual-polarisation input and needs a square channel count
# (kernel.c:31-35), so its sample of a workload keeps the workload's signal count as dual-pol
# antennas: 64 signals as 32 dual-pol antennas x 1024 ch for the cfg2 geometry (the default, also
# used for workloads the reference cannot run), the dual-pol variant of cfg0 (4 ant x 2 pol x 256 ch).
REF_GEOMS = {"cfg0": dict(nant=4, nchan=256, bw=32e6, lo=1.4e9, nfft=20000,
                          what="4 ant x 2 pol (the P=2 variant of this workload)"),
             "default": dict(nant=32, nchan=1024, bw=64e6, lo=1.4e9, nfft=600,
                             what="32 ant x 2 pol (the reference's only input format; 64 signals like the GPU "
                                  "workload)")}
REF_GEOM = REF_GEOMS["default"]


def ref_geom_for(workload):
    global REF_GEOM
    REF_GEOM = REF_GEOMS.get(workload, REF_GEOMS["default"])
    return REF_GEOM


def ref_workload_desc(nfft):
    return f"reference kernel.c (+ IPP stand-in) on {REF_GEOM['what']} x {REF_GEOM['nchan']} ch, {nfft} FFTs"


def ref_run_shard(nfft, seed, hoisted=False):
    """One bounded run of the reference CPU correlator (as written, or with allocKernel hoisted
    out of its FFT x antenna loop); returns (seconds, samples)."""
    from difx_tests_b200 import synth
    from oracle import refcall
    g = REF_GEOM
    job = synth.random_job(nant=g["nant"], npol=2, nchan=g["nchan"], numffts=nfft, bw=g["bw"], lo=g["lo"],
                           seed=seed)
    t0 = time.perf_counter()
    refcall.run_reference(job.data[0], job.delays, job.fileoffsets, g["nchan"], nfft, g["bw"], g["lo"],
                          hoisted=hoisted)
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


def cpu_baseline_one_core(nfft=None):
    from oracle import refcall
    if not refcall.available():
        return None
    nfft = nfft or REF_GEOM["nfft"]
    dt, samp = _quiet_call(ref_run_shard, nfft, 99)
    out = {"value": samp / dt / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
           "sample": ref_workload_desc(nfft) + f", 1 process, {dt:.1f} s"}
    if refcall.available(hoisted=True):
        dh, sh = _quiet_call(ref_run_shard, nfft, 99, True)
        out["allockernel_hoisted"] = {"value": sh / dh / 1e9, "unit": UNIT, "cores": 1,
                                      "sample": "the same, kernel.c with allocKernel moved out of its FFT x antenna "
                                                f"loop (kernel.c:727-728), {dh:.1f} s"}
    return out


def ref_parallel_step(nproc, nfft_per_proc, seed, hoisted=False):
    """All host cores: nproc forked processes over FFT shards (the reference's own
    split decomposition, main.c:398-408); each exits after its shard (kernel.c
    leaks ~75 KB per FFT x antenna unless allocKernel is hoisted)."""
    pipes = []
    t0 = time.perf_counter()
    for i in range(nproc):
        r, wfd = os.pipe()
        pid = os.fork()
        if pid == 0:
            os.close(r)
            try:
                dt, samp = _quiet_call(ref_run_shard, nfft_per_proc, seed + i, hoisted)
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
    ref_geom_for(args.workload)
    if not refcall.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfxref.so not built"}))
        return 0
    # load the reference library in this process too (the forked children inherit the mapping)
    refcall.lib()
    hoisted = refcall.available(hoisted=True)
    if hoisted:
        refcall.lib(hoisted=True)
    nproc = len(os.sched_getaffinity(0))
    # bound the leak: <= ~24 GB in flight over all processes
    per_call_kb = 75.0
    nfft = int(max(8, min(160 * 32 // REF_GEOM["nant"], 24e6 / (nproc * REF_GEOM["nant"] * per_call_kb))))
    for _ in range(args.warmup):
        ref_parallel_step(nproc, nfft, 7)
    times, samples = [], []
    for k in range(args.steps):
        dt, s = ref_parallel_step(nproc, nfft, 1000 + 37 * k)
        times.append(dt)
        samples.append(s)
    tot = sum(times)
    val = sum(samples) / tot / 1e9
    extra = {}
    if hoisted:
        # the secondary figure: kernel.c with allocKernel hoisted out of its FFT x antenna loop
        ref_parallel_step(nproc, nfft, 7, True)
        th, sh = [], []
        for k in range(args.steps):
            dt, s_ = ref_parallel_step(nproc, nfft, 1000 + 37 * k, True)
            th.append(dt)
            sh.append(s_)
        extra["allockernel_hoisted"] = {
            "value": sum(sh) / sum(th) / 1e9, "unit": UNIT, "cores": nproc,
            "ms_per_step": 1e3 * sum(th) / args.steps,
            "sample": f"as the headline, kernel.c with allocKernel moved out of its FFT x antenna loop "
                      f"(kernel.c:727-728; oracle/hoist_allockernel.py), {nproc} processes x {nfft} FFTs"}
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["desc"], "reference_sample": ref_workload_desc(nfft) + f" per process x {nproc}"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "reference",
                         "sample": f"{nproc} forked processes x {nfft} FFTs each per step"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line.update(extra)
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU arm
# DRAM bytes per input sample of the F-stage kernels (2048-point FFTs), dram__bytes_read.sum +
# dram__bytes_write.sum from one ncu capture each on the 64-antenna x 1024-channel profiling case,
# divided by the samples of that launch: key (fstage, F16 output)
# (profiles/kernels_cfg2s_ncu_full.txt for k_fstage, profiles/k_ftc_cfg2s_ncu.txt for k_ftc,
# profiles/k_ftc32_cfg2s_ncu.txt for k_ftc32).
FSTAGE_DRAM_BYTES_PER_SAMPLE = {(1, True): 2.17, (1, False): 4.16, (2, True): 2.17, (3, True): 2.18}


# form -> (fxc_config.xmode, fxc_config.fstage)
FORMS = {"plain": (0, 1),     # FXC_X_PLAIN_FP32, FXC_F_FFT32
         "tc": (1, 1),        # FXC_X_TC_FP16 on the FP32 FFT F stage
         "tc16f": (1, 2),     # FXC_X_TC_FP16 on the FP16 tensor-core F stage (FXC_F_TC16)
         "tc32f": (1, 3),     # FXC_X_TC_FP16 on the FP32-grade tensor-core F stage (FXC_F_TC32), the headline
         "fp8": (2, 1)}       # FXC_X_TC_FP8 on the FP32 FFT F stage
XMODES = {k: v[0] for k, v in FORMS.items()}
DTYPES = {"plain": "f32 (FFT F stage and X stage on the CUDA cores)",
          "tc": "f32 FFT F stage (CUDA cores), spectra cast to f16 for the tensor-core X stage, f32 accumulate",
          "tc16f": "f16 tensor-core F stage (k_ftc: f16 DFT matrices and intermediate), f16 X inputs, "
                   "f32 accumulate",
          "tc32f": "f32-grade tensor-core F stage (k_ftc32: f16 hi+lo operand pairs, three products per GEMM, "
                   "f32 accumulate), spectra cast to f16 for the tensor-core X stage, f32 accumulate",
          "fp8": "f32 FFT F stage (CUDA cores), spectra cast to e4m3 scaled per signal and channel for the "
                 "tensor-core X stage, f32 accumulate"}
F_KERNELS = {1: "k_fstage (fused unpack/shift/fringe/FFT/frac-delay, FP32 radix-16 FFT on the CUDA cores)",
             2: "k_ftc (tcgen05 F stage: unpack/fringe, 32x64 DFT as two FP16 tensor-core GEMMs, twiddles, "
                "frac-delay, F16 store)",
             3: "k_ftc32 (tcgen05 F stage, FP32-grade: 32x64 DFT as two tensor-core GEMMs on FP16 hi+lo pairs, "
                "three products each, twiddles, frac-delay)"}


def tcf_geometry(w):
    """The tensor-core F stages cover 1024 channels x 1 polarisation (2048-point real FFTs)."""
    return w["nchan"] == 1024 and w["npol"] == 1


def form_params(form, w):
    """(xmode, fstage) of a form on workload w: a tensor-core F stage falls back to the FP32 FFT where
    the geometry is not covered."""
    xmode, fstage = FORMS[form]
    if fstage in (2, 3) and not tcf_geometry(w):
        fstage = 1
    return xmode, fstage


def spectra_f16(xmode, fstage, w):
    """Whether the F stage writes the FP16 K-major spectra layout: the tensor-core forms, except the
    FP16 form on the FFT F stage at up to 64 signals and a multiple of 4 channels, whose X stage
    reads FP32 spectra and casts them itself (the library's rule, fx_api.cu ctx_create)."""
    import difx_tests_b200 as fx
    if xmode == fx.FXC_X_PLAIN_FP32:
        return False
    return not (xmode == fx.FXC_X_TC_FP16 and fstage in (0, 1) and w["nant"] * w["npol"] <= 64
                and w["nchan"] % 4 == 0 and os.environ.get("FXC_TC_SPECTRA") != "f16")


def form_dtype(form, w):
    """dtype label of the form as it runs on w (a tensor-core F form that fell back reads as tc)."""
    return DTYPES[form] if form_params(form, w) == FORMS[form] else DTYPES["tc"]


def select_forms(xmode, w):
    """Forms to time, the headline first: all -> tc32f, tc, tc16f, fp8, plain; both -> tc32f, plain;
    a form name -> that form.  Geometries the tensor-core F stages do not cover (other than
    1024 channels x 1 polarisation) take the tc form in their place."""
    forms = {"all": ["tc32f", "tc", "tc16f", "fp8", "plain"], "both": ["tc32f", "plain"]}.get(xmode, [xmode])
    if not tcf_geometry(w):
        forms = list(dict.fromkeys("tc" if f in ("tc16f", "tc32f") else f for f in forms))
    return forms


def time_form(torch, dist, fx, w, form, data, pitch, delays, offs, steps, warmup, world, dev, stream):
    """Warm up, then time `steps` subintegrations of one form; returns a result dict."""
    F = 2 * w["nchan"]
    nsig = w["nant"] * w["npol"]
    xmode, fstage = form_params(form, w)
    cfg = fx.make_config(w["nant"], w["nchan"], w["numffts"], w["bw"], w["lo"], npol=w["npol"], nsubband=w["nsb"],
                         xmode=xmode, fstage=fstage)
    corr = fx.Correlator(cfg)
    corr.set_stream(stream.cuda_stream)
    samples = w["nant"] * w["npol"] * w["nsb"] * w["numffts"] * F

    def step():
        corr.reset()
        corr.process_device(data.data_ptr(), pitch, delays, offs)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    corr.enable_stage_timing(True)
    corr.stage_times(reset=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    stage_ms, launches = corr.stage_times(reset=True)
    corr.enable_stage_timing(False)
    from difx_tests_b200 import sharding
    ms_max = sharding.max_over_ranks(ms, device=dev)   # device time: max over ranks
    f_launches = max(1, int(launches[1]))
    x_launches = max(1, int(launches[2]))
    ffts_per_launch = w["numffts"] * steps / f_launches
    samples_per_launch = nsig * w["nsb"] * ffts_per_launch * F
    x_flop_step = 8.0 * w["nchan"] * w["numffts"] * w["nsb"] * nsig * (nsig + 1) / 2   # Hermitian incl. autos
    return dict(corr=corr, cfg=cfg, ms_max=ms_max, value=world * samples * steps / (ms_max / 1e3) / 1e9,
                stage_ms=stage_ms, launches=launches, clocks=clk, samples=samples,
                f_ms_launch=stage_ms[1] / f_launches, x_ms_launch=stage_ms[2] / x_launches,
                samples_per_launch=samples_per_launch, ffts_per_launch=ffts_per_launch,
                x_tflops=x_flop_step * steps / (stage_ms[2] / 1e3) / 1e12, x_flop_step=x_flop_step)


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
    F = 2 * w["nchan"]
    nsig = w["nant"] * w["npol"]
    probe = fx.make_config(w["nant"], w["nchan"], w["numffts"], w["bw"], w["lo"], npol=w["npol"], nsubband=w["nsb"])
    subint = fx.lib().fxc_subint_bytes(probe)
    pitch = (subint + 16 + 255) // 256 * 256
    delays, offs = delay_model(w["nant"], w["nchan"], w["bw"], seed=42 + rank)
    # a dedicated (non-default) stream: the correlator's kernels and the timing events share it
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    data = gen_device_data(torch, w["nsb"], w["nant"], w["npol"], subint, pitch, w["rho"], seed=1000 + rank,
                           device=dev)
    torch.cuda.synchronize()

    forms = select_forms(args.xmode, w)
    res, failed = {}, {}
    for form in forms:
        try:
            res[form] = time_form(torch, dist, fx, w, form, data, pitch, delays, offs, args.steps, args.warmup, world,
                                  dev, stream)
        except fx.FxcError as e:
            if form == forms[0]:
                raise
            failed[form] = str(e)      # recorded in the line; the other forms still run
            continue
        if form != forms[0]:
            res[form]["corr"].close()
    forms = [f for f in forms if f in res]
    head = res[forms[0]]
    xmode, fstage = form_params(forms[0], w)

    # ---- roofline of the dominant kernel of the headline form (the F stage)
    hbm, tc_peak, peak_kind = peaks()
    f16 = spectra_f16(xmode, fstage, w)
    spec_bpc = 4 if f16 else 8       # bytes per complex spectrum value written
    f_bytes = head["samples_per_launch"] * (0.25 + 0.5 * spec_bpc)
    f_gbs = f_bytes / (head["f_ms_launch"] / 1e3) / 1e9
    sm = head["stage_ms"]
    dram = FSTAGE_DRAM_BYTES_PER_SAMPLE.get((fstage, f16)) if w["nchan"] == 1024 else None
    roof = {"kernel": F_KERNELS[fstage] + (", FP16 spectra out" if f16 else ", FP32 spectra out"),
            "bound": "hbm", "achieved": f_gbs,
            "peak": hbm, "unit": "GB/s", "frac": f_gbs / hbm,
            "traffic": dram * head["samples_per_launch"] if dram else None,
            "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_launch": f_bytes, "launch_ms": head["f_ms_launch"],
            "share": sm[1] / max(1e-9, sm.sum()),
            "note": ("latency-bound warp-specialised pipeline; HBM fraction shown for its algorithmic bytes"
                     if fstage in (2, 3) else
                     "FP32 FFT is issue-bound on the CUDA cores; HBM fraction shown for its algorithmic bytes")}

    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_max"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": form_dtype(forms[0], w),
        "data": "synthetic (seeded, generated on device)",
        "config": {"workload": w["desc"], "form": forms[0], "parallelism": f"replicas x{world}",
                   "l2": "inputs (8.2 GB packed per step at cfg2) exceed L2; no flush",
                   "chunk_ffts": int(round(head["ffts_per_launch"]))},
        "stages_ms_per_step": {"delay+counts": sm[0] / args.steps, "F": sm[1] / args.steps,
                               "X": sm[2] / args.steps},
        "x_stage": {"tflops": head["x_tflops"], "flop_per_step": head["x_flop_step"],
                    "ms_per_step": sm[2] / args.steps},
        "roofline": roof,
        "clocks": head["clocks"],
        "gpu_launches": int(head["launches"].sum()),
    }
    for form in forms[1:]:
        p = res[form]
        line[form] = {"value": p["value"], "unit": UNIT, "ms_per_step": p["ms_max"] / args.steps, "dtype": form_dtype(form, w),
                      "stages_ms_per_step": {"F": p["stage_ms"][1] / args.steps, "X": p["stage_ms"][2] / args.steps},
                      "x_tflops": p["x_tflops"], "clocks": p["clocks"], "gpu_launches": int(p["launches"].sum())}
    if "plain" in res and forms[0] != "plain":
        p = res["plain"]
        line["tc_vs_plain"] = {"gsamps": head["value"] / p["value"],
                               "x_stage_only": (p["stage_ms"][2] / max(1e-9, sm[2])),
                               "form": forms[0]}
        # the other forms' ratios, by form name (the headline's is tc_vs_plain above)
        line["forms_vs_plain"] = {
            f: {"gsamps": res[f]["value"] / p["value"],
                "x_stage_only": p["stage_ms"][2] / max(1e-9, res[f]["stage_ms"][2])}
            for f in ("tc32f", "tc", "tc16f", "fp8") if f in res and f != forms[0]}

    corr = head["corr"]
    # ---- end to end through the C ABI with pinned host buffers (rank-local)
    if not args.no_e2e:
        host = torch.empty((w["nsb"] * w["nant"], subint), dtype=torch.uint8, pin_memory=True)
        host.copy_(data[:, :subint])
        torch.cuda.synchronize()
        rows = host.numpy().reshape(w["nsb"], w["nant"], subint)
        vis_n = w["nsb"] * (w["nant"] * (w["nant"] - 1) // 2 + w["nant"]) * w["npol"] ** 2 * w["nchan"]
        e2e_steps = max(1, min(args.steps, 3))
        vis_host = torch.empty(2 * vis_n, dtype=torch.float32, pin_memory=True).numpy()   # pinned read-back
        corr.process(rows, delays, offs)   # warm
        corr.visibilities(out=vis_host)
        torch.cuda.synchronize()
        # CUDA events on the correlator's stream around host-buffer calls: copies (on the library's
        # copy stream, ordered by events), compute and the read-back all fall inside
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(e2e_steps):
            corr.reset()
            corr.process(rows, delays, offs)
            corr.visibilities(out=vis_host)
        ev1.record(stream)
        torch.cuda.synchronize()
        t = ev0.elapsed_time(ev1) / 1e3 / e2e_steps
        from difx_tests_b200 import sharding
        t_max = sharding.max_over_ranks(t, device=dev)
        line["e2e"] = {"value": world * head["samples"] / t_max / 1e9, "unit": UNIT,
                       "h2d_bytes_per_step": int(w["nsb"] * w["nant"] * subint),
                       "d2h_bytes_per_step": int(vis_n * 8 + 4 * (w["nant"] * (w["nant"] - 1) // 2 + w["nant"])),
                       "steps": e2e_steps, "ms_per_step": 1e3 * t_max,
                       "path": "fxc_process_host + fxc_get_visibilities, pinned host input and output buffers"}

    for f, msg in failed.items():
        line[f] = {"error": msg}
    if rank == 0 and not args.no_accuracy:
        line["accuracy"] = {f: accuracy_sample(w, *form_params(f, w)) for f in forms}
    if rank == 0 and world == 1 and not args.no_cpu:
        ref_geom_for(args.workload)
        cb = cpu_baseline_one_core()
        if cb is not None:
            line["cpu_baseline"] = cb
    corr.close()
    if rank == 0 and world == 1 and args.workload == "cfg2" and not args.no_extra:
        # bounded runs of the batched (cfg3) and large-array (cfg4) workloads, each with its own
        # clocks and accuracy, recorded beside the headline
        del data, res, head
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = 3, 3
        line["cfg3"] = run_batch_arm(sub, emit=False)
        torch.cuda.empty_cache()
        sub.steps, sub.warmup = 2, 1
        line["cfg4"] = run_large_arm(sub, emit=False, max_windows=2)
        # configs 1 and 0 (their own processes: fresh device memory, their own clocks)
        line["cfg1"] = sub_bench(["--workload", "cfg1", "--xmode", "both", "--steps", "3", "--warmup", "3"])
        line["cfg0"] = sub_bench(["--workload", "cfg0", "--xmode", "plain", "--steps", "10", "--warmup", "3"])
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def sub_bench(argv):
    """One bounded bench.py run of another workload in a child process -> its JSON line (or the
    error), recorded beside the headline."""
    cmd = [sys.executable, os.path.abspath(__file__), *argv, "--no-extra", "--no-cpu"]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode == 0 and lines:
            return json.loads(lines[-1])
        return {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}"}
    except (subprocess.TimeoutExpired, ValueError) as e:
        return {"error": str(e)[:300]}


def run_shard_arm(args):
    """One subintegration of the workload split over the ranks (strong scaling): "time" shards
    (each rank a range of FFTs of every subband, one all-reduce of visibilities and counts) or
    "subband" shards (each rank whole subbands, one all-gather), correlated through the library
    and merged inside the timed step (NCCL on the device).  Time = max over ranks of CUDA-event
    time on each rank's stream."""
    import torch
    import torch.distributed as dist

    import difx_tests_b200 as fx
    from difx_tests_b200 import sharding

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    w = WORKLOADS[args.workload]
    sform = args.xmode if args.xmode in FORMS else ("tc32f" if w["nchan"] == 1024 and w["npol"] == 1 else "tc")
    xmode, fstage = form_params(sform, w)
    cfg = fx.make_config(w["nant"], w["nchan"], w["numffts"], w["bw"], w["lo"], npol=w["npol"], nsubband=w["nsb"],
                         xmode=xmode, fstage=fstage)
    subint = fx.lib().fxc_subint_bytes(cfg)
    pitch = (subint + 16 + 255) // 256 * 256
    delays, offs = delay_model(w["nant"], w["nchan"], w["bw"], seed=42)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    data = gen_device_data(torch, w["nsb"], w["nant"], w["npol"], subint, pitch, w["rho"], seed=1000, device=dev)
    rcfg, f0, n, s0 = sharding.shard_config(fx, cfg, args.shard, world, rank)
    corr = fx.Correlator(rcfg)
    corr.set_stream(stream.cuda_stream)

    def step():
        return sharding.correlate_shard(fx, corr, args.shard, data.data_ptr(), pitch, delays, offs, f0, n, s0,
                                        w["nsb"], dev)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sharding.max_over_ranks(e0.elapsed_time(e1) / args.steps, device=dev)
    samples = w["nant"] * w["npol"] * w["nsb"] * w["numffts"] * 2 * w["nchan"]
    corr.close()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": samples / (ms / 1e3) / 1e9, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": form_dtype(sform, w),
            "data": "synthetic (seeded, generated on device)",
            "config": {"workload": w["desc"], "parallelism": f"{args.shard} shards x{world}",
                       "merge": "all-reduce of visibilities and counts" if args.shard == "time" else "all-gather",
                       "l2": "inputs exceed L2; no flush"},
            "clocks": clk}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch_arm(args, emit=True):
    """12 uneven jobs through fxc_batch_* (grouped persistent launches, CUDA graph replay,
    autotuned plans) against the same jobs run one after another through the single-job path.
    Returns the result line (printed when emit)."""
    import torch

    import difx_tests_b200 as fx

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    jobs = batch_jobs()
    cfgs, host, models = [], [], []
    total = 0
    for jb in jobs:
        cfg = fx.make_config(jb["nant"], jb["nchan"], jb["numffts"], jb["bw"], jb["lo"], npol=1, nsubband=jb["nsb"],
                             sb_spacing=jb["bw"])
        subint = fx.lib().fxc_subint_bytes(cfg)
        pitch = (subint + 16 + 255) // 256 * 256
        d = gen_device_data(torch, jb["nsb"], jb["nant"], 1, subint, pitch, jb["rho"], jb["seed"], dev)
        host.append(d[:, :subint].cpu().numpy().reshape(jb["nsb"], jb["nant"], subint))
        del d
        models.append(delay_model(jb["nant"], jb["nchan"], jb["bw"], seed=jb["seed"]))
        cfgs.append(cfg)
        total += jb["nant"] * jb["nsb"] * jb["numffts"] * 2 * jb["nchan"]
    torch.cuda.synchronize()

    def timed(step, steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    b = fx.Batch(cfgs)
    b.set_stream(stream.cuda_stream)
    for j in range(len(jobs)):
        b.upload(j, host[j])
        b.set_model(j, *models[j])
    t0 = time.perf_counter()
    b.autotune(reps=2)
    tune_s = time.perf_counter() - t0

    def bstep():
        b.reset()
        b.process()

    for _ in range(args.warmup):   # the first call runs eagerly, the second records the graph
        bstep()
    clocks = ClockSampler(0)
    clocks.start()
    ms_batch = timed(bstep, args.steps)
    clk = clocks.stop()
    plans = [b.plan(j) for j in range(len(jobs))]
    launches = b.launch_count()
    b.use_graph(False)
    ms_eager = timed(bstep, max(1, args.steps // 2))
    b.close()

    # the same jobs one after another through the single-job path (device-resident input)
    corrs = []
    for j, cfg in enumerate(cfgs):
        c = fx.Correlator(cfg)
        c.set_stream(stream.cuda_stream)
        c.upload(host[j])
        corrs.append(c)
    ptrs = [c.device_input() for c in corrs]

    def sstep():
        for j, c in enumerate(corrs):
            c.reset()
            c.process_device(ptrs[j][0], ptrs[j][1], *models[j])

    for _ in range(args.warmup):
        sstep()
    ms_seq = timed(sstep, max(1, args.steps // 2))
    for c in corrs:
        c.close()
    line = {
        "metric": METRIC, "value": total / (ms_batch / 1e3) / 1e9, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batch, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, config-0 generator per job)",
        "config": {"workload": "batch of 12 uneven jobs (fxc_batch, graph replay, autotuned plans)",
                   "jobs": [dict(nant=jb["nant"], fft=2 * jb["nchan"], nsb=jb["nsb"], numffts=jb["numffts"])
                            for jb in jobs],
                   "total_samples": total, "l2": "1.6 GB packed input > L2; no flush"},
        "batch_eager": {"ms_per_step": ms_eager, "value": total / (ms_eager / 1e3) / 1e9},
        "sequential_single_job": {"ms_per_step": ms_seq, "value": total / (ms_seq / 1e3) / 1e9},
        "batch_vs_sequential": ms_seq / ms_batch,
        "plans": [{"fft_block": tb, "x_variant": alt} for tb, alt in plans],
        "autotune_s": tune_s,
        "clocks": clk,
        "gpu_launches": launches * args.steps,
    }
    if emit:
        print(json.dumps(line))
    return line


# Large array: 256 antennas x 2 polarisations (512 signals) x 16 subbands x 4096 channels,
# 1 s at 128 MS/s (15625 FFTs of 8192 per subband), 1.05e12 input samples = 262 GB packed per
# subintegration: more than HBM holds, so the input streams through device windows
# (window_ffts FFTs of every row) while the accumulators (69 GB) stay on the device.
LARGE = dict(nant=256, npol=2, nchan=4096, nsb=16, numffts=15625, bw=64e6, lo=1.4e9, rho=0.02, window_ffts=1024)


def large_subset_accuracy(xmode, nsub=16, nf=64):
    """Error of the 256-antenna correlation against the FP64 oracle on a 16-antenna subset
    (1 subband, nf FFTs): the subset's baselines are cut out of the full-array output."""
    import difx_tests_b200 as fx
    from difx_tests_b200 import synth
    from oracle import fxoracle as fo
    L = LARGE
    job = synth.make_job(nant=L["nant"], npol=L["npol"], nchan=L["nchan"], numffts=nf, bw=L["bw"], lo=L["lo"],
                         rho=L["rho"], seed=4444)
    cfg = fx.make_config(job.nant, job.nchan, nf, job.bw, job.lo, npol=job.npol, xmode=xmode)
    with fx.Correlator(cfg) as c:
        c.process(job.data, job.delays, job.fileoffsets)
        vis, counts = c.visibilities()
    sub = np.arange(nsub) * (L["nant"] // nsub)          # every 16th antenna
    bl_all = {p: i for i, p in enumerate(fo.baseline_order(L["nant"]))}
    nbl = len(bl_all)
    rows = [bl_all[(int(sub[i]), int(sub[j]))] for i in range(nsub - 1) for j in range(i + 1, nsub)]
    rows += [nbl + int(a) for a in sub]
    got = vis[0][rows]
    ref, rc = fo.correlate(job.data[0][sub], job.delays[sub], job.fileoffsets[sub], job.bw, job.lo, job.nchan,
                           job.npol, numffts=nf)
    mx, rms = fo.vis_error(got, ref)
    return {"max_rel": float(mx.max()), "rms_rel": float(rms.max()), "vs": "FP64 oracle",
            "sample": f"{nsub}-antenna subset of the 256 x 2 pol x 4096 ch correlation, 1 subband x {nf} FFTs",
            "counts_match": bool(np.array_equal(counts[rows], rc))}


def run_large_arm(args, emit=True, max_windows=None):
    """The large array streamed through device windows; max_windows bounds the sample (the first
    windows of the subintegration).  Returns the result line (printed when emit)."""
    import torch

    import difx_tests_b200 as fx

    L = LARGE
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    F = 2 * L["nchan"]
    spb = 4 // L["npol"]
    W = L["window_ffts"]
    row_bytes = (W + 4) * F // spb
    pitch = (row_bytes + 32 + 255) // 256 * 256
    nsig = L["nant"] * L["npol"]
    delays, offs = delay_model(L["nant"], L["nchan"], L["bw"], seed=42)
    # one window of seeded data per row, generated on the device and reused by every window of
    # the subintegration (throughput does not depend on the sample values)
    t0 = time.perf_counter()
    data = gen_device_data(torch, L["nsb"], L["nant"], L["npol"], row_bytes, pitch, L["rho"], seed=7, device=dev)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    windows = [(w0, min(W, L["numffts"] - w0)) for w0 in range(0, L["numffts"], W)]
    if max_windows:
        windows = windows[:max_windows]

    def run(corr, wins):
        corr.reset()
        for w0, n in wins:
            base = np.full(L["nant"], max(0, (w0 - 2) * F), np.int64)
            corr.process_device_window(data.data_ptr(), pitch, base, row_bytes, delays, offs, w0, n)

    def timed(xmode, wins, steps, warmup):
        cfg = fx.make_config(L["nant"], L["nchan"], L["numffts"], L["bw"], L["lo"], npol=L["npol"], nsubband=L["nsb"],
                             xmode=xmode, window_ffts=W)
        corr = fx.Correlator(cfg)
        corr.set_stream(stream.cuda_stream)
        for _ in range(warmup):
            run(corr, wins)
        corr.synchronize()
        corr.enable_stage_timing(True)
        corr.stage_times(reset=True)
        clocks = ClockSampler(0)
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            run(corr, wins)
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        corr.synchronize()
        ms = e0.elapsed_time(e1) / steps
        stage_ms, launches = corr.stage_times(reset=True)
        corr.close()
        nfft = sum(n for _, n in wins)
        samples = L["nant"] * L["npol"] * L["nsb"] * nfft * F
        xflop = 8.0 * L["nchan"] * nfft * L["nsb"] * nsig * (nsig + 1) / 2
        return dict(ms=ms, value=samples / (ms / 1e3) / 1e9, samples=samples, stage_ms=stage_ms / steps,
                    launches=launches, clocks=clk, x_tflops=xflop * steps / (stage_ms[2] / 1e3) / 1e12,
                    nfft=nfft, xflop=xflop)

    tc = timed(fx.FXC_X_TC_FP16, windows, args.steps, args.warmup)
    plain = timed(fx.FXC_X_PLAIN_FP32, windows[:1], 1, 1)   # bounded sample: the first window
    hbm, tc_peak, peak_kind = peaks()
    f_bytes = tc["samples"] * (0.25 + 2.0)
    f_gbs = f_bytes / (tc["stage_ms"][1] / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": tc["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tc["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES["tc"], "data": "synthetic (seeded, generated on device; one window reused for every window)",
        "config": {"workload": "256 ant x 2 pol x 16 subbands x 4096 ch, 1 s @ 128 MS/s (15625 FFTs/subband), "
                               f"streamed in windows of {W} FFTs", "form": "tc",
                   "l2": "262 GB of input per step, far above L2; no flush",
                   "sample": (f"first {len(windows)} of {-(-L['numffts'] // W)} windows per step"
                              if max_windows else "whole subintegration per step")},
        "stages_ms_per_step": {"delay+counts": tc["stage_ms"][0], "F": tc["stage_ms"][1], "X": tc["stage_ms"][2]},
        "x_stage": {"tflops": tc["x_tflops"], "flop_per_step": tc["xflop"], "peak_tflops": tc_peak,
                    "frac": tc["x_tflops"] / tc_peak,
                    "note": "algorithmic Hermitian flops; 128x128 block pairs compute 12% more"},
        "roofline": {"kernel": "k_fstage", "bound": "hbm", "achieved": f_gbs, "peak": hbm, "unit": "GB/s",
                     "frac": f_gbs / hbm, "traffic": None, "peak_source": peak_kind + " (MEASURED_PEAKS.json)",
                     "note": "F stage is FP32-issue-bound"},
        "clocks": tc["clocks"],
        "gpu_launches": int(tc["launches"].sum()),
        "plain": {"value": plain["value"], "unit": UNIT, "ms": plain["ms"],
                  "sample": f"first window: {plain['nfft']} FFTs x 16 subbands",
                  "stages_ms": {"F": plain["stage_ms"][1], "X": plain["stage_ms"][2]},
                  "x_tflops": plain["x_tflops"], "clocks": plain["clocks"]},
        "tc_vs_plain": {"gsamps": tc["value"] / plain["value"]},
        "data_gen_s": gen_s,
    }
    del data
    torch.cuda.empty_cache()
    if not args.no_accuracy:
        line["accuracy"] = {"tc": large_subset_accuracy(fx.FXC_X_TC_FP16)}
    if emit:
        print(json.dumps(line))
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS) + ["cfg3", "cfg4"],
                    help="cfg3: the batched uneven workload (12 jobs through fxc_batch_*); cfg4: the large "
                         "array (512 signals x 4096 channels x 16 subbands) streamed through device windows")
    ap.add_argument("--xmode", default="all", choices=["all", "both"] + sorted(FORMS),
                    help="all: the FP16 tensor-core X form on the FP32-grade tensor-core F stage (tc32f) is the "
                         "headline value; the same X form on the FP32 FFT F stage (tc) and on the FP16 tensor-core "
                         "F stage (tc16f), the FP8 form and the FP32 plain form are timed beside it; both: the "
                         "headline and plain")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--shard", default="replica", choices=["replica", "time", "subband"],
                    help="replica: every rank its own subintegration (weak scaling, the default); time / subband: "
                         "one subintegration split over the ranks and merged on the device (strong scaling)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the bounded cfg3 (batch) and cfg4 (large array) runs of the default workload")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.shard != "replica":
        return run_shard_arm(args)
    if args.workload == "cfg3":
        run_batch_arm(args)
        return 0
    if args.workload == "cfg4":
        run_large_arm(args)
        return 0
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
