"""Throughput bench of the B200 accelsearch engine.

One step = one complete accelsearch of one synthetic spectrum (every block
and harmonic stage, candidates collected) through the engine.  The default
workload is the larger acceleration search: N = 2^23 samples at 64 us,
zmax = 600, numharm = 16, sigma = 2, with 3 injected 8-harmonic pulsars
(seeded synthetic data of that shape).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours       : value = f-fdot cells/s with the spectrum resident in HBM
             (device-timed with CUDA events on the engine's stream, L2
             flushed between steps); e2e = the same metric through the
             public C ABI with the spectrum in pinned host memory
             (host->device copy and the candidate read-back inside the
             timed region).  Under torchrun every rank searches its own
             spectra (independent DM trials: replicas, weak scaling).
reference  : the CPU restatement of the reference's accelsearch (FP32
             arithmetic like its FFTW path, all host threads) timed on a
             bounded sample of blocks of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes moved per byte of f-fdot planes, from one ncu capture of each
# kernel on the zmax=600 numharm=16 search at N=2^20 (one batch of 49 blocks,
# 1.87 GB of planes): the 4096-point correlation launch read 0.17 GB and wrote
# 1.81 GB for its 1.84 GB of planes (profiles/k_corr_4096_accelsearch_zmax600_
# N2e20.md); the harmonic sum read 1.885 GB and wrote 0.005 GB for the batch's
# 1.87 GB (profiles/k_harmsum_std5_accelsearch_zmax600_N2e20.md).  Both move
# bytes in proportion to the planes, so full-size launches scale by their
# plane bytes.
CORR_DRAM_PER_PLANE_BYTE = (0.17 + 1.81) / 1.84
HARMSUM_DRAM_PER_PLANE_BYTE = (1.885 + 0.005) / 1.87

WORKLOADS = {
    "cfg2": dict(N=1 << 23, dt=64e-6, zmax=600, wmax=None, numharm=16, sigma=2.0,
                 desc="accelsearch N=2^23 dt=64us zmax=600 numharm=16 sigma=2; "
                      "3 injected 8-harmonic pulsars (A=0.02/harmonic), N(0,1) noise"),
    "cfg2s": dict(N=1 << 20, dt=64e-6, zmax=600, wmax=None, numharm=16, sigma=2.0,
                  desc="profiling case: cfg2 search parameters on N=2^20"),
    "cfg1": dict(N=1 << 20, dt=64e-6, zmax=200, wmax=None, numharm=8, sigma=2.0,
                 desc="accelsearch N=2^20 dt=64us zmax=200 numharm=8 sigma=2 (in-memory); "
                      "one sinusoid f=123.4 Hz z=40 A=0.05"),
    "cfg3": dict(N=1 << 22, dt=64e-6, zmax=200, wmax=300, numharm=8, sigma=2.0,
                 desc="jerk search N=2^22 dt=64us zmax=200 wmax=300 numharm=8 sigma=2; "
                      "2 injected 4-harmonic sinusoids"),
}
METRIC = "f-fdot cells/s"
UNIT = "cells/s"


def make_spectrum(name, seed_offset=0, synth=None):
    if synth is None:
        from presto_b200 import synth
    w = WORKLOADS[name]
    if name in ("cfg2", "cfg2s"):
        return synth.cfg2_spectrum(N=w["N"], dt=w["dt"], seed=2000 + seed_offset)[0]
    if name == "cfg3":
        return synth.cfg3_spectrum(N=w["N"], dt=w["dt"], seed=3000 + seed_offset)[0]
    return synth.cfg1_spectrum(N=w["N"], dt=w["dt"], seed=1000 + seed_offset)


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.proc = device, None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "out", "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def load_synth():
    """presto_b200/synth.py (numpy only) loaded by path, so that the CPU legs
    generate the same seeded spectra without importing the engine package."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "_bench_synth", os.path.join(ROOT, "presto_b200", "synth.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def config_dict(name, blocks, cells):
    """The workload as both arms name it (identical dicts)."""
    w = WORKLOADS[name]
    return {"workload": name, "desc": w["desc"], "N": w["N"], "zmax": w["zmax"],
            "wmax": w["wmax"], "numharm": w["numharm"], "blocks": blocks,
            "cells_per_search": cells,
            "l2": "GPU arm: 256 MiB buffer written between timed steps",
            "parallelism": "replicas (independent spectra per GPU); CPU arm: rank 0 only"}


CPU_SAMPLE_STRIDE = 20          # every 20th block: a 5 % sample spread over the spectrum


def cpu_sample(name, threads, fft=None, stride=CPU_SAMPLE_STRIDE, extras=False, max_blocks=None):
    """The oracle port (FP32 arithmetic like the reference's FFTW path, OpenMP
    over templates like the reference) timed on one search's template banks
    plus every stride-th block of the main loop, scaled to the whole search
    (in-memory searches run whole: their plane needs every block).  Geometry,
    block count and cells come from the oracle's own obs_init.  Returns a
    dict: cells/s, searches/s, the step's wall ms, description and, with
    extras, the FFT share of thread time, a one-thread block-loop point and
    the -march=native build's point."""
    from oracle import pyoracle as po
    w = WORKLOADS[name]
    if fft is None:
        fft = make_spectrum(name, synth=load_synth())
    p = po.make_params(w["N"], w["dt"], fft.size, zmax=w["zmax"], wmax=w["wmax"],
                       numharm=w["numharm"], sigma=w["sigma"])
    obs = po.obs_init(p, 32)
    counts = po.search_counts(obs)
    nb = counts["blocks"]
    first, count = (0, nb) if obs.inmem else (stride // 2, max(1, (nb - stride // 2 + stride - 1)
                                                                 // stride))
    if max_blocks is not None:
        count = min(count, max_blocks)
    t0 = time.perf_counter()
    done, t_setup, t_blocks, fft_s, loop_s = po.accelsearch_sample(
        p, fft, threads, first, count, 1 if obs.inmem else stride)
    step_ms = (time.perf_counter() - t0) * 1e3
    per_block = t_blocks / max(done, 1)
    t_search = t_setup + per_block * nb
    out = {"cells_per_s": counts["cells"] / t_search, "searches_per_s": 1.0 / t_search,
           "step_ms": step_ms, "blocks": nb, "cells": counts["cells"],
           "desc": (f"oracle port FP32 (project scalar mixed-radix FFT, not FFTW), {threads} "
                    f"threads: template banks {t_setup:.2f} s + {done} of {nb} blocks "
                    f"(every {1 if obs.inmem else stride}th from block {first}) at "
                    f"{per_block * 1e3:.1f} ms/block, scaled to {nb} blocks"),
           "fft_share": fft_s / max(loop_s, 1e-9)}
    if extras and not obs.inmem:
        k = max(1, count // 16)             # one-thread loop: a sixteenth of the sample
        d1, _, tb1, _, _ = po.accelsearch_sample(p, fft, threads, first, k, stride * (count // k),
                                                 loop_threads=1)
        pb1 = tb1 / max(d1, 1)
        out["one_thread"] = {"ms_per_block": pb1 * 1e3,
                             "block_loop_cells_per_s": counts["cells"] / nb / pb1,
                             "blocks_timed": d1,
                             "openmp_speedup": pb1 / per_block,
                             "what": "the block loop on 1 thread (template banks built on "
                                     f"{threads} threads, not counted)"}
        nat = po.build_native()
        if nat:
            dn, tsn, tbn, _, _ = po.accelsearch_sample(p, fft, threads, first, count, stride,
                                                       libpath=nat)
            tn = tsn + tbn / max(dn, 1) * nb
            out["march_native"] = {"cells_per_s": counts["cells"] / tn,
                                   "template_banks_s": tsn,
                                   "ms_per_block": tbn / max(dn, 1) * 1e3,
                                   "speedup_vs_default_build": t_search / tn,
                                   "what": "the same oracle compiled with -march=native "
                                           "on this host, same sample"}
    return out


def cpu_polish_sample(fft, lobin, cands, threads, jerk=False, max_cands=16):
    """Times the polishing oracle (optimize_accelcand restated, OpenMP over
    candidates) on the first max_cands candidates; returns (ms per candidate,
    description)."""
    from oracle import pyoracle as po
    sample = [(c[2], c[3], c[4], c[5]) for c in cands[:max_cands]]
    if not sample:
        return None, "no candidates"
    t0 = time.perf_counter()
    po.optimize_cands_w(fft, lobin, sample, jerk=jerk, nthreads=threads)
    ms = (time.perf_counter() - t0) * 1e3 / len(sample)
    what = "max_rzw_arr_harmonics" if jerk else "max_rz_arr_harmonics"
    return ms, f"polishing oracle ({what}), {threads} threads, {len(sample)} candidates"


def run_reference(args):
    """The reference's CPU algorithm (the oracle port; the reference program
    built here runs over a test-stand-in FFT and is never timed) on this
    host's cores.  Nothing of the engine package is imported or loaded."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    name = args.workload
    fft = make_spectrum(name, synth=load_synth())
    for _ in range(args.warmup):
        cpu_sample(name, threads, fft=fft, max_blocks=1)         # banks + one block
    steps = [cpu_sample(name, threads, fft=fft, extras=(k == 0)) for k in range(args.steps)]
    first = steps[0]
    v = statistics.median(st["cells_per_s"] for st in steps)
    base = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": first["desc"] + "; median of the steps",
            "fft_share_of_thread_time": first["fft_share"]}
    for key in ("one_thread", "march_native"):
        if key in first:
            base[key] = first[key]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(st["step_ms"] for st in steps),
            "ms_per_step_is": "wall time of one step's sample (template banks + the block "
                              "sample), not of a whole search",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": config_dict(name, first["blocks"], first["cells"]),
            "searches_per_s": v / first["cells"],
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import presto_b200 as pb
    from presto_b200 import replicas

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    name = args.workload
    w = WORKLOADS[name]
    fft = make_spectrum(name, seed_offset=rank)
    ctx = pb.Context(local)
    tc = args.corr in ("tc", "tc16")
    if tc:
        ctx.set_corr_path(pb.CORR_TC_SPLIT_BF16 if args.corr == "tc" else pb.CORR_TC_SPLIT_FP16)
    if args.scratch_mb:
        ctx.L.ab_ctx_set_hbm_budget(ctx.ptr, int(args.scratch_mb) * 4 << 20)
    obs = pb.obs_init(pb.make_params(w["N"], w["dt"], fft.size, zmax=w["zmax"], wmax=w["wmax"],
                                     numharm=w["numharm"], sigma=w["sigma"]))
    counts = pb.algorithmic_counts(obs)
    stream = torch.cuda.ExternalStream(ctx.stream, device=local)
    dev_fft = torch.from_numpy(fft.view(np.float32).copy()).to(f"cuda:{local}")
    torch.cuda.synchronize()
    flush = torch.empty(64 << 20, dtype=torch.float32, device=f"cuda:{local}")   # 256 MiB > L2

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident value ----
    for _ in range(args.warmup):
        ctx.search(obs, None, device_ptr=dev_fft.data_ptr())
    ctx.reset_kernel_times()
    ctx.set_profiling(True)
    launches0 = ctx.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    ncands = 0
    barrier()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
            ev[k][0].record(stream)
            ncands = len(ctx.search(obs, None, device_ptr=dev_fft.data_ptr()))
            ev[k][1].record(stream)
        barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    launches = ctx.launch_count() - launches0
    kms, kn = ctx.kernel_times()
    ctx.set_profiling(False)
    ms_max = replicas.max_over_ranks(ms, dist, device=f"cuda:{local}")
    total_cells = counts["cells"] * args.steps * world
    value = total_cells / (ms_max / 1e3)

    # ---- end to end through the C ABI with pinned host buffers ----
    # each step: L2 flushed as in the device loop (outside the timed span),
    # then the call with the spectrum in pinned host memory; the call returns
    # once the candidates are on the host
    host = torch.from_numpy(fft.view(np.float32).copy()).pin_memory()
    host_np = host.numpy().view(np.complex64)
    ctx.search(obs, host_np)
    barrier()
    wall_ms = ev_ms = 0.0
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        ctx.search(obs, host_np)
        e1.record(stream)
        t1 = time.perf_counter()
        e1.synchronize()
        wall_ms += (t1 - t0) * 1e3
        ev_ms += e0.elapsed_time(e1)
    barrier()
    e2e_ms = max(ev_ms, wall_ms)
    e2e_ms = replicas.max_over_ranks(e2e_ms, dist, device=f"cuda:{local}")
    nhits = len(ctx.last_hits()[0])

    # ---- the time-series input path (realfft + deredden) at this N ----
    series = torch.randn(w["N"], dtype=torch.float32, device=f"cuda:{local}")
    sfft = torch.empty(w["N"], dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(2):
        ctx.L.ab_series_to_fft(ctx.ptr, series.data_ptr(), w["N"], w["dt"], 1, sfft.data_ptr(), 1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        rcs = ctx.L.ab_series_to_fft(ctx.ptr, series.data_ptr(), w["N"], w["dt"], 1,
                                     sfft.data_ptr(), 1)
    torch.cuda.synchronize()
    s_ms = (time.perf_counter() - t0) * 1e3 / reps
    series_line = {"n": w["N"], "ms": s_ms, "status": int(rcs),
                   "gb_per_s_algorithmic": 8.0 * w["N"] / (s_ms / 1e3) / 1e9,
                   "what": "realfft + deredden(6, 200, Nyquist, N dt), device in and out, wall "
                           "time per call including the host block plan"}
    del series, sfft

    # ---- subband dedispersion, the DM trials' producer (device in and out) ----
    dd_line = dedisp_measure(ctx, torch, local)

    # ---- candidate polishing (optimize_accelcand) of the search's candidates ----
    cl = ctx.search(obs, None, device_ptr=dev_fft.data_ptr())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.optimize_cands(obs, None, cl, device_ptr=dev_fft.data_ptr())
    torch.cuda.synchronize()
    polish = {"candidates": len(cl), "gpu_ms": (time.perf_counter() - t0) * 1e3,
              "what": "optimize_accelcand (harmonic polishing: max_rz%s_arr_harmonics) of every "
                      "candidate, device" % ("w" if obs.numw else "")}

    # ---- roofline of the dominant kernel (correlation) ----
    corr_ms_per_search = kms[2] / args.steps
    harm_ms = kms[3] / args.steps
    # DRAM traffic per launch, standard mode: each kernel's measured DRAM bytes
    # per byte of f-fdot planes (one ncu capture each on the zmax=600 numharm=16
    # search at N=2^20) times this search's plane bytes per launch
    corr_traffic = harm_traffic = None
    if not obs.inmem and not tc and kn[2] and kn[3]:
        planes = counts["harmsum_min_bytes"] * args.steps
        corr_traffic = CORR_DRAM_PER_PLANE_BYTE * planes / kn[2]
        harm_traffic = HARMSUM_DRAM_PER_PLANE_BYTE * planes / kn[3]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    if tc:
        # split-BF16 contraction, timed inside a long step: sustained BF16 peak
        tflops = counts["tc_flops"] / (corr_ms_per_search / 1e3) / 1e12
        bf16 = peaks.get("bf16_tflops_sustained")
        src = "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)"
        if bf16 is None:
            bf16, src = 1400.0, "fallback sustained BF16 1.4 PFLOP/s (of fallback)"
        roof = {"bound": "tensor", "kernel": "k_corr_tc (split-%s banded contraction)"
                % ("BF16" if args.corr == "tc" else "FP16"),
                "achieved": tflops, "peak": bf16, "unit": "TFLOP/s", "frac": tflops / bf16,
                "traffic": None, "flops_per_search": counts["tc_flops"],
                "kernel_ms_per_search": corr_ms_per_search, "peak_source": src}
    else:
        achieved = counts["corr_flops"] / (corr_ms_per_search / 1e3) / 1e12
        fp32_peak = measured_fp32_peak(ctx)
        roof = {"bound": "fp32", "kernel": "k_corr (template correlation)",
                "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": corr_traffic,
                "traffic_unit": "DRAM bytes per launch (average over the search's correlation "
                                "launches), scaled from profiles/k_corr_4096_accelsearch_zmax600"
                                "_N2e20.md by plane bytes" if corr_traffic else None,
                "flops_per_search": counts["corr_flops"],
                "kernel_ms_per_search": corr_ms_per_search,
                "peak_source": "measured in-run FP32 FMA loop (MEASURED_PEAKS.json "
                               "holds no FP32 CUDA-core figure)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("bf16" if args.corr == "tc" else "fp16") + " hi+lo products, f32 accumulate"
                     if tc else "f32",
            "data": "synthetic",
            "config": config_dict(name, counts["blocks"], counts["cells"]),
            "corr": {"fft": "fft_f32", "tc": "tc_split_bf16", "tc16": "tc_split_fp16"}[args.corr],
            "searches_per_s": value / counts["cells"],
            "candidates_per_search": ncands,
            "gpu_launches": int(launches),
            "e2e": {"value": counts["cells"] * args.steps * world / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(fft.nbytes),
                    "d2h_bytes_per_step": int(4 + 12 * nhits),
                    "searches_per_s": args.steps * world / (e2e_ms / 1e3)},
            "roofline": roof,
            "roofline_harmsum": {"bound": "hbm", "kernel": "k_harmsum (sum + search)",
                                 "achieved": counts["harmsum_min_bytes"] / (harm_ms / 1e3) / 1e9,
                                 "peak": hbm, "unit": "GB/s",
                                 "frac": counts["harmsum_min_bytes"] / (harm_ms / 1e3) / 1e9 / hbm,
                                 "bytes": "planes read once (the fused kernel's minimum)",
                                 "traffic": harm_traffic,
                                 "traffic_unit": "DRAM bytes per launch, scaled from profiles/"
                                                 "k_harmsum_std5_accelsearch_zmax600_N2e20.md by "
                                                 "plane bytes" if harm_traffic else None,
                                 "unfused_equivalent_gbs":
                                     counts["harmsum_bytes"] / (harm_ms / 1e3) / 1e9,
                                 "kernel_ms_per_search": harm_ms},
            "kernel_ms_per_search": {"templates": kms[0] / args.steps, "prep": kms[1] / args.steps,
                                     "corr": corr_ms_per_search, "harmsum": harm_ms},
            "host_ms_per_search": {"outside_replay": kms[4] / args.steps,
                                   "sort_and_replay_overlapped": kms[5] / args.steps},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu:
            cs = cpu_sample(name, os.cpu_count() or 1, fft=fft)
            line["cpu_baseline"] = {"value": cs["cells_per_s"], "unit": UNIT,
                                    "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": cs["desc"], "searches_per_s": cs["searches_per_s"],
                                    "fft_share_of_thread_time": cs["fft_share"]}
            dcs = cpu_dedisp_sample()
            if dcs:
                dd_line["cpu_baseline"] = dcs
            if polish and polish["candidates"]:
                pms, pdesc = cpu_polish_sample(fft, obs.lobin, cl, os.cpu_count() or 1,
                                               jerk=bool(obs.numw))
                polish["cpu_ms_per_candidate"] = pms
                polish["cpu_sample"] = pdesc
        if polish:
            line["polish"] = polish
        line["series_to_fft"] = series_line
        line["dedisperse"] = dd_line
    ctx.close()
    if rank == 0 and world == 1 and not args.no_pool:
        # the pool patterns against the plain path on the same GPU (after the
        # timed search, which they do not touch): cfg4 on both correlation
        # paths, cfg5 at 2000 requests/s
        line["batched"] = [pool_compare("batched", args.requests, workers=args.workers),
                           pool_compare("batched", args.requests, workers=args.workers,
                                        corr="tc")]
        line["served"] = [pool_compare("served", 2 * args.requests, rate=args.rate,
                                       workers=args.workers),
                          pool_compare("served", 2 * args.requests, rate=args.rate,
                                       workers=args.workers, corr="tc16")]
    if rank == 0 and world == 1 and not args.no_pipeline:
        # filterbank spectra to candidates over 32 DM trials (one pass each way)
        try:
            line["pipeline"] = pipeline_measure(1)
        except Exception as e:          # a side measurement: the line stands without it
            line["pipeline"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def dedisp_measure(ctx, torch, local, nspec=1 << 20, nchan=1024, nsub=64, ndm=128, reps=3):
    """ab_dedisperse of nspec x nchan float spectra into ndm DM trials (device
    buffers), timed by CUDA events on the context's stream."""
    dev = f"cuda:{local}"
    x = torch.randn((nspec, nchan), dtype=torch.float32, device=dev)
    out = torch.empty((ndm, nspec), dtype=torch.float32, device=dev)
    dms = np.linspace(0.0, 300.0, ndm)
    args = (None, 1400.0, 0.25, 64e-6, nsub, dms)
    kw = dict(device_ptr=x.data_ptr(), nspec=nspec, nchan=nchan, out_ptr=out.data_ptr())
    ctx.dedisperse(*args, **kw)                               # warm-up
    torch.cuda.synchronize()
    ctx.reset_kernel_times()
    ctx.set_profiling(True)
    for _ in range(reps):
        ctx.dedisperse(*args, **kw)
    kms, _ = ctx.kernel_times()
    ctx.set_profiling(False)
    ms = kms[7] / reps
    algo = 4.0 * nspec * nchan + 4.0 * ndm * nspec            # spectra read once, trials written
    del x, out
    torch.cuda.empty_cache()
    return {"nspec": nspec, "nchan": nchan, "nsub": nsub, "ndm": ndm, "ms": ms,
            "trials_per_s": ndm / (ms / 1e3),
            "gb_per_s_algorithmic": algo / (ms / 1e3) / 1e9,
            "what": "subband sums at the DMs' mean from the time-major spectra, then DM sums "
                    "(prepsubband's two stages, 1400 MHz + 256 MHz band, DM 0-300), device in "
                    "and out; algorithmic bytes = spectra read once + trials written"}


def cpu_dedisp_sample(nspec=1 << 17, nchan=1024, nsub=64, ndm=128, full_nspec=1 << 20):
    """The reference's own dedisp_subbands / float_dedisp (src/dispersion.c,
    compiled unmodified into oracle/_ref/libref_dedisp.so; dedisp_subbands is
    OpenMP-parallel over subbands) streamed in 8192-spectrum blocks as
    prepsubband streams them, on a 1/8-length sample of dedisp_measure's
    workload; trials/s at the full length, scaled by spectra.  None where the
    library is absent."""
    from oracle import pyoracle as po
    L = po.ref_dedisp_lib()
    if L is None:
        return None
    X = np.random.default_rng(5).standard_normal((nspec, nchan), dtype=np.float32)
    dms = np.linspace(0.0, 300.0, ndm)
    t0 = time.perf_counter()
    po.ref_dedisperse(L, X, 1400.0, 0.25, 64e-6, nsub, dms, 1, 8192)
    full_ms = (time.perf_counter() - t0) * 1e3 * full_nspec / nspec
    cores = os.cpu_count() or 1
    return {"value": ndm / (full_ms / 1e3), "unit": "trials/s", "cores": cores,
            "kind": "reference", "ms_full_length": full_ms,
            "sample": f"{nspec} of {full_nspec} spectra x {nchan} channels into {ndm} DM trials "
                      f"(nsub {nsub}), blocks of 8192 with the transposes prepsubband makes, "
                      f"OpenMP threads up to {cores}; scaled to the full length by spectra"}


def measured_fp32_peak(ctx):
    import ctypes as C
    import presto_b200 as pb
    v = C.c_double()
    rc = pb.lib().ab_measure_fp32_peak(ctx.ptr, C.byref(v))
    return v.value if rc == 0 else None


class SpectrumCache:
    """Seeded synthetic spectra by (N, injected) so a long request mix does not
    spend minutes generating time series; the mix itself is seeded."""

    def __init__(self, dt, seed):
        self.dt, self.seed, self.cache = dt, seed, {}

    def get(self, N, inject, rng):
        key = (N, inject)
        if key not in self.cache:
            from presto_b200 import synth
            ps = []
            if inject:
                T = N * self.dt
                f = float(np.exp(rng.uniform(np.log(5.0), np.log(300.0))))
                ps = [dict(r=f * T, z=float(rng.uniform(-200, 200)),
                           harms=[(0.02, float(rng.uniform(0, 6.28))) for _ in range(8)])]
            self.cache[key] = synth.spectrum(synth.time_series(N, self.seed + len(self.cache), ps))
        return self.cache[key]


def batched_requests(n, seed):
    """cfg4 recipe: lengths uniform in {2^20..2^23}, zmax in {50, 200, 600},
    numharm 8, wmax 0 (not given), 5 % with an injected 8-harmonic pulsar."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(1 << int(rng.integers(20, 24)))
        out.append(dict(N=N, inject=bool(rng.random() < 0.05),
                        opts=dict(zmax=int(rng.choice([50, 200, 600])), numharm=8)))
    return out, rng


def served_requests(n, seed, rate):
    """cfg5 recipe: Poisson arrivals, N log-uniform in 2^19..2^23 (on a
    half-octave grid), zmax in {0,100,300,600}, wmax in {0,0,0,200},
    numharm in {4,8,16}, noise and injection as in the batched mix."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        N = int(round(2 ** (19 + 0.5 * int(rng.integers(0, 9))) / 2)) * 2
        opts = dict(zmax=int(rng.choice([0, 100, 300, 600])), numharm=int(rng.choice([4, 8, 16])))
        w = int(rng.choice([0, 0, 0, 200]))
        if w:
            opts["wmax"] = w
        out.append(dict(t=t, N=N, inject=bool(rng.random() < 0.05), opts=opts))
    return out, rng


def pool_compare(mode, nreq, rate=2000.0, workers=4, corr="fft"):
    """The request pool (ab_pool: continuous batching, HBM admission) against
    the plain single-request path on the same requests and GPU.  mode
    "batched": the cfg4 recipe (all requests queued at once); "served": the
    cfg5 recipe with Poisson arrivals at `rate` per second.  corr "tc": both
    paths on the split-BF16 tensor-core correlation.  Template banks of every
    request geometry are built before timing (resident, shared by all
    contexts).  The plain path's device-busy fraction is its kernels' CUDA-
    event time over its wall time."""
    import presto_b200 as pb
    from presto_b200 import serve
    dt = 64e-6
    if mode == "batched":
        reqs, rng = batched_requests(nreq, 4000)
    else:
        reqs, rng = served_requests(nreq, 5000, rate)
    cache = SpectrumCache(dt, 4100)
    ffts = [cache.get(r["N"], r["inject"], rng) for r in reqs]
    obss = [pb.obs_init(pb.make_params(r["N"], dt, f.size, **r["opts"])) for r, f in zip(reqs, ffts)]
    cells = sum(pb.algorithmic_counts(o)["cells"] for o in obss)
    paths = {"tc": pb.CORR_TC_SPLIT_BF16, "tc16": pb.CORR_TC_SPLIT_FP16}
    ctx = pb.Context(0)
    if corr in paths:
        ctx.set_corr_path(paths[corr])
    seen = set()
    t0 = time.perf_counter()
    for r, o in zip(reqs, obss):
        key = (r["N"], tuple(sorted(r["opts"].items())))
        if key not in seen:
            seen.add(key)
            ctx.prepare(o)
    t_banks = time.perf_counter() - t0
    for o, f in list(zip(obss, ffts))[:3]:                   # warm-up
        ctx.search(o, f)
    ctx.reset_kernel_times()
    ctx.set_profiling(True)
    t0 = time.perf_counter()
    plain = [ctx.search(o, f) for o, f in zip(obss, ffts)]
    t_plain = time.perf_counter() - t0
    kms, _ = ctx.kernel_times()
    ctx.set_profiling(False)
    ctx.close()
    busy = sum(kms[:4]) / 1e3 / t_plain
    pool = serve.SearchPool(0, nworkers=workers)
    try:
        if corr in paths:
            pool.set_corr_path(paths[corr])
        for r, f in zip(reqs[:workers], ffts[:workers]):      # warm-up
            pool.wait(pool.submit(f, r["N"], dt, **r["opts"]))
        pool.reset_stats()
        t0 = time.perf_counter()
        tickets = []
        for r, f in zip(reqs, ffts):
            if mode == "served":
                delay = r["t"] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            tickets.append(pool.submit(f, r["N"], dt, **r["opts"]))
        got = [pool.wait(t)[0] for t in tickets]
        t_pool = time.perf_counter() - t0
        st = pool.stats()
    finally:
        pool.close()
    recipe = ("cfg4 (batched DM trials: N uniform in 2^20..2^23, zmax 50/200/600, numharm 8)"
              if mode == "batched" else
              f"cfg5 (served stream: Poisson arrivals at {rate:g}/s, N log-uniform 2^19..2^23, "
              "zmax 0/100/300/600, wmax 0/0/0/200, numharm 4/8/16)")
    return {"mode": mode, "recipe": recipe, "requests": len(reqs), "workers": workers,
            "corr": {"fft": "fft_f32", "tc": "tc_split_bf16", "tc16": "tc_split_fp16"}[corr],
            "searches_per_s": len(reqs) / t_pool,
            "plain_searches_per_s": len(reqs) / t_plain,
            "speedup_vs_plain": t_plain / t_pool,
            "cells_per_s": cells / t_pool, "plain_cells_per_s": cells / t_plain,
            "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"]},
            "plain_device_busy_fraction": busy,
            "results_identical_to_plain": all(a == b for a, b in zip(got, plain)),
            "distinct_geometries": len(seen), "bank_build_s": t_banks,
            "spectra": "seeded synthetic, one noise and one injected spectrum per length reused "
                       "across requests; wall-clock timing (host arrays in, candidates out)"}


def run_dedisp_mode(args):
    """--mode dedisperse: the dedispersion measurement alone, one line."""
    import torch
    import presto_b200 as pb
    ctx = pb.Context(0)
    try:
        dd = dedisp_measure(ctx, torch, 0, nspec=args.dd_nspec, reps=max(1, args.steps))
    finally:
        ctx.close()
    if not args.no_cpu:
        dcs = cpu_dedisp_sample(nspec=min(1 << 17, args.dd_nspec), full_nspec=args.dd_nspec)
        if dcs:
            dd["cpu_baseline"] = dcs
    line = {"metric": "DM trials/s", "value": dd["trials_per_s"], "unit": "trials/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "steps": max(1, args.steps), "ms_per_step": dd["ms"], "dedisperse": dd}
    print(json.dumps(line), flush=True)
    return 0


def run_pipeline_mode(args):
    """--mode pipeline: pipeline_measure as a line of its own."""
    line = pipeline_measure(max(1, args.steps))
    print(json.dumps(line), flush=True)
    return 0


def pipeline_measure(steps):
    """Float filterbank spectra (1024 channels x 2^20 samples of 64 us,
    1400 MHz + 256 MHz, a pulsar at DM 150, 0.05 sigma per channel) to
    candidates: 32 DM trials over 0-300 searched with the smaller search's
    parameters (zmax 200, numharm 8), all on the device
    (ab_search_dedispersed), against the same steps chained through host
    arrays.  Wall-clock per step; the spectra start in host memory in both,
    then once more already in device memory."""
    import presto_b200 as pb
    nspec, nchan, nsub, ndm, dt = 1 << 20, 1024, 64, 32, 64e-6
    import torch
    rng = np.random.default_rng(11)
    X = rng.standard_normal((nspec, nchan), dtype=np.float32)
    freqs = 1400.0 + 0.25 * np.arange(nchan)
    shift = np.rint(150.0 / (0.000241 * freqs ** 2) / dt).astype(np.int64)
    shift -= shift[-1]
    ms_ = int(shift.max())
    base = (0.05 * (np.cos(2 * np.pi * np.arange(-ms_, nspec) * dt * 31.7) > 0.97)).astype(np.float32)
    for c in range(nchan):
        X[:, c] += base[ms_ - shift[c]:ms_ - shift[c] + nspec]
    dms = np.linspace(0.0, 300.0, ndm)
    n = nspec & ~1
    ctx = pb.Context(0)
    try:
        obs = pb.obs_init(pb.make_params(n, dt, n // 2, zmax=200, numharm=8, sigma=2.0))
        ctx.search_dedispersed(X, 1400.0, 0.25, dt, nsub, dms, obs)          # warm-up
        dev_ms, host_ms, ncand = [], [], 0
        for _ in range(steps):
            t0 = time.perf_counter()
            res = ctx.search_dedispersed(X, 1400.0, 0.25, dt, nsub, dms, obs)
            dev_ms.append((time.perf_counter() - t0) * 1e3)
            ncand = sum(len(r) for r in res)
            t0 = time.perf_counter()
            trials = ctx.dedisperse(X, 1400.0, 0.25, dt, nsub, dms)
            chain = [ctx.search(obs, ctx.series_to_fft(trials[d][:n], dt)) for d in range(ndm)]
            host_ms.append((time.perf_counter() - t0) * 1e3)
            assert chain == res, "device pipeline differs from the host chain"
        best = max(range(ndm), key=lambda d: max((c[1] for c in res[d]), default=0.0))
        # the same with the spectra already in device memory
        dx = torch.from_numpy(X).cuda()
        res_dev_ms = []
        ctx.reset_kernel_times()
        ctx.set_profiling(True)
        for _ in range(steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rd = ctx.search_dedispersed(None, 1400.0, 0.25, dt, nsub, dms, obs,
                                        device_ptr=dx.data_ptr(), nspec=nspec, nchan=nchan)
            res_dev_ms.append((time.perf_counter() - t0) * 1e3)
            assert rd == res
        kms, _ = ctx.kernel_times()
        ctx.set_profiling(False)
        per_trial = {k: v / (ndm * len(res_dev_ms)) for k, v in
                     zip(("templates", "prep", "corr", "harmsum", "host_outside_replay",
                          "replay_overlapped", "wait_and_readback"), kms[:7])}
        per_trial["dedispersion"] = kms[7] / (ndm * len(res_dev_ms))
        del dx
    finally:
        ctx.close()
    ms = statistics.median(dev_ms)
    line = {"metric": "DM trials searched/s (filterbank to candidates)", "value": ndm / (ms / 1e3),
            "unit": "trials/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "steps": len(dev_ms), "ms_per_step": ms,
            "config": {"workload": "pipeline", "nspec": nspec, "nchan": nchan, "nsub": nsub,
                       "ndm": ndm, "dm_range": [0.0, 300.0], "zmax": 200, "numharm": 8},
            "spectra_on_device_ms_per_step": statistics.median(res_dev_ms),
            "ms_per_trial_by_stage": per_trial,
            "spectra_h2d_bytes_per_step": int(X.nbytes),
            "host_chain_ms_per_step": statistics.median(host_ms),
            "device_vs_host_chain": statistics.median(host_ms) / ms,
            "candidates": ncand, "strongest_trial_dm": float(dms[best]),
            "what": "ab_search_dedispersed: spectra in host memory, dedispersion, then per trial "
                    "realfft + deredden + search on the device; host_chain = the same steps with "
                    "the trials and spectra through host arrays (identical candidates)"}
    return line


def run_pool_mode(args):
    """--mode batched | served: one pool_compare line."""
    line = pool_compare(args.mode, args.requests, args.rate, args.workers, args.corr)
    line.update({"metric": "DM-trial searches/s", "value": line["searches_per_s"],
                 "unit": "searches/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
                 "data": "synthetic"})
    print(json.dumps(line), flush=True)
    return 0 if line["results_identical_to_plain"] else 1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="cfg2")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--scratch-mb", type=int, default=0,
                    help="cap the engine's block scratch (profiling runs)")
    ap.add_argument("--corr", choices=["fft", "tc", "tc16"], default="fft",
                    help="correlation path: FP32 FFTs, or the tensor-core contraction with "
                         "split-BF16 (tc) or split-FP16 (tc16) operands")
    ap.add_argument("--mode", choices=["plain", "batched", "served", "dedisperse", "pipeline"],
                    default="plain",
                    help="batched/served: the request pool vs the plain path (one GPU); "
                         "dedisperse: subband dedispersion alone; pipeline: filterbank "
                         "spectra to candidates over 32 DM trials")
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--rate", type=float, default=2000.0, help="served: arrivals per second")
    ap.add_argument("--dd-nspec", type=int, default=1 << 20,
                    help="dedisperse mode: spectra (of 1024 channels) to dedisperse")
    ap.add_argument("--no-pipeline", action="store_true",
                    help="leave the filterbank-to-candidates pipeline out of the default line")
    ap.add_argument("--no-pool", action="store_true",
                    help="leave the batched / served comparison out of the default line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.mode == "dedisperse" and args.impl == "ours":
        return run_dedisp_mode(args)
    if args.mode == "pipeline" and args.impl == "ours":
        return run_pipeline_mode(args)
    if args.mode != "plain" and args.impl == "ours":
        return run_pool_mode(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
