"""Benchmark of the B200 JW step (one JSON line on rank 0).

Workload (the configuration the headline metric is quoted on): N = 1024 rows,
65 536 complex right-hand sides in strided XXII layout, a 5-band matvec fused
ahead of the tridiagonal solve (PfSolve jw_type 13, upperBanded 2) and the
XXII -> packed conversion (block 7) fused behind it: one kernel per step.
Synthetic seeded inputs with the named shapes and distributions; inputs are
2 GiB (larger than the 126 MB L2), so no L2 flush is needed between steps.

value  : complex RHS/s over the whole job (all ranks), inputs resident in HBM.
e2e    : same metric through the C ABI with host buffers: pinned H2D of the
         step's input, the fused kernel, D2H of the step's output.
roofline: algorithmic bytes (read XXII + write packed: 2*N*16 B per complex RHS,
         plus bands once) / kernel time, against MEASURED_PEAKS.json hbm_gbs.
--impl reference: the reference's CPU verification algorithm (sequential
         band matvec + Thomas per RHS, restated in C) on the host cores.
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

M_ROWS = 1024
N_CPLX = 65536
METRIC = "JW-step RHS/s (N=1024, 65536 complex RHS, 5-band matvec + tridiagonal solve, XXII->packed), FP64"
UNIT = "complex RHS/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_sample(target_s=12.0, threads=None, mode="d"):
    """Time the reference's CPU verification path (port: banded matvec plus
    sequential Thomas per RHS, in double, or in __float128 with mode "q") on a
    bounded sample of the workload; returns (complex RHS/s, cores, sample
    description)."""
    from oracle import oracle as O
    from pfsolve_b200 import workloads as WL
    threads = threads or os.cpu_count() or 1
    probe = 64 if mode == "d" else 8
    wl = WL.config2(B=probe)
    M = wl.M

    def run(ncplx, rhs):
        c1 = O.Case(M=M, batch=2 * ncplx, LDA=5, KU=2, KL=2, jw_type=0)
        y = O.dgbmv(c1, wl.dgbmv, rhs, mode=mode, nthreads=threads)
        c2 = O.Case(M=M, batch=2 * ncplx, upperBanded=2, jw_type=13)
        O.jw_step(c2, wl.jw_bands, y, mode=mode, nthreads=threads)

    t0 = time.perf_counter()
    run(probe, wl.rhs[:2 * M * probe])
    t = time.perf_counter() - t0
    n = int(min(N_CPLX, max(probe, probe * target_s / max(t, 1e-6))))
    rng = np.random.default_rng(1)
    rhs = rng.standard_normal(2 * M * n)
    t0 = time.perf_counter()
    run(n, rhs)
    t = time.perf_counter() - t0
    kind = "double" if mode == "d" else "__float128"
    return n / t, threads, f"{n} of {N_CPLX} complex RHS (N=1024), {kind}, {threads} OpenMP threads, {t:.1f} s"


def cpu_reference_variants(target_s=3.0):
    """The same CPU path single-threaded (as the reference's test drivers run
    it) and in __float128 on all host cores: short bounded samples, reported
    beside the main CPU baseline."""
    out = []
    for threads, mode in ((1, "d"), (None, "q")):
        v, cores, desc = cpu_reference_sample(target_s=target_s, threads=threads, mode=mode)
        out.append({"value": v, "unit": UNIT, "cores": cores, "sample": desc})
    return out


def spread_sample(nsys, ngroups, n=64, seed=7):
    """Systems their group solves first, second and last (group y mod
    ngroups takes system y at its (y div ngroups)-th turn), plus others."""
    rng = np.random.default_rng(seed)
    g = rng.choice(min(ngroups, nsys), n // 4, replace=False)
    parts = [g, g + ngroups, g + ngroups * ((nsys - 1 - g) // ngroups), rng.choice(nsys, n // 4, replace=False)]
    return np.unique(np.concatenate(parts) % nsys)


def parity_check(snap_in, snap_out, dgbmv, bands, M, ys):
    """Checker for the timed output: the sampled systems' XXII inputs through
    the __float128 oracle chain (dgbmv -> JW step -> block 7), against the
    packed results the GPU wrote in its last timed step."""
    from oracle import oracle as O
    n = len(ys)
    th = os.cpu_count() or 1
    y = O.dgbmv(O.Case(M=M, batch=2 * n, LDA=5, KU=2, KL=2, jw_type=0), dgbmv, snap_in.ravel(), nthreads=th)
    x = O.jw_step(O.Case(M=M, batch=2 * n, upperBanded=2, jw_type=13), bands, y, "q", nthreads=th)
    ref = O.block(O.Case(M=M, batch=n, block=7, jw_type=0), x, np.zeros(2 * M * n)).reshape(n, -1)
    got = snap_out.reshape(n, -1)
    rel = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    return {"max_rel_err": float(rel.max()), "systems_checked": int(n), "tolerance": 1e-13,
            "ok": bool(rel.max() <= 1e-13),
            "oracle": "__float128 chain (dgbmv -> JW step -> block 7) on the host",
            "sample": "systems solved first, second and last by their group, plus random ones, "
                      "from the output of the last timed step"}


def reference_arm(args, rank, world):
    if rank != 0:
        return
    vals = []
    info = None
    for _ in range(args.warmup):
        cpu_reference_sample(target_s=2.0)
    for _ in range(args.steps):
        v, cores, desc = cpu_reference_sample(target_s=8.0)
        vals.append(v)
        info = (cores, desc)
    v = statistics.median(vals)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * N_CPLX / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded, N(0,1) complex RHS, dominant tridiagonal, U(-1,1) 5-band)",
            "config": {"workload": "config2: N=1024, 65536 complex RHS, XXII in -> packed out, dgbmv(5) + "
                                   "tridiagonal JW step (jw_type 13)", "rhs_per_gpu": N_CPLX},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": info[0], "kind": "port", "sample": info[1]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def gpu_arm(args, rank, world):
    import torch
    import torch.distributed as dist

    from pfsolve_b200 import replicas
    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App, append_chain, last_launch, launch_count

    nc = args.ncplx
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wl = WL.config2(seed=1 + rank, B=nc)
    M = wl.M
    tA = torch.from_numpy(wl.dgbmv).to(dev)
    tb = torch.from_numpy(wl.jw_bands).to(dev)
    rhs = torch.from_numpy(wl.rhs).to(dev)  # XXII, 1 GiB
    out = torch.empty(2 * M * nc, dtype=torch.float64, device=dev)
    del wl
    dg = App(device=local, buffer=tA, outputBuffer=rhs, M_size=M, size=(M, 2 * nc), LDA=5, KU=2, KL=2,
             doublePrecision=1)
    jw = App(device=local, buffer=tb, outputBuffer=rhs, M_size=M, size=(M, 2 * nc), upperBanded=2, jw_type=13,
             doublePrecision=1, scaleC=1.0, rowsPerThread=args.rows, kernelPath=args.path)
    bl = App(device=local, buffer=rhs, outputBuffer=out, M_size=M, size=(M, nc), block=7, doublePrecision=1)
    lps = [dg.launch_params(), jw.launch_params(), bl.launch_params()]
    apps = [dg, jw, bl]

    def step():
        append_chain(apps, lps)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    n0 = launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = launch_count() - n0
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    # the kernel instance that ran, and a spread sample of the last timed
    # step's output (checked against the oracle in the CPU leg below)
    kinfo = last_launch()
    ys = spread_sample(nc, max(1, kinfo["gridCTAs"] * kinfo["groupsPerCTA"]))
    ys_t = torch.from_numpy(ys).to(dev)
    snap_out = out.view(nc, M, 2)[ys_t].cpu().numpy()
    snap_in = rhs.view(nc, 2, M)[ys_t].cpu().numpy()
    ms_max = replicas.max_over_ranks(ms, dev)
    value = replicas.job_throughput(nc, ms_max, world)
    bytes_alg = 2.0 * M * 16 * nc + (5 + 3) * M * 8
    achieved = bytes_alg / (ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    # DRAM bytes (read + write) of one full-size launch of this kernel, from a
    # single-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) at
    # 32768 systems scaled to 65536 (reads in proportion: 1.074 GB; writes the
    # same less the output tail still in L2 at kernel end: ~1.02 GB).
    traffic = 2.09e9 if (nc == N_CPLX and jw.shape()["streaming"] == 1) else None

    # ---- e2e through the C ABI with host buffers (pinned), copies inside the timed region
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_case": True, "ncplx": nc, "ms_per_step": ms_max, "gbs": achieved,
                              "gpu_launches": int(launches), "kernel": jw.shape()}), flush=True)
        return
    # Double-buffered on three streams, in chunks: each step's systems are cut
    # into CH chunks, each copied in (PCIe up), solved and copied out (PCIe
    # down) on its own, so the two directions overlap chunk by chunk and the
    # pipeline fills and drains in a chunk rather than a whole step.  Every
    # step still copies its whole input in and its whole result out inside
    # the timed region.
    CH = 8 if nc % 8 == 0 else 1
    ncc = nc // CH  # complex systems per chunk
    host_in = torch.empty(2 * M * nc, dtype=torch.float64, pin_memory=True)
    host_in.copy_(rhs.cpu())
    host_out = [torch.empty(2 * M * nc, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    dev_in = [rhs, torch.empty_like(rhs)]
    dev_out = [out, torch.empty_like(out)]
    s_up, s_comp, s_down = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    dg_e = App(device=local, stream=s_comp.cuda_stream, buffer=tA, outputBuffer=rhs, M_size=M, size=(M, 2 * ncc),
               LDA=5, KU=2, KL=2, doublePrecision=1)
    jw_e = App(device=local, stream=s_comp.cuda_stream, buffer=tb, outputBuffer=rhs, M_size=M, size=(M, 2 * ncc),
               upperBanded=2, jw_type=13, doublePrecision=1, scaleC=1.0, rowsPerThread=args.rows,
               kernelPath=args.path)
    bl_e = App(device=local, stream=s_comp.cuda_stream, buffer=rhs, outputBuffer=out, M_size=M, size=(M, ncc),
               block=7, doublePrecision=1)
    apps_e = [dg_e, jw_e, bl_e]
    span = 2 * M * ncc  # doubles of one chunk, in and out

    def piece(t, c):
        return t[c * span:(c + 1) * span]

    lps_e = [[[dg_e.launch_params(outputBuffer=piece(dev_in[b], c)), jw_e.launch_params(outputBuffer=piece(dev_in[b], c)),
               bl_e.launch_params(buffer=piece(dev_in[b], c), outputBuffer=piece(dev_out[b], c))] for c in range(CH)]
             for b in range(2)]
    ev_up = [[torch.cuda.Event() for _ in range(CH)] for _ in range(2)]
    ev_comp = [[torch.cuda.Event() for _ in range(CH)] for _ in range(2)]
    ev_down = [[torch.cuda.Event() for _ in range(CH)] for _ in range(2)]

    def e2e_step(k):
        b = k & 1
        for c in range(CH):
            s_up.wait_event(ev_comp[b][c])  # the solve of step k-2 has read this chunk of dev_in[b]
            with torch.cuda.stream(s_up):
                piece(dev_in[b], c).copy_(piece(host_in, c), non_blocking=True)
            ev_up[b][c].record(s_up)
            s_comp.wait_event(ev_up[b][c])
            s_comp.wait_event(ev_down[b][c])  # the D2H of step k-2 has read this chunk of dev_out[b]
            append_chain(apps_e, lps_e[b][c])
            ev_comp[b][c].record(s_comp)
            s_down.wait_event(ev_comp[b][c])
            with torch.cuda.stream(s_down):
                piece(host_out[b], c).copy_(piece(dev_out[b], c), non_blocking=True)
            ev_down[b][c].record(s_down)

    e_steps = max(4, min(args.steps, 10))
    for k in range(2):
        e2e_step(k)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s_up)
    for k in range(e_steps):
        e2e_step(k)
    t1.record(s_down)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1) / e_steps
    e2e_value = replicas.job_throughput(nc, replicas.max_over_ranks(e2e_ms, dev), world)
    for a in apps_e:
        a.close()

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu:
        parity = parity_check(snap_in, snap_out, tA.cpu().numpy(), tb.cpu().numpy(), M, ys)
        v, cores, desc = cpu_reference_sample(target_s=12.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": desc,
               "variants": cpu_reference_variants()}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded, N(0,1) complex RHS, dominant tridiagonal, U(-1,1) 5-band)",
                "config": {"workload": "config2: N=1024, 65536 complex RHS per GPU, XXII in -> packed out, "
                                       "dgbmv(5) + tridiagonal JW step (jw_type 13) fused, one kernel per step",
                           "rhs_per_gpu": nc, "l2": "inputs 2 GiB > L2, no flush", "kernel": jw.shape(),
                           "kernel_instance": kinfo,
                           "parallelism": f"replicas x{world} (independent RHS shards, no collective)"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                             "bytes_per_launch": bytes_alg},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * M * nc * 8,
                        "d2h_bytes_per_step": 2 * M * nc * 8, "steps": e_steps, "ms_per_step": e2e_ms,
                        "pipeline": f"pinned host buffers; H2D, fused kernel and D2H on three streams, "
                                    f"double-buffered, {CH} chunks per step: each chunk's upload overlaps the "
                                    f"previous chunks' downloads", "chunks_per_step": CH},
                "gpu_launches": int(launches), "clocks": clocks, "cpu_baseline": cpu, "parity": parity}
        if not args.no_extras and world == 1:
            line["extras"] = extras_arm(args)
        print(json.dumps(line), flush=True)


def extras_arm(args):
    """Other parts of the metric, measured on the same GPU: config 3 (N=512,
    131072 real RHS, weakly dominant) in FP64 and in mixed precision (FP32
    solve + 2 FP64 refinement sweeps) with the mixed result's error against
    FP64, config 4 (one spectral timestep, l = 0..511, one persistent
    launch, captured CUDA graph, autotuned shape), K = 2 and 4 consecutive
    steps in one launch, a long system (N = 16384) and the config 5 serving
    loop."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App, Batch
    out = {}
    wl = WL.config3()
    M, B = wl.M, wl.nrhs
    tb = torch.from_numpy(wl.jw_bands).cuda()
    base = torch.from_numpy(wl.rhs).cuda()
    bytes_alg = 2.0 * M * 8 * B + 3 * M * 8
    res = {}
    for name, refine in (("fp64", 0), ("mixed", 2)):
        x = base.clone()
        app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1,
                  scaleC=1.0, mixedPrecisionRefinement=refine)
        app.append()
        torch.cuda.synchronize()
        res[name] = x.clone()
        for _ in range(3):
            app.append()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            app.append()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        out[f"config3_{name}"] = {"rhs_per_s": B / (ms * 1e-3), "ms": ms, "gbs": bytes_alg / (ms * 1e-3) / 1e9}
        app.close()
        del x
    d = (res["mixed"] - res["fp64"]).view(B, M).norm(dim=1) / res["fp64"].view(B, M).norm(dim=1)
    out["config3_mixed_vs_fp64_rel_l2_max"] = float(d.max().item())
    out["config3_mixed_speedup"] = out["config3_fp64"]["ms"] / out["config3_mixed"]["ms"]
    # the same system and right-hand sides on FP32 storage (8-byte rows: 4 bytes
    # in, 4 out): the reference's default precision (FP32 arithmetic) and
    # doublePrecisionFloatMemory (FP64 arithmetic); error against the FP64 result
    tb32 = tb.float()
    base32 = base.float()
    bytes32 = 2.0 * M * 4 * B + 3 * M * 4
    for name, dpfm in (("f32", 0), ("f32mem", 1)):
        x = base32.clone()
        app = App(buffer=tb32, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=0,
                  doublePrecisionFloatMemory=dpfm, scaleC=1.0)
        app.append()
        torch.cuda.synchronize()
        err = ((x.double() - res["fp64"]).view(B, M).norm(dim=1) / res["fp64"].view(B, M).norm(dim=1)).max().item()
        for _ in range(3):
            app.append()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            app.append()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        out[f"config3_{name}"] = {"rhs_per_s": B / (ms * 1e-3), "ms": ms, "gbs": bytes32 / (ms * 1e-3) / 1e9,
                                  "rel_l2_vs_fp64_max": err, "kernel": app.shape(),
                                  "speedup_vs_fp64": out["config3_fp64"]["ms"] / ms}
        app.close()
        del x
    del res, base, base32, tb32
    out["config1_latency"] = config1_measure()
    step = WL.config4()
    dev = torch.device("cuda")
    inp = torch.from_numpy(step.rhs).to(dev)
    outb = torch.zeros_like(inp)
    keep, entries = [], []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tj = torch.from_numpy(step.jw_bands[k]).to(dev)
        ta = torch.from_numpy(step.dgbmv[k]).to(dev)
        keep += [tj, ta]
        off = int(step.rhs_offsets[k])
        entries.append(dict(M=int(N), nsys=int(ns), bands=tj, dgbmvBands=ta, input=inp.data_ptr() + 8 * off,
                            output=outb.data_ptr() + 8 * off, inputStride=int(N), outputStride=int(N),
                            lshift=int(l), scaleS=step.scale_s, scaleC=1.0))
    batch = Batch(entries, upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    st = torch.cuda.Stream()
    batch.autotune(st, iterations=3)
    batch.capture(st)
    for _ in range(3):
        batch.append(st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(10):
        batch.append(st)
    e1.record(st)
    st.synchronize()
    ms = e0.elapsed_time(e1) / 10
    rows = int((step.Ns * step.nsys).sum())
    out["config4_uneven_step"] = {"complex_rhs_per_s": int(step.nsys.sum()) / (ms * 1e-3), "ms": ms,
                                  "gbs": 2.0 * rows * 16 / (ms * 1e-3) / 1e9, "shape": batch.shape(),
                                  "graph": True,
                                  "launches_per_step": 2 if batch.shape()["rowsPerThread"] == 0 else 1}
    batch.close()
    del inp, outb, keep
    torch.cuda.empty_cache()
    # K consecutive steps in one launch (numConsecutiveJWIterations)
    for K in (2, 4):
        out[f"ksteps_K{K}_ub1_t10_N512_B131072"] = ksteps_measure(512, 131072, K, steps=10, warmup=3)
    torch.cuda.empty_cache()
    # long systems, beyond one CTA group (the reference's multi-upload range)
    out["long_t13_N16384_B8192"] = long_measure(16384, 8192)
    out["long_t13_N16384_B8192_single_pass"] = long_measure(16384, 8192, path=4)
    out["long_t13_N65536_B2048"] = long_measure(65536, 2048)
    out["long_t13_N20000_B6553"] = long_measure(20000, 6553)
    out["dct2_N512_B131072"] = dct_measure(512, 131072, 2)
    out["dct3_N512_B131072"] = dct_measure(512, 131072, 3)
    out["dct2_N4096_B16384"] = dct_measure(4096, 16384, 2)
    out["alt_t113_N1024_B131072"] = alt_measure(1024, 131072)
    out["alt_t113_N1024_B131072_group"] = alt_measure(1024, 131072, path=1)
    torch.cuda.empty_cache()
    out["config5_serving"] = serving_leg()
    # each HBM-bound entry's fraction of the measured HBM peak
    peak, kind = peaks()
    for v in out.values():
        if isinstance(v, dict) and "gbs" in v and "note" not in v:
            v["hbm_frac"] = v["gbs"] / peak
            v["hbm_peak_kind"] = kind
    return out


def config1_measure(steps=200, warmup=20):
    """Config 1 (the test-1 form: N = 256, 512 real RHS, a 3-band dgbmv
    fused ahead of the upper-bidiagonal JW step, jw_type 13, upperBanded 0),
    and the JW step alone as the reference times it: per-step latency of
    back-to-back launches on one stream (CUDA events over `steps` launches
    after `warmup`; 2.1 MB of right-hand sides, L2-resident).  Each is timed
    twice: called from Python through the C ABI one launch at a time (host
    overhead included), and as `steps` launches captured once in a CUDA graph
    and replayed (device time per launch)."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App, append_chain
    wl = WL.config1()
    M, B = wl.M, wl.nrhs
    tA = torch.from_numpy(wl.dgbmv).cuda()
    tb = torch.from_numpy(wl.jw_bands).cuda()
    tr = torch.from_numpy(wl.rhs.copy()).cuda()
    st = torch.cuda.Stream()
    dg = App(buffer=tA, outputBuffer=tr, M_size=M, size=(M, B), LDA=3, KU=1, KL=1, doublePrecision=1,
             stream=st.cuda_stream)
    jw = App(buffer=tb, outputBuffer=tr, M_size=M, size=(M, B), upperBanded=0, jw_type=13, doublePrecision=1,
             scaleC=1.0, stream=st.cuda_stream)
    lps = [dg.launch_params(), jw.launch_params()]
    res = {}
    for name, fn in (("fused_chain", lambda: append_chain([dg, jw], lps)), ("jw_only", lambda: jw.append(lps[1]))):
        with torch.cuda.stream(st):
            for _ in range(warmup):
                fn()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            st.synchronize()
            e0.record(st)
            for _ in range(steps):
                fn()
            e1.record(st)
        st.synchronize()
        ms = e0.elapsed_time(e1) / steps
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            for _ in range(steps):
                fn()
        with torch.cuda.stream(st):  # a graph replays on the current stream
            for _ in range(3):
                g.replay()
            st.synchronize()
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(st)
            for _ in range(5):
                g.replay()
            g1.record(st)
        st.synchronize()
        gms = g0.elapsed_time(g1) / (5 * steps)
        del g
        res[name] = {"ms": ms, "rhs_per_s": B / (ms * 1e-3), "gbs": 2.0 * M * 8 * B / (ms * 1e-3) / 1e9,
                     "graph_ms": gms, "graph_rhs_per_s": B / (gms * 1e-3)}
    dg.close()
    jw.close()
    res["reference_jw_ms"] = 0.0042  # its own JW kernel on the same pool: 20 launches from C++, no graph
    res["note"] = ("L2-resident (2.1 MB): latency of back-to-back launches, not an HBM roofline; ms from Python "
                   "calls (host overhead included), graph_ms from a replayed CUDA graph of the same launches")
    return res


def serving_leg(rate=20000.0, duration_s=1.5, pool=256, warm=2000):
    """Config 5: Poisson arrivals at `rate` of JW-step requests (N log-uniform
    in [32, 1024], RHS log-uniform in [1, 4096], 80 % mixed precision, 20 %
    double-double storage) through the serving engine; inputs device-resident
    (a pool of `pool` distinct requests, reused cyclically).  Latency = submit
    -> completion on the GPU, per request."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.serving import Server, run_load
    specs = WL.config5_requests(pool, seed=4)
    srv = Server(hbm_budget_bytes=16 << 30, streams=8, max_batch_requests=32, refine_sweeps=2)
    ops, templ = {}, []
    g = torch.Generator(device="cuda").manual_seed(4)
    keep = []
    for sp in specs:
        if sp.M not in ops:
            tb = torch.from_numpy(WL.serve_operator_bands(np.random.default_rng(sp.M), sp.M)).cuda()
            keep.append(tb)
            ops[sp.M] = srv.add_operator(sp.M, tb)
        x = torch.rand(sp.M * sp.nrhs, dtype=torch.float64, device="cuda", generator=g) * 2 - 1
        if sp.precision == 2:
            x = torch.stack([x, torch.zeros_like(x)], -1).reshape(-1)
        templ.append((ops[sp.M], sp.precision, sp.nrhs, x, torch.empty_like(x)))
    run_load(srv, [templ[i % pool] for i in range(warm)], WL.poisson_arrivals(warm, rate, seed=5))
    n = int(rate * duration_s)
    reqs = [templ[i % pool] for i in range(n)]
    st0 = srv.stats()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    lat, wall, lag = run_load(srv, reqs, WL.poisson_arrivals(n, rate, seed=4))
    clocks = sampler.stop()
    st1 = srv.stats()
    srv.close()
    lat_all = np.asarray(lat)
    prec = np.asarray([r[1] for r in reqs])
    slow = [dict(M=int(specs[i % pool].M), nrhs=int(reqs[i][2]), precision=int(reqs[i][1]), ms=float(lat_all[i]))
            for i in np.argsort(-lat_all)[:8]]
    by_prec = {("mixed" if p == 1 else "dd"): {"p50_ms": float(np.percentile(lat_all[prec == p], 50)),
                                               "p99_ms": float(np.percentile(lat_all[prec == p], 99))}
               for p in (1, 2) if (prec == p).any()}
    lat = np.sort(lat_all)
    rhs = sum(r[2] for r in reqs)
    nbytes = sum(r[3].numel() * 8 * 2 for r in reqs)
    return {"requests": n, "offered_rate_per_s": rate, "achieved_rate_per_s": n / wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat[-1]), "rhs_per_s": rhs / wall, "hbm_gbs_offered": nbytes / wall / 1e9,
            "batches": st1["batches"] - st0["batches"], "submitter_max_lag_ms": 1e3 * lag,
            "server_p99_queue_ms": st1["p99QueueMs"], "server_p99_device_ms": st1["p99DeviceMs"], "clocks": clocks,
            "by_precision": by_prec, "slowest": slow,
            "mix": "80% mixed (FP32 solve + 2 FP64 refinement sweeps), 20% double-double storage",
            "streams": 8, "max_batch_requests": 32, "hbm_budget_bytes": 16 << 30}


def config3_profile(args):
    """Profiling case: config 3 (N = 512 real tridiagonal, weakly dominant),
    `--ncplx` systems, FP64 or mixed precision (`--refine`), or FP32 storage
    (`--prec f32` / `f32mem`), K timed steps; prints one JSON line with the
    kernel time."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App
    wl = WL.config3(M=args.m, B=args.ncplx)
    M, B = wl.M, wl.nrhs
    tb = torch.from_numpy(wl.jw_bands).cuda()
    x = torch.from_numpy(wl.rhs).cuda()
    prec = dict(doublePrecision=1)
    es = 8
    if args.prec != "f64":  # FP32 storage: FP32 arithmetic, or FP64 arithmetic (doublePrecisionFloatMemory)
        tb, x, es = tb.float(), x.float(), 4
        prec = dict(doublePrecision=0, doublePrecisionFloatMemory=1 if args.prec == "f32mem" else 0)
    app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, scaleC=1.0,
              mixedPrecisionRefinement=args.refine, rowsPerThread=args.rows, kernelPath=args.path,
              stagingBuffers=args.staging, **prec)
    for _ in range(max(1, args.warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"profile_case": "config3", "M": M, "rhs": B, "refine": args.refine, "prec": args.prec,
                      "ms_per_step": ms, "gbs": 2.0 * M * es * B / (ms * 1e-3) / 1e9, "kernel": app.shape()}),
          flush=True)
    app.close()


def long_measure(M, B, steps=10, warmup=3, path=0):
    """A long tridiagonal system (config 3's coefficients at N = M rows), B
    real right-hand sides in place, FP64: the plan's default long-system
    kernel (path 3: two passes only; 4: the single pass only; 2: the cluster
    kernel).  Algorithmic bytes: M rows read and written per system."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App
    wl = WL.config3(M=M, B=B)
    tb = torch.from_numpy(wl.jw_bands).cuda()
    x = torch.from_numpy(wl.rhs).cuda()
    app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=1,
              scaleC=1.0, kernelPath=path)
    for _ in range(max(1, warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    shape = app.shape()
    app.close()
    del x, tb
    return {"M": M, "rhs": B, "ms": ms, "rhs_per_s": B / (ms * 1e-3), "gbs": 2.0 * M * 8 * B / (ms * 1e-3) / 1e9,
            "kernel": shape}


def dct_measure(N, B, dct_type=2, steps=10, warmup=3):
    """The DCT step (performDCT 2 or 3): B rows of N points, FP64, out of
    place; algorithmic bytes: each row read once and written once."""
    import torch

    from pfsolve_b200.api import App
    rng = np.random.default_rng(5)
    x = torch.from_numpy(rng.standard_normal(N * B)).cuda()
    y = torch.empty_like(x)
    app = App(buffer=x, outputBuffer=y, FFTdim=1, size=(N, B), performDCT=dct_type, doublePrecision=1)
    for _ in range(max(1, warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    app.close()
    del x, y
    return {"N": N, "rows": B, "type": dct_type, "ms": ms, "rows_per_s": B / (ms * 1e-3),
            "gbs": 2.0 * N * 8 * B / (ms * 1e-3) / 1e9}


def alt_measure(M, B, steps=10, warmup=3, path=0, rows=0):
    """ALT stride-2 mode (jw_type 113: the even and the odd rows of each row
    set are two tridiagonal systems), M rows per row set, B real row sets in
    place, FP64: the streaming kernel (path 1: the group kernel).  Algorithmic
    bytes: M rows read and written per row set."""
    import numpy as np
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App
    rng = np.random.default_rng(4242)
    tb = torch.from_numpy(WL.alt_bands(rng, M, 2)).cuda()
    x = torch.from_numpy(rng.uniform(-1, 1, M * B)).cuda()
    app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=113, doublePrecision=1,
              scaleC=1.0, kernelPath=path, rowsPerThread=rows)
    for _ in range(max(1, warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    shape = app.shape()
    app.close()
    del x, tb
    return {"M": M, "rhs": B, "ms": ms, "rhs_per_s": B / (ms * 1e-3), "gbs": 2.0 * M * 8 * B / (ms * 1e-3) / 1e9,
            "kernel": shape}


def dd_profile(args):
    """Profiling case: config 3's weakly dominant tridiagonal system (N = --m)
    in double-double, --ncplx right-hand sides: {hi, lo} storage
    (quadDoubleDoublePrecision), or with --refine 1 double-double arithmetic
    on FP64 storage (quadDoubleDoublePrecisionDoubleMemory).  Prints one JSON
    line with the kernel time, the storage GB/s and the double-double FLOP
    rate in FP64 operations (about 20 FP64 operations per double-double
    multiply-add)."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App

    def to_dd(a):  # FP64 values -> double-double {hi, lo = 0} pairs
        return np.stack([a, np.zeros_like(a)], -1).ravel()
    wl = WL.config3(M=args.m, B=args.ncplx)
    M, B = wl.M, wl.nrhs
    f64mem = args.refine == 1
    bands = wl.jw_bands if f64mem else to_dd(wl.jw_bands)
    rhs = wl.rhs if f64mem else to_dd(wl.rhs)
    tb = torch.from_numpy(bands).cuda()
    x = torch.from_numpy(rhs).cuda()
    mode = dict(quadDoubleDoublePrecisionDoubleMemory=1) if f64mem else dict(quadDoubleDoublePrecision=1)
    app = App(buffer=tb, outputBuffer=x, M_size=M, size=(M, B), upperBanded=2, jw_type=13, doublePrecision=0,
              scaleC=1.0, rowsPerThread=args.rows, **mode)
    for _ in range(max(1, args.warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    word = 8 if f64mem else 16
    print(json.dumps({"profile_case": "dd", "storage": "f64" if f64mem else "dd", "M": M, "rhs": B,
                      "ms_per_step": ms, "gbs": 2.0 * M * word * B / (ms * 1e-3) / 1e9,
                      "rhs_per_s": B / (ms * 1e-3), "kernel": app.shape()}), flush=True)
    app.close()


def ksteps_measure(M, B, K, steps=20, warmup=5, rows=0, path=0):
    """K consecutive JW steps in one launch (upperBanded 1, jw_type 10:
    bidiagonal matvec + lower bidiagonal solve per step, per-step band
    buffers), N = M rows, B systems (inputs > L2, no flush); K = 1 runs the
    single-step kernel on the same operator.  Algorithmic bytes: M rows read
    and M - K + 1 written per system."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import App
    rng = np.random.default_rng(5)
    bands = WL.steps_bands(rng, M, 1, max(K, 2))[:max(K, 1)]
    tbs = [torch.from_numpy(b).cuda() for b in bands]
    x = torch.from_numpy(rng.uniform(-1, 1, M * B)).cuda()
    extra = dict(numConsecutiveJWIterations=K, useMultipleInputBuffers=K) if K > 1 else {}
    app = App(buffer=tbs if K > 1 else tbs[0], outputBuffer=x, M_size=M, size=(M, B), upperBanded=1, jw_type=10,
              doublePrecision=1, scaleC=1.0, rowsPerThread=rows, kernelPath=path, **extra)
    for _ in range(max(1, warmup)):
        app.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        app.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    shape = app.shape()
    app.close()
    del x, tbs
    mout = M - K + 1
    return {"M": M, "rhs": B, "K": K, "ms": ms, "rhs_per_s": B / (ms * 1e-3),
            "gbs": (M + mout) * 8 * B / (ms * 1e-3) / 1e9, "kernel": shape}


def steps_profile(args):
    """Profiling case: K steps in one launch (--m rows, --ncplx systems,
    --ksteps K, --path 1 for the K-step partition kernel).  Prints one JSON line."""
    r = ksteps_measure(args.m, args.ncplx, args.ksteps, args.steps, args.warmup, args.rows, args.path)
    print(json.dumps(dict(profile_case="ksteps", ms_per_step=r.pop("ms"), **r)), flush=True)


def config4_profile(args):
    """Profiling case: config 4 (one spectral timestep, degrees l = 0..--lmax),
    one persistent uneven-batch launch per step (no graph), K timed steps."""
    import torch

    from pfsolve_b200 import workloads as WL
    from pfsolve_b200.api import Batch
    step = WL.config4(lmax=args.lmax)
    inp = torch.from_numpy(step.rhs).cuda()
    outb = torch.zeros_like(inp)
    keep, entries = [], []
    for k, (l, N, ns) in enumerate(zip(step.ls, step.Ns, step.nsys)):
        tj = torch.from_numpy(step.jw_bands[k]).cuda()
        ta = torch.from_numpy(step.dgbmv[k]).cuda()
        keep += [tj, ta]
        off = int(step.rhs_offsets[k])
        entries.append(dict(M=int(N), nsys=int(ns), bands=tj, dgbmvBands=ta, input=inp.data_ptr() + 8 * off,
                            output=outb.data_ptr() + 8 * off, inputStride=int(N), outputStride=int(N),
                            lshift=int(l), scaleS=step.scale_s, scaleC=1.0))
    desc = dict(upperBanded=0, jw_type=13, LDA=3, KU=1, KL=1, block=307)
    if args.rows:
        desc["rowsPerThread"] = args.rows
    batch = Batch(entries, **desc)
    for _ in range(max(1, args.warmup)):
        batch.append()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        batch.append()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    rows = int((step.Ns * step.nsys).sum())
    print(json.dumps({"profile_case": "config4", "lmax": args.lmax, "ms_per_step": ms,
                      "gbs": 2.0 * rows * 16 / (ms * 1e-3) / 1e9, "shape": batch.shape()}), flush=True)
    batch.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ncplx", type=int, default=N_CPLX, help="complex RHS per GPU (profiling cases only)")
    ap.add_argument("--profile", action="store_true", help="kernel steps only: no e2e leg, no CPU baseline")
    ap.add_argument("--rows", type=int, default=0, help="rows per thread (0: the plan's default)")
    ap.add_argument("--staging", type=int, default=0,
                    help="config 3 profiling case: TMA staging buffers per group (stagingBuffers; 0: default)")
    ap.add_argument("--no-extras", action="store_true", help="skip the config 3 / config 4 measurements")
    ap.add_argument("--serve", action="store_true", help="only the serving leg (config 5); prints its JSON")
    ap.add_argument("--workload", default="config2",
                    choices=["config2", "config3", "config4", "ksteps", "dd", "alt", "dct"],
                    help="profiling case (--profile): the config 2 chain, config 3 (--ncplx real systems), "
                         "config 4 (degrees 0..--lmax), K steps, config 3's system in double-double, or ALT mode "
                         "(--m rows per row set, --ncplx row sets)")
    ap.add_argument("--lmax", type=int, default=511, help="config 4 profiling case: highest harmonic degree")
    ap.add_argument("--m", type=int, default=512, help="config 3 / K-step profiling case: rows per system")
    ap.add_argument("--ksteps", type=int, default=4, help="K-step profiling case: consecutive steps")
    ap.add_argument("--refine", type=int, default=0, help="config 3 profiling case: mixed-precision sweeps (0: FP64)")
    ap.add_argument("--prec", default="f64", choices=["f64", "f32", "f32mem"],
                    help="config 3 profiling case: FP64 storage, or FP32 storage with FP32 or FP64 arithmetic")
    ap.add_argument("--path", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="kernelPath: 0 streaming kernel where possible (long systems: two passes, the single "
                         "pass for unaligned rows), 1 group kernel only, 2 long systems on the cluster "
                         "kernel, 3 long systems in two passes only, 4 long systems in the single pass only")
    args = ap.parse_args()
    if args.profile:
        args.no_cpu = True
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    if args.serve:
        print(json.dumps({"config5_serving": serving_leg()}), flush=True)
        return
    if args.profile and args.workload == "config3":
        config3_profile(args)
        return
    if args.profile and args.workload == "config4":
        config4_profile(args)
        return
    if args.profile and args.workload == "dd":
        dd_profile(args)
        return
    if args.profile and args.workload == "ksteps":
        steps_profile(args)
        return
    if args.profile and args.workload == "dct":
        print(json.dumps(dict(profile_case="dct", **dct_measure(args.m, args.ncplx, 2 if args.refine == 0 else 3,
                                                                 steps=args.steps, warmup=args.warmup))), flush=True)
        return
    if args.profile and args.workload == "alt":
        print(json.dumps(alt_measure(args.m, args.ncplx, steps=args.steps, warmup=args.warmup, path=args.path,
                                     rows=args.rows)),
              flush=True)
        return
    try:
        if args.impl == "reference":
            reference_arm(args, rank, world)
        else:
            gpu_arm(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
