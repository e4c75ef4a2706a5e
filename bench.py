#!/usr/bin/env python
"""Benchmark of the B200 circulant-embedding path.

Workload (one step = one realization): 3D Matern nu=1.5 (`matern32`), sigma^2=1,
axiparallel correlation lengths (0.2, 0.1, 0.05) on [0,1]^3 with 256^3 cells,
embedding factor 2 (512^3 torus).  FP64 spectrum (built once, untimed), FP32
realizations with seeded on-device noise.  Metric: field cells/s.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

--impl reference times the FP64 CPU restatement of the reference's algorithm
(oracle/) on the host cores (the reference itself needs FFTW-MPI, MPI and
dune-common, which this image lacks).  Under torchrun each rank runs an
independent replica (no data-path collective); rank 0 prints one JSON line.
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
sys.path.insert(0, os.path.join(ROOT, "parafields-core_b200"))

WORKLOAD = dict(dim=3, cells=(256, 256, 256), covariance="matern32", variance=1.0,
                corr_length=(0.2, 0.1, 0.05), anisotropy="axiparallel", embedding_factor=2,
                approximate=True)
METRIC = "field cells/s (3D Matern-3/2 256^3 realization, 512^3 torus)"
CONFIG = {"workload": "3d-matern32-axiparallel-256^3-factor2-fp32-realizations",
          "cells": [256, 256, 256], "torus": [512, 512, 512], "spectrum": "fp64 DCT-I (untimed, once)",
          "embedding.approximate": "true (the factor-2 embedding has 15269 eigenvalues below -1e-14, "
                                   "min -7.3e-8, which the reference clamps only with this key set)",
          "noise": "counter-based Philox4x32-10 on device (one call per frequency pair k, k+T/2), seed per step",
          "planning": "pf_plan_autotune before the timed region; K realizations per pf_generate_batch call",
          "l2": "no flush: per-step traffic ~1 GB through intermediates of 269 MB and 135 MB (> 126 MB L2)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def realization_work(cells, torus):
    """Compulsory HBM bytes and FFT flops of one FP32 realization with in-register noise
    (per-unit figures of the measurement plan): bytes = sqrt(lambda) on the prod(T/2+1) DCT
    cells (FP32) + the field (FP32); flops = 2.5 N log2 N for the real 3D transform of the
    torus, N = prod(T).  Also, per pass of the pruned three-pass schedule the library runs,
    the bytes that pass cannot avoid (each input read once from HBM, each output written
    once) and its flops (complex pencils: 5 L log2 L; the final complex-to-real rows:
    2.5 L log2 L):
      gen_noise_last  sqrt(lambda) on the DCT cells (mirrored reads of a cell are L2 hits)
                      + the (T0/2+1) T1 n2 complex64 planes it keeps
      gen_c2c_d1      those planes in + (T0/2+1) n1 n2 complex64 out
      gen_c2r_d0      that array in + the n0 n1 n2 FP32 field out"""
    import math
    t0, t1, t2 = torus
    n0, n1, n2 = cells
    N = t0 * t1 * t2
    c0 = t0 // 2 + 1
    sq = c0 * (t1 // 2 + 1) * (t2 // 2 + 1) * 4
    out = n0 * n1 * n2 * 4
    w1 = c0 * t1 * n2 * 8
    w2 = c0 * n1 * n2 * 8
    c = lambda L: 5.0 * L * math.log2(L)  # noqa: E731
    passes = {"gen_noise_last": c0 * t1 * c(t2),   # last axis, every pencil of the half spectrum
              "gen_c2c_d1": c0 * n2 * c(t1),       # axis 1 on the n2 kept planes
              "gen_c2c_d1_tma": c0 * n2 * c(t1),
              "gen_c2r_d0": n1 * n2 * 0.5 * c(t0),  # complex-to-real rows of the kept cells
              "gen_c2r_d0_bulk": n1 * n2 * 0.5 * c(t0)}
    pass_bytes = {"gen_noise_last": sq + w1, "gen_c2c_d1": w1 + w2, "gen_c2r_d0": w2 + out}
    schedule = sum(pass_bytes.values())
    pass_bytes["gen_c2c_d1_tma"] = pass_bytes["gen_c2c_d1"]  # the same pass, TMA-staged tiles
    pass_bytes["gen_c2r_d0_bulk"] = pass_bytes["gen_c2r_d0"]  # the same pass, rows staged by bulk copies
    return {"compulsory_bytes": sq + out, "flops": 2.5 * N * math.log2(N), "pass_flops": passes,
            "pass_bytes": pass_bytes, "schedule_bytes": schedule}


def ncu_traffic():
    """per-launch DRAM bytes of each kernel from the committed ncu summary, if any"""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    out = {}
    if os.path.exists(p):
        for line in open(p):
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#"):
                out[parts[0]] = float(parts[1])
    return out


class ClockSampler:
    """nvidia-smi sampling during the timed region (clocks + throttle reasons)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = f"/tmp/pf_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path).read().strip().splitlines()]
            sm = [float(r[0]) for r in rows]
            mx = float(rows[0][1])
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].strip() == "Active"})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(sm)}
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def dist_setup(n):
    import torch
    import torch.distributed as dist
    if n > 1 or "WORLD_SIZE" in os.environ:
        rank = int(os.environ.get("RANK", 0))
        local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        return rank, dist.get_world_size(), local
    return 0, 1, 0


def replica_seed(rank):
    """Base seed of one replica's realizations: every rank generates its own, distinct fields."""
    return 1000003 * (rank + 1)


def max_over_ranks(value, world, device):
    """The slowest rank's value (every rank takes part in the reduction)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, units, steps, seconds):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units * steps / seconds


def cpu_oracle_realization(threads):
    """One FP64 realization of the workload with the CPU restatement (spectrum and noise
    untimed).  Returns its time, the cell count, the noise buffer (reference draw order)
    and the field, so the same noise can be fed to the GPU and the result checked."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import pfb200
    O.set_threads(threads)
    d = pfb200.make_desc(**WORKLOAD)
    g = O.resolve(d)
    lam, _, _ = O.spectrum(d)
    noise = O.noise(20261203, g.noise)
    t0 = time.perf_counter()
    field, _ = O.generate(d, lam, noise)
    return time.perf_counter() - t0, g.domain, noise, field, lam


def cpu_oracle_field(noise, lam, desc_kw=WORKLOAD):
    """the oracle's FP64 realization of a workload from a given noise buffer"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import pfb200
    field, _ = O.generate(pfb200.make_desc(**desc_kw), lam, noise)
    return field


def cpu_scipy_realization(threads, lam, noise, cells=WORKLOAD["cells"]):
    """The same realization with scipy.fft (pocketfft, `workers` threads) for the transform:
    eigenvalue-scaled half spectrum (the oracle's noise and eigenvalues, R2C layout with the
    DCT mirror and the transposed 3D storage order), one irfftn over the torus (2 cells per
    cell and axis), extraction of the domain.  A library-grade CPU reference point for the
    transform, timed as the oracle is."""
    import scipy.fft as sf
    n = cells
    t = [2 * c for c in n]
    c0 = t[0] // 2 + 1
    D = [x // 2 + 1 for x in t]
    # DCT layout, dimension 0 fastest, stored dimensions (0, 2, 1) in 3D
    sq = np.sqrt(lam.reshape(D[1], D[2], D[0])).swapaxes(0, 1)
    t0 = time.perf_counter()
    # stored frequency (k0, k1, k2) with the 3D transposed layout: noise pair index
    # k0 + c0 * (k2 + t2 * k1); eigenvalue at the mirrored DCT cell
    m1 = np.minimum(np.arange(t[1]), t[1] - np.arange(t[1]))
    m2 = np.minimum(np.arange(t[2]), t[2] - np.arange(t[2]))
    z = noise.view(np.complex128).reshape(t[1], t[2], c0).transpose(1, 0, 2)  # (k2, k1, k0)
    lamc = sq[np.ix_(m2, m1, np.arange(c0))]
    selfc = np.zeros((t[2], t[1], c0), dtype=bool)
    selfc[np.ix_([0, t[2] // 2], [0, t[1] // 2], [0, t[0] // 2])] = True
    spec = np.where(selfc, lamc * z.real, lamc * np.sqrt(0.5) * z)
    field = sf.irfftn(spec, s=(t[2], t[1], t[0]), workers=threads, norm="forward")[: n[2], : n[1], : n[0]]
    dt = time.perf_counter() - t0
    return dt, np.ascontiguousarray(field).ravel()


def run_reference(args):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import pfb200
    O.set_threads(threads)
    d = pfb200.make_desc(**WORKLOAD)
    g = O.resolve(d)
    lam, _, _ = O.spectrum(d)
    noise = O.noise(1, g.noise)
    for _ in range(args.warmup):
        O.generate(d, lam, noise)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.generate(d, lam, noise)
    dt = time.perf_counter() - t0
    v = g.domain * args.steps / dt
    line = {"metric": METRIC, "value": v, "unit": "cells/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": CONFIG,
            "cpu_baseline": {"value": v, "unit": "cells/s", "cores": threads, "kind": "port",
                             "sample": "each step = 1 full FP64 realization (c2r of the 257x512x512 half "
                                       "spectrum + extraction); noise drawn outside the timed region"},
            "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "FP64 CPU restatement of the reference algorithm (FFTW-MPI/MPI/dune-common are not "
                    "installed, so the reference itself cannot be built)"}
    print(json.dumps(line), flush=True)


def run_b200(args):
    import torch
    import pfb200
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    d = pfb200.make_desc(**WORKLOAD, precision=pfb200.PREC_F32)
    P = pfb200.Plan(d)
    P.set_stream(stream.cuda_stream)
    P.spectrum_build()
    if not args.no_tune:
        P.autotune()  # measured planning of the realization passes (outside the timed region)
    fpeaks = pfb200.measure_peaks(local) if rank == 0 else None  # CUDA-core FMA peaks (untimed)
    n = P.info.domain_size
    out = torch.empty(n, dtype=torch.float32, device=dev)
    # the K timed realizations go through one pf_generate_batch call, which alternates them
    # over two streams (one realization's noise pass overlaps the other's transform passes)
    outs = torch.empty(max(args.steps, args.warmup, 2) * n, dtype=torch.float32, device=dev)
    seed0 = replica_seed(rank)
    P.generate_batch(seed=seed0, count=max(args.warmup, 2), out=outs[: max(args.warmup, 2) * n])
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    l0 = P.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        P.generate_batch(seed=seed0 + 100, count=args.steps, out=outs[: args.steps * n])
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = P.launch_count() - l0
    # the drop-in use, one pf_generate call per realization (as RandomField::generate drives the
    # matrix), device output: reported beside the line, not the headline
    e0.record(stream)
    for i in range(args.steps):
        P.generate(seed=seed0 + 200 + i, out=out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_one = max_over_ranks(e0.elapsed_time(e1), world, dev)
    # per-kernel durations for the roofline: the same realizations one at a time (no overlap)
    P.profile(True)
    for i in range(args.steps):
        P.generate(seed=seed0 + 300 + i, out=out)
    torch.cuda.synchronize()
    prof = P.profile_read()
    P.profile(False)
    if world > 1:
        torch.distributed.barrier()
    ms = max_over_ranks(ms, world, dev)
    value = aggregate_rate(world, n, args.steps, ms / 1e3)

    # end to end through the public call with a host result buffer (D2H inside the region):
    # pf_generate_batch into pinned host memory, every realization copied to the host while
    # the next one is computed; the 67 MB copy per realization over PCIe bounds this figure
    ke = max(4, min(args.steps, 16))
    hp = torch.empty(ke * n, dtype=torch.float32).pin_memory().numpy()
    P.generate_batch(seed=7, count=ke, out=hp)  # warm-up: touches every page of the host buffer
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P.generate_batch(seed=seed0 + 500, count=ke, out=hp)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    e2e = aggregate_rate(world, n, ke, max_over_ranks(dt, world, dev))

    if rank == 0:
        peak, peak_kind = load_peaks()
        work = realization_work(WORKLOAD["cells"], CONFIG["torus"])
        dom = max(prof, key=lambda r: r["total_ms"]) if prof else None
        roof = None
        if dom:
            avg_ms = dom["total_ms"] / dom["launches"]
            bytes_per = work["pass_bytes"].get(dom["name"], dom["bytes"] / dom["launches"])
            ach = bytes_per / (avg_ms / 1e3) / 1e9
            tr = ncu_traffic().get(dom["name"])
            sched_gbs = work["schedule_bytes"] / (ms / args.steps / 1e3) / 1e9
            roof = {"kernel": dom["name"], "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                    "note": "achieved = the pass's compulsory bytes (each input read once, each output "
                            "written once) / its mean CUDA-event duration on the plan's stream, over the "
                            "same number of realizations generated one at a time after the timed "
                            "(pipelined) region; traffic = ncu DRAM bytes of one launch "
                            "(profiles/ncu_traffic.txt); the pass is instruction-issue-bound, not "
                            "DRAM-bound (see compute.dominant_kernel)",
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 4),
                    "traffic": tr, "algorithmic_bytes_per_launch": bytes_per, "avg_launch_ms": avg_ms,
                    "schedule": {"bytes_per_realization": work["schedule_bytes"],
                                 "gbs": round(sched_gbs, 1), "frac": round(sched_gbs / peak, 4),
                                 "note": "all three passes' compulsory bytes per realization / ms_per_step"},
                    "kernels": [dict({k: (round(v, 4) if isinstance(v, float) else v) for k, v in r.items()},
                                     compulsory_bytes_per_launch=work["pass_bytes"].get(r["name"]))
                                for r in prof]}
        f32peak = max(fpeaks["fp32_ffma_tflops"], fpeaks["fp32_ffma2_tflops"])
        real_s = ms / args.steps / 1e3
        compute = {
            "fp32_peak_tflops": round(f32peak, 1), "fp32_ffma_tflops": round(fpeaks["fp32_ffma_tflops"], 1),
            "fp64_peak_tflops": round(fpeaks["fp64_dfma_tflops"], 1),
            "peak_source": "in-register FMA microbenchmark (pf_measure_peaks) on this GPU before the timed region",
            "realization": {
                "compulsory_bytes": work["compulsory_bytes"],
                "hbm_gbs": round(work["compulsory_bytes"] / real_s / 1e9, 1),
                "hbm_frac": round(work["compulsory_bytes"] / real_s / 1e9 / peak, 4),
                "flops": work["flops"], "tflops": round(work["flops"] / real_s / 1e12, 2),
                "fp32_frac": round(work["flops"] / real_s / 1e12 / f32peak, 4),
                "note": "per realization of the timed (pipelined) region: sqrt(lambda) FP32 on the DCT "
                        "cells + FP32 field; 2.5 N log2 N flops of the full real 3D transform"}}
        if dom and dom["name"] in work["pass_flops"]:
            pf = work["pass_flops"][dom["name"]]
            tfl = pf / (avg_ms / 1e3) / 1e12
            compute["dominant_kernel"] = {"kernel": dom["name"], "flops": pf, "tflops": round(tfl, 2),
                                          "fp32_frac": round(tfl / f32peak, 4)}
        cpu = cpu_lib = err = None
        if not args.no_cpu_baseline and world == 1:
            threads = os.cpu_count() or 1
            dt_cpu, cells, noise, ofield, lam = cpu_oracle_realization(threads)
            cpu = {"value": cells / dt_cpu, "unit": "cells/s", "cores": threads, "kind": "port",
                   "sample": "1 FP64 realization of the same workload by the CPU restatement (oracle/), "
                             f"{dt_cpu:.1f} s; spectrum and noise drawn outside the timed region"}
            dt_lib, sfield = cpu_scipy_realization(threads, lam, noise)
            cpu_lib = {"value": cells / dt_lib, "unit": "cells/s", "cores": threads, "kind": "library",
                       "sample": "the same FP64 realization with scipy.fft.irfftn (pocketfft, workers="
                                 f"{threads}) for the transform, {dt_lib:.1f} s; eigenvalue scaling and "
                                 "extraction in numpy",
                       "rel_l2_vs_oracle": float(np.linalg.norm(sfield - ofield) / np.linalg.norm(ofield))}
            # the FP32 GPU realization from the oracle's noise buffer (reference draw order),
            # outside the timed region
            hn = torch.from_numpy(noise).to(dev)
            P.generate(noise=hn, out=out)
            torch.cuda.synchronize()
            gf = out.double().cpu().numpy()
            # the first realization of the timed batch itself (seeded on-device noise): its
            # noise exported in the reference draw order and fed to the oracle
            tnoise = P.export_noise(seed0 + 100)
            tfield = cpu_oracle_field(tnoise, lam)
            tf = outs[:n].double().cpu().numpy()
            err = {"rel_l2_error_vs_oracle": float(np.linalg.norm(gf - ofield) / np.linalg.norm(ofield)),
                   "max_abs_error_vs_oracle": float(np.abs(gf - ofield).max()),
                   "timed_realization_rel_l2_error_vs_oracle":
                       float(np.linalg.norm(tf - tfield) / np.linalg.norm(tfield)),
                   "note": "one FP32 realization of the timed workload fed the oracle's N(0,1) buffer "
                           "(seed 20261203, reference draw order), against the FP64 oracle on the same "
                           "buffer; and the first realization of the timed batch (seeded on-device noise, "
                           "exported with pf_export_noise) against the oracle fed that noise; tolerance "
                           "of the parity tests 1e-5"}
            del hn
        clocks = clk.summary()
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(CONFIG, parallelism=f"replicas{world}",
                               **({"planning": "default pass choices (--no-tune); K realizations per "
                                               "pf_generate_batch call"} if args.no_tune else {})),
                "e2e": {"value": e2e, "unit": "cells/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": n * 4,
                        "note": f"pf_generate_batch(seed, count={ke}, pinned host out): seed passed by value, "
                                "every realization copied to the host inside the region while the next one is "
                                "computed (wall clock)"},
                "rel_l2_error_vs_oracle": err["rel_l2_error_vs_oracle"] if err else None, "error": err,
                "one_at_a_time": {"value": aggregate_rate(world, n, args.steps, ms_one / 1e3), "unit": "cells/s",
                                  "ms_per_step": ms_one / args.steps,
                                  "note": "pf_generate per realization (device output), no overlap between "
                                          "realizations"},
                "planning": pfb200.wisdom_export().strip().splitlines(),
                "gpu_launches": launches, "roofline": roof, "compute": compute, "cpu_baseline": cpu,
                "cpu_baseline_library_fft": cpu_lib,
                "clocks": {"sm_mhz": clocks["sm_mhz"], "sm_max_mhz": clocks["sm_max_mhz"],
                           "reasons": clocks["reasons"]}}
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        torch.distributed.destroy_process_group()


# ---------------------------------------------------------------------------
# further workloads (one JSON line each; the default run above is the headline)
# ---------------------------------------------------------------------------
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def run_plain2d(args):
    """Plain method, 2D: 512^2 exponential (sigma^2=1, l=0.1, isotropic), factor 2 (1024^2
    torus), FP64, one realization from N(0,1) noise drawn on the host from a seed and fed in
    the reference's draw order (host buffer in, host field out)."""
    import torch
    import pfb200
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    d = pfb200.make_desc(dim=2, cells=(512, 512), covariance="exponential", corr_length=0.1,
                         precision=pfb200.PREC_F64)
    P = pfb200.Plan(d)
    P.spectrum_build()
    g = O.resolve(d)
    noise = torch.tensor(O.noise(20261203, g.noise)).pin_memory().numpy()
    out = torch.empty(g.domain, dtype=torch.float64).pin_memory().numpy()
    for _ in range(args.warmup):
        P.generate(noise=noise, out=out)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        P.generate(noise=noise, out=out)
    dt = (time.perf_counter() - t0) / args.steps
    lam, _, _ = O.spectrum(d)
    ref, _ = O.generate(d, lam, O.noise(20261203, g.noise))
    err = float(np.linalg.norm(out - ref) / np.linalg.norm(ref))
    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    O.generate(d, lam, O.noise(20261203, g.noise))
    cpu = time.perf_counter() - t0
    print(json.dumps({"metric": "field cells/s (2D exponential 512^2, 1024^2 torus, FP64, host noise in, host field out)",
                      "value": g.domain / dt, "unit": "cells/s", "ms_per_step": dt * 1e3, "dtype": "f64",
                      "rel_l2_error_vs_oracle": err, "h2d_bytes_per_step": g.noise * 8,
                      "d2h_bytes_per_step": g.domain * 8,
                      "cpu_baseline": {"value": g.domain / cpu, "unit": "cells/s", "cores": os.cpu_count(),
                                       "kind": "port"}}), flush=True)


def c3_descs(count, precision, seed=20261203):
    """Batched uneven ensemble: sides log-uniform on [128, 2048] per axis, covariance uniform over
    {exponential, gaussian, spherical, cubic}, l ~ U[0.02, 0.3], sigma^2 ~ U[0.5, 2], geometric
    anisotropy l * R(theta) with theta ~ U[0, pi), embedding.approximate = true."""
    import math
    import pfb200
    rng = np.random.default_rng(seed)
    covs = ["exponential", "gaussian", "spherical", "cubic"]
    out = []
    for _ in range(count):
        nx, ny = (int(round(math.exp(rng.uniform(math.log(128), math.log(2048))))) for _ in range(2))
        cov = covs[int(rng.integers(4))]
        ell, var, th = rng.uniform(0.02, 0.3), rng.uniform(0.5, 2.0), rng.uniform(0, math.pi)
        c, s = math.cos(th), math.sin(th)
        out.append(pfb200.make_desc(dim=2, cells=(nx, ny), covariance=cov, variance=var,
                                    corr_length=(ell * c, -ell * s, ell * s, ell * c), anisotropy="geometric",
                                    approximate=True, precision=precision))
    return out


def ensemble_oracle_sample(E, descs, out, seed, epoch, count=6):
    """CPU baseline leg of the ensemble workload: the FP64 oracle on a sample of fields, fed
    each field's exported noise (seed + i, the ensemble call `epoch`), timed and used as the
    checker of the GPU fields of that call"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import pfb200
    O.set_threads(os.cpu_count() or 1)
    idx = sorted(set(int(i) for i in np.linspace(0, len(descs) - 1, count)))
    errs, cells, secs = [], 0, 0.0
    for i in idx:
        d = descs[i]
        P = pfb200.Plan(d)
        noise = P.export_noise(seed + i, epoch)
        P.close()
        lam, _, _ = O.spectrum(d)
        t0 = time.perf_counter()
        ref, _ = O.generate(d, lam, noise)
        secs += time.perf_counter() - t0
        cells += ref.size
        f = out[int(E.offsets[i]):int(E.offsets[i + 1])].double().cpu().numpy()
        errs.append(float(np.linalg.norm(f - ref) / np.linalg.norm(ref)))
    return ({"fields": idx, "rel_l2": errs, "max": max(errs)},
            {"value": cells / secs, "unit": "cells/s", "cores": os.cpu_count(), "kind": "port",
             "sample": f"{len(idx)} fields of the ensemble, one FP64 realization each by the oracle"})


def run_ensemble(args):
    """Uneven 2D fields: mixed (FP32 realizations, FP64 spectra) graph replay vs FP64 replay
    vs the plain FP64 path (one plan and one pf_generate per field, every field)."""
    import torch
    import pfb200
    count = args.fields
    res = {}
    for name, prec in (("fp32", pfb200.PREC_F32), ("fp64", pfb200.PREC_F64)):
        descs = c3_descs(count, prec)
        E = pfb200.Ensemble(descs, seed=1)
        t0 = time.perf_counter()
        st = E.spectra()
        torch.cuda.synchronize()
        tspec = time.perf_counter() - t0
        t0 = time.perf_counter()
        timed = E.autotune(repetitions=1) if not args.no_tune else 0
        ttune = time.perf_counter() - t0
        out = torch.empty(E.total, dtype=torch.float32 if prec else torch.float64, device="cuda")
        E.generate(out)
        s = torch.cuda.current_stream()
        for _ in range(max(1, args.warmup)):
            E.launch(s.cuda_stream)
        e0, e1 = _events()
        e0.record(s)
        for _ in range(args.steps):
            E.launch(s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        errs, cpu = None, None
        if prec == pfb200.PREC_F32 and not args.no_cpu_baseline:
            errs, cpu = ensemble_oracle_sample(E, descs, out, seed=1, epoch=1)
        res[name] = {"cells": E.total, "ms_per_ensemble": ms, "cells_per_s": E.total / (ms / 1e3),
                     "error_vs_oracle_sample": errs, "cpu_baseline_sample": cpu,
                     "spectra_s": tspec, "autotune_s": ttune, "fields_timed_by_autotune": timed,
                     "fields_with_negative_eigenvalues": sum(1 for x in st if x["negative"]),
                     "launches_per_replay": E.launches_per_replay()}
        E.close()
        del out
        torch.cuda.empty_cache()
    sub = c3_descs(count, pfb200.PREC_F64)
    cells, ms_tot = 0, 0.0
    s = torch.cuda.current_stream()
    for dsc in sub:
        P = pfb200.Plan(dsc)
        P.set_stream(s.cuda_stream)
        P.spectrum_build()
        o = torch.empty(P.info.domain_size, dtype=torch.float64, device="cuda")
        P.generate(seed=3, out=o)
        e0, e1 = _events()
        e0.record(s)
        P.generate(seed=4, out=o)
        e1.record(s)
        torch.cuda.synchronize()
        ms_tot += e0.elapsed_time(e1)
        cells += P.info.domain_size
        P.close()
    res["fp64_plain_per_field"] = {"fields": len(sub), "cells": cells, "cells_per_s": cells / (ms_tot / 1e3)}
    res["mixed_batched_vs_plain_fp64"] = res["fp32"]["cells_per_s"] / res["fp64_plain_per_field"]["cells_per_s"]
    print(json.dumps({"metric": f"ensemble field cells/s ({count} uneven 2D fields)", "unit": "cells/s",
                      "value": res["fp32"]["cells_per_s"], "dtype": "f32", "detail": res}), flush=True)


def run_cinv(args):
    """C^-1 on n^3 exponential with a seeded random rotation diag(0.15, 0.08, 0.04): plain
    PCG vs learned-corrected PCG to the 1e-8 FP64 true residual (FP32 inner matvecs)."""
    import torch
    import pfb200
    n = args.cells
    rng = np.random.default_rng(20261203)
    Q, R = np.linalg.qr(rng.standard_normal((3, 3)))
    Q = Q * np.sign(np.diag(R))
    A = Q @ np.diag([0.15, 0.08, 0.04])
    d = pfb200.make_desc(dim=3, cells=(n, n, n), covariance="exponential", corr_length=tuple(A.ravel()),
                         anisotropy="geometric", approximate=True)
    P = pfb200.Plan(d)
    st = P.spectrum_build()
    N = P.info.domain_size
    K_train, K_test = args.train_pairs, args.rhs
    Bt = torch.tensor(rng.standard_normal((K_train, N)), device="cuda")
    Xt = torch.empty_like(Bt)
    t0 = time.perf_counter()
    for i in range(K_train):
        P.multiply_inverse(Bt[i], x=Xt[i], mode=pfb200.CG_RESIDUAL, tolerance=1e-8, inner_fp32=True,
                           max_iterations=20000)
    torch.cuda.synchronize()
    tpairs = time.perf_counter() - t0
    Lp = pfb200.Learned(P, hidden=8, seed=11, residual_loss=args.residual_loss)
    loss0, _ = Lp.loss_grad(Bt, Xt, fp32=True)
    t0 = time.perf_counter()
    loss1 = Lp.train(Bt, Xt, epochs=args.epochs, lr=args.lr, fp32=True)
    ttrain = time.perf_counter() - t0
    Bs = torch.tensor(rng.standard_normal((K_test, N)), device="cuda")
    X = torch.empty_like(Bs)
    out = {}
    for name, attach, lanes in (("plain", False, args.lanes), ("plain_one_lane", False, 1),
                                ("learned", True, 1)):
        Lp.attach(attach)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, reps = P.multiply_inverse_batch(Bs, X, lanes=lanes, mode=pfb200.CG_RESIDUAL, tolerance=1e-8,
                                           inner_fp32=True, max_iterations=20000)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        it = sum(r["iterations"] for r in reps)
        out[name] = {"solves_per_s": K_test / dt, "s_per_solve": dt / K_test, "iterations_per_solve": it / K_test,
                     "max_relative_residual": max(r["relative_residual"] for r in reps), "lanes": lanes,
                     "s_per_iteration": dt / max(it, 1) * min(lanes, K_test)}
    Lp.attach(False)
    print(json.dumps({"metric": f"C^-1 solves/s ({n}^3 exponential, geometric anisotropy, 1e-8 FP64 residual)",
                      "unit": "solves/s", "value": out["plain"]["solves_per_s"], "dtype": "f32 inner / f64 residual",
                      "eigen": st, "plain": out["plain"], "plain_one_lane": out["plain_one_lane"],
                      "learned": out["learned"],
                      "training": {"pairs": K_train, "pair_generation_s": tpairs, "epochs": args.epochs,
                                   "loss": "residual norm" if args.residual_loss else "solution norm",
                                   "lr": args.lr, "train_s": ttrain, "loss_before": loss0,
                                   "loss_after": loss1}}), flush=True)
    Lp.close()


def run_lognormal(args):
    """Log-normal exp(Z) realizations, 192^3 Matern nu=1.5 (l=0.1), FP32, transform applied in
    the last pass."""
    import torch
    import pfb200
    d = pfb200.make_desc(dim=3, cells=(192, 192, 192), covariance="matern32", corr_length=0.1,
                         approximate=True, precision=pfb200.PREC_F32, transform="logNormal")
    P = pfb200.Plan(d)
    s = torch.cuda.current_stream()
    P.set_stream(s.cuda_stream)
    P.spectrum_build()
    if not args.no_tune:
        P.autotune()
    n = P.info.domain_size
    # the K timed realizations in one pf_generate_batch call (two streams), as the headline;
    # one at a time for comparison
    K = max(args.steps, 2)
    outs = torch.empty(K * n, dtype=torch.float32, device="cuda")
    out = outs[:n]
    P.generate_batch(seed=0, count=min(K, max(args.warmup, 2)), out=outs[:min(K, max(args.warmup, 2)) * n],
                     apply_transform=True)
    e0, e1 = _events()
    e0.record(s)
    P.generate_batch(seed=100, count=K, out=outs, apply_transform=True)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    e0.record(s)
    for i in range(K):
        P.generate(seed=100 + i, out=out, apply_transform=True)
    e1.record(s)
    torch.cuda.synchronize()
    ms1 = e0.elapsed_time(e1) / K
    print(json.dumps({"metric": "log-normal field cells/s (192^3, 384^3 torus, FP32)", "unit": "cells/s",
                      "value": n / (ms / 1e3), "ms_per_step": ms, "dtype": "f32",
                      "one_at_a_time": {"value": n / (ms1 / 1e3), "ms_per_step": ms1},
                      "planning": pfb200.wisdom_export().strip().splitlines(),
                      "min": float(out.min()), "mean": float(out.mean())}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="matern3d",
                    choices=["matern3d", "plain2d", "ensemble", "cinv", "lognormal"])
    ap.add_argument("--fields", type=int, default=2048)
    ap.add_argument("--cells", type=int, default=128)
    ap.add_argument("--rhs", type=int, default=4)
    ap.add_argument("--train-pairs", type=int, default=16)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--residual-loss", action="store_true")
    ap.add_argument("--lr", type=float, default=0.005)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--lanes", type=int, default=4)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "matern3d":
        run_b200(args)
    else:
        {"plain2d": run_plain2d, "ensemble": run_ensemble, "cinv": run_cinv, "lognormal": run_lognormal}[
            args.workload](args)


if __name__ == "__main__":
    main()
