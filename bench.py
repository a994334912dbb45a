#!/usr/bin/env python
"""Benchmark of the two-electron hot path on B200.

One step = the Coulomb/exchange build from Cholesky vectors for the
1500-basis-function cluster (120 atoms, rank-200 density, ThrCom 1e-6) plus
the two-electron nuclear gradient of the 460-basis-function cluster (20
atoms 4s3p2d, rank-40 density, Schwarz 1e-12).  The J/K leg runs in the
mixed-precision path; the same step in the plain FP64 GPU path is timed
beside it, with the energy difference between the two.  Inputs are seeded
synthetic molecules (no data files).  Set-up (integrals, Cholesky
decomposition) is outside the timed region.

Second metric (key "eri"): FP64 ERI throughput in quartets/s of the batched
Drv2El-style entry point over a seeded 2 000 000-quartet sample of the
Schwarz-screened (1e-12) unique shell quartets of the 40-atom / 600-function
cluster with uneven classes (l <= 3, 1-12 primitives per shell).

Prints one JSON line (rank 0).  --impl reference times the CPU restatement
of the reference path (oracle port) on a bounded sample instead.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

JK_CFG = "c3"
GRAD_CFG = "c4"
ERI_CFG = "c2"
ERI_SAMPLE = 2_000_000
C3_NVEC = 12865  # Cholesky vectors of the 1500-function cluster at ThrCom 1e-6
JK_SLICES = (6, 7)  # 8-bit slices of MG_PREC_MIXED: half-transform, exchange product (include/molgpu.h)
THRCOM = 1e-6
CUTINT = 1e-12


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for ln in self.p.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- FP64 peak
FP64_PEAK_SRC = r"""
extern "C" __global__ void dfma_peak(double* out, int iters) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double b = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}
"""


def measure_fp64_peak(torch):
    """DFMA throughput (TFLOP/s, FMA = 2 flops) of a register-only kernel on all SMs."""
    from torch.utils.cpp_extension import load_inline  # noqa: F401  (not used: compile via nvcc below)
    import ctypes
    import tempfile
    d = tempfile.mkdtemp()
    src = os.path.join(d, "k.cu")
    so = os.path.join(d, "k.so")
    with open(src, "w") as f:
        f.write(FP64_PEAK_SRC + r"""
#include <cuda_runtime.h>
extern "C" float run_peak(int blocks, int threads, int iters) {
  double* out; cudaMalloc(&out, sizeof(double) * blocks * threads);
  dfma_peak<<<blocks, threads>>>(out, 16);
  cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
  cudaEventRecord(e0); dfma_peak<<<blocks, threads>>>(out, iters); cudaEventRecord(e1);
  cudaEventSynchronize(e1); float ms; cudaEventElapsedTime(&ms, e0, e1); cudaFree(out); return ms;
}
""")
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC", "-shared",
                        "-o", so, src], capture_output=True, text=True)
    if r.returncode != 0:
        return None
    lib = ctypes.CDLL(so)
    lib.run_peak.restype = ctypes.c_float
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, threads, iters = sms * 8, 256, 4000
    ms = lib.run_peak(blocks, threads, iters)
    flops = 2.0 * 8 * 16 * iters * blocks * threads
    return flops / (ms * 1e-3) / 1e12


# --------------------------------------------------------------- workload
def max_over_ranks(x, dist, device):
    """Largest value of x over all ranks (device time of the slowest rank);
    x itself when not distributed."""
    if not dist:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def eri_aggregate(eri, world, max_ms):
    """Whole-job ERI throughput of `world` replicas that each ran the same
    sample, over the slowest replica's time."""
    eri["ms"] = float(max_ms)
    eri["value"] = world * eri["quartets"] / (eri["ms"] / 1e3)
    return eri


def eri_leg(torch, device, reps=2):
    """FP64 ERI throughput over a seeded sample of the screened unique quartets
    (one warm-up call, then `reps` timed calls through MolGpu.eri_quartets;
    host quartet lists, device output)."""
    from openmolcas_b200 import basis as B
    from openmolcas_b200.molgpu import MolGpu, unique_quartets, lib as mglib
    m2 = B.config_molecule(ERI_CFG)
    g2 = MolGpu(m2, device)
    tm = g2.schwarz()
    q = unique_quartets(len(m2.shells), tm, CUTINT)
    rng = np.random.default_rng(0)
    sel = q[np.sort(rng.choice(len(q), min(ERI_SAMPLE, len(q)), replace=False))]
    off = g2.quartet_offsets(sel)
    out = torch.empty(int(off[-1]), dtype=torch.float64, device=f"cuda:{device}")
    g2.eri_quartets(sel, out)
    torch.cuda.synchronize()
    ms = []
    n0 = mglib().mg_kernel_launches()
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g2.eri_quartets(sel, out)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = (mglib().mg_kernel_launches() - n0) // reps
    ms_mean = float(np.mean(ms))
    prim_q, flops = g2.eri_work(sel)
    res = {"value": len(sel) / (ms_mean / 1e3), "unit": "quartets/s", "ms": ms_mean, "quartets": int(len(sel)),
           "screened_unique_quartets": int(len(q)), "integrals_gb": float(off[-1]) * 8 / 1e9,
           "workload": f"{ERI_CFG}: 40 atoms, {m2.nbf} bf, Schwarz {CUTINT}, seeded sample of {len(sel)} of "
                       f"{len(q)} unique quartets", "gpu_launches": int(launches), "dtype": "f64",
           "primitive_quartets_per_s": prim_q / (ms_mean / 1e3), "algorithmic_flops": flops,
           "achieved_tflops": flops / (ms_mean / 1e3) / 1e12,
           "sample_quartets": sel}
    del out
    torch.cuda.empty_cache()
    return res


def eri_cpu_baseline(sel, budget_s=10.0, threads=None):
    """Oracle ERIs over random quartets of the same seeded sample, one quartet
    per call on `threads` host threads (all cores by default), until the time
    budget is used: quartets/s."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    from openmolcas_b200 import basis as B
    threads = threads or os.cpu_count() or 1
    o = O.Oracle(B.config_molecule(ERI_CFG))
    order = np.random.default_rng(1).permutation(len(sel))
    counts = [0] * threads
    t0 = time.time()
    stop = t0 + budget_s

    def work(w):
        for k in range(w, len(order), threads):
            if time.time() > stop:
                break
            o.eri_quartet(*[int(v) for v in sel[order[k]]])
            counts[w] += 1

    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(work, range(threads)))
    dt = time.time() - t0
    n = sum(counts)
    return {"value": n / dt, "unit": "quartets/s", "cores": threads, "kind": "port",
            "sample": f"{n} random quartets of the same seeded sample in {dt:.1f}s"}


def setup(torch, device):
    from openmolcas_b200 import basis as B
    from openmolcas_b200.molgpu import MolGpu
    m3 = B.config_molecule(JK_CFG)
    g3 = MolGpu(m3, device)
    g3.schwarz()  # basis set-up outside the decomposition's clock
    import torch as _t
    _t.cuda.synchronize()
    t0 = time.time()
    info = g3.cho_drv(thrcom=THRCOM)
    t_cho = time.time() - t0
    # bytes the passes' column updates must read: the previous vectors once per pass
    # (X -= L LQ^T reads nrs x M_prev FP64 values, Cho_VecBuf_Subtr)
    _, pass_of = g3.cho_pivots()
    counts = np.bincount(pass_of, minlength=info["npass"])
    m_prev = np.concatenate([[0], np.cumsum(counts)[:-1]])
    info["subtr_bytes"] = float(8.0 * info["nrs"] * m_prev.sum())
    C3 = torch.from_numpy(B.density_factor(m3.nbf, B.CONFIGS[JK_CFG]["rank"], B.CONFIGS[JK_CFG]["seed"]))
    m4 = B.config_molecule(GRAD_CFG)
    g4 = MolGpu(m4, device)
    C4 = B.density_factor(m4.nbf, B.CONFIGS[GRAD_CFG]["rank"], B.CONFIGS[GRAD_CFG]["seed"])
    D4 = torch.from_numpy(C4 @ C4.T)
    return dict(m3=m3, g3=g3, C3=C3, m4=m4, g4=g4, D4=D4, cho=info, t_cho=t_cho)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="molgpu", choices=["molgpu", "reference"])
    ap.add_argument("--leg", default=None, choices=["eri", "grad", "jk", "c5"],
                    help="run one leg alone (timing / profiling driver), no JSON line")
    ap.add_argument("--cfg", default=None, help="--leg eri/grad: configuration (c2, c4, small, medium)")
    ap.add_argument("--quartets", type=int, default=20000, help="--leg eri: sample size")
    ap.add_argument("--natom", type=int, default=40, help="--leg jk: atoms of the 1500-function cluster mix")
    ap.add_argument("--reps", type=int, default=2, help="--leg: timed repetitions")
    ap.add_argument("--precision", default="mixed,fp64", help="--leg jk: precisions to run (mixed, fp64, s<k>)")
    args = ap.parse_args()
    if args.leg:
        return run_leg(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        return run_reference(args)
    return run_gpu(args, rank, world)


def run_gpu(args, rank, world):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from openmolcas_b200.molgpu import MolGpu, lib as mglib
    if dist:
        dist.barrier()
    eri = eri_leg(torch, local)
    if dist:  # replicas: every rank runs the same sample; whole-job throughput over the slowest rank
        eri_aggregate(eri, world, max_over_ranks(eri["ms"], dist, f"cuda:{local}"))
    S = setup(torch, local)
    g3, g4, C3, D4 = S["g3"], S["g4"], S["C3"], S["D4"]
    dev = f"cuda:{local}"
    C3d = C3.to(dev)
    D4d = D4.to(dev)
    st = torch.cuda.current_stream()
    prec_mixed = MolGpu.PREC_MIXED
    try:
        g3.cho_jk(C3d, precision=prec_mixed)
    except Exception:
        prec_mixed = MolGpu.PREC_FP64  # mixed path unavailable: report FP64 and say so
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step(prec, ev=None):
        if ev is not None:
            ev[0].record(st)
        J, K = g3.cho_jk(C3d, precision=prec)
        if ev is not None:
            ev[1].record(st)
        gr = g4.drvg1(D4d, cutint=CUTINT)
        if ev is not None:
            ev[2].record(st)
        return J, K, gr

    def timed(prec, K, W):
        for _ in range(W):
            step(prec)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
        n0 = mglib().mg_kernel_launches()
        out = None
        for k in range(K):
            flush.zero_()  # L2 flush between steps, outside the events
            out = step(prec, evs[k])
        torch.cuda.synchronize()
        launches = mglib().mg_kernel_launches() - n0
        if dist:
            dist.barrier()
        jk = [e[0].elapsed_time(e[1]) for e in evs]
        gr = [e[1].elapsed_time(e[2]) for e in evs]
        return np.array(jk), np.array(gr), launches, out

    # mixed path (headline)
    clk = ClockSampler(local)
    clk.start()
    jk_m, gr_m, launches, out_m = timed(prec_mixed, args.steps, args.warmup)
    clocks = clk.stop()
    # plain FP64 path, same step
    jk_d, gr_d, _, out_d = timed(MolGpu.PREC_FP64, max(2, min(args.steps, 3)), 1)
    step_m = (jk_m + gr_m) / 1e3
    step_d = (jk_d.mean() + gr_d.mean()) / 1e3
    ms = max_over_ranks(float(step_m.mean() * 1e3), dist, dev)
    # energies of both paths
    J, K, grad = out_m
    Jd, Kd, gradd = out_d
    D3 = C3d @ C3d.t()
    E_m = float(0.5 * (D3 * J).sum() - 0.25 * (D3 * K).sum())
    E_d = float(0.5 * (D3 * Jd).sum() - 0.25 * (D3 * Kd).sum())
    # e2e through the public API with host buffers (pinned), copies inside
    C3h = C3.clone().pin_memory()
    D4h = D4.clone().pin_memory()
    torch.cuda.synchronize()
    e2e_times = []
    for k in range(max(2, args.steps)):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Cd = C3h.to(dev, non_blocking=True)
        Dd = D4h.to(dev, non_blocking=True)
        Jx, Kx = g3.cho_jk(Cd, precision=prec_mixed)
        gx = g4.drvg1(Dd, cutint=CUTINT)
        Jh, Kh, gh = Jx.cpu(), Kx.cpu(), gx.cpu()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e = float(np.mean(e2e_times[1:] if len(e2e_times) > 2 else e2e_times))
    h2d = C3h.numel() * 8 + D4h.numel() * 8
    d2h = 2 * g3.nbf * g3.nbf * 8 + g4.natom * 3 * 8
    # rooflines of the two legs
    peaks, src = _peaks()
    fp64_peak = measure_fp64_peak(torch)
    n, r, M = g3.nbf, C3.shape[1], S["cho"]["M"]
    jk_flops = 4.0 * n * n * r * M  # half-transform + exchange product, exact (FP64-equivalent) flops
    jk_s = float(jk_m.mean()) / 1e3
    gr_s = float(gr_m.mean()) / 1e3
    gflops = grad_flops(g4)
    # issued 8-bit tensor work of the sliced exchange GEMMs: s(s+1)/2 products of the
    # padded shapes (half-transform: ld x npad x ld per vector; exchange product: the
    # lower 128 x 128 tiles of ld x ld over M r); int8 dense peak taken as twice the
    # measured BF16 burst (the B200 rates are 4.5 and 2.25 dense POPS/PFLOPS)
    sx, sk = JK_SLICES
    ld = -(-n // 128) * 128
    nmax = min(256, (512 // sx) // 16 * 16)
    nnt = -(-r // nmax)
    npad = nnt * (-(-(-(-r // nnt)) // 16) * 16)
    ntile = (ld // 128) * (ld // 128 + 1) // 2
    i8_ops = (sx * (sx + 1) // 2) * 2.0 * ld * npad * ld * M + (sk * (sk + 1) // 2) * 2.0 * ntile * 128 * 128 * (M * r)
    i8_peak = 2.0 * peaks["bf16_tflops"]
    legs = {
        "jk": {"bound": "tensor", "achieved": i8_ops / jk_s / 1e12, "peak": i8_peak, "unit": "TOP/s (int8)",
               "frac": i8_ops / jk_s / 1e12 / i8_peak,
               "peak_source": f"{src}: 2 x measured bf16 burst (int8 dense = 2 x bf16 dense on B200)",
               "algorithmic_int8_ops": i8_ops, "slices": {"half_transform": sx, "exchange": sk},
               "fp64_equivalent_flops": jk_flops,
               "fp64_equivalent_tflops": jk_flops / jk_s / 1e12, "seconds": jk_s},
        "grad": {"bound": "fp64", "achieved": gflops / gr_s / 1e12 if gflops else None, "peak": fp64_peak,
                 "unit": "TFLOP/s", "frac": (gflops / gr_s / 1e12 / fp64_peak) if (gflops and fp64_peak) else None,
                 "peak_source": "DFMA microbenchmark measured in this run", "algorithmic_flops": gflops,
                 "seconds": gr_s},
    }
    dom = "jk" if jk_s >= gr_s else "grad"
    roof = dict(legs[dom])
    roof["kernel"] = dom
    roof["traffic"] = None
    cpu = cpu_baseline(S)
    eri["fp64_peak_tflops"] = fp64_peak
    eri["frac_of_fp64_peak"] = (eri["achieved_tflops"] / fp64_peak) if fp64_peak else None
    eri_sel = eri.pop("sample_quartets")
    if rank == 0 and world == 1:
        eri["cpu_baseline"] = eri_cpu_baseline(eri_sel)
    res = {
        "metric": "J/K+grad seconds per step (J/K mixed @1500 bf + 2e gradient @460 bf)",
        "value": ms / 1e3 * 1.0,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("f64 (gradient, Cholesky, vectors); J/K exchange in 8-bit slices of the f64 vectors with exact "
                  "int32 tensor-core accumulation" if prec_mixed else "f64"),
        "data": "synthetic (seeded molecules, random contractions and densities)",
        "config": {"workload": f"J/K: {JK_CFG} 120 atoms {g3.nbf} bf, M={M} Cholesky vectors (ThrCom {THRCOM}), "
                               f"rank {r} density; gradient: {GRAD_CFG} 20 atoms {g4.nbf} bf, rank 40 density, "
                               f"Schwarz {CUTINT}", "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas x{world}", "jk_precision": "mixed" if prec_mixed else "fp64"},
        "legs_s": {"jk_mixed": jk_s, "grad": gr_s, "jk_fp64": float(jk_d.mean()) / 1e3},
        "fp64_path_s": step_d,
        "speedup_vs_fp64_path": step_d / (ms / 1e3),
        "energy": {"E_mixed": E_m, "E_fp64": E_d, "dE": E_m - E_d},
        "cholesky": {"M": M, "npass": S["cho"]["npass"], "seconds": S["t_cho"],
                     "roofline": {"bound": "hbm", "achieved": S["cho"]["subtr_bytes"] / S["t_cho"] / 1e9,
                                  "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                  "frac": S["cho"]["subtr_bytes"] / S["t_cho"] / 1e9 / peaks["hbm_gbs"],
                                  "algorithmic_bytes": S["cho"]["subtr_bytes"],
                                  "note": "bytes = the previous vectors read once per pass by the column update "
                                          "(sum over passes of nrs x M_prev x 8); the passes' ERI columns and "
                                          "host qualification are inside the time"}},
        "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches // max(1, args.steps)),
        "roofline": roof,
        "roofline_legs": legs,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "eri": eri,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def grad_flops(g):
    return float(g.drvg1_flops(CUTINT))


CPU_SAMPLE_FACTOR = 100  # each CPU leg times at least 1/100 of its workload


class CpuRef:
    """The CPU restatement of the reference path on bounded samples of the
    step's workload, extrapolated to one full step:
      J/K       CHO_LK_SCF through numpy's BLAS (oracle.cho_jk_blas: DGEMV for J,
                DGEMM for the half-transform and the exchange product, as the
                reference calls its BLAS) over nv of the M vectors,
                nv = max(8 per thread, M / 100), scaled by M / nv (the cost does
                not depend on the vector values);
      gradient  the oracle's Drvg1 restatement (OpenMP over shell quartets) over
                every 100th Schwarz-screened unique quartet, scaled by 100; each
                step starts at the next offset, so successive steps time
                disjoint samples.
    Both arms of the bench use this same sampler."""

    def __init__(self, M=None, threads=None):
        from oracle import oracle as O
        from openmolcas_b200 import basis as B
        self.O = O
        self.threads = threads or os.cpu_count() or 1
        m3 = B.config_molecule(JK_CFG)
        self.M = int(M or C3_NVEC)
        self.n = m3.nbf
        o3 = O.Oracle(m3)
        o3.rs_compact(THRCOM)  # the AO pairs the vectors are stored over
        self.rs_a, self.rs_b, _ = o3.rs_list()
        nrs = self.rs_a.size
        self.nv = max(8 * self.threads, -(-self.M // CPU_SAMPLE_FACTOR))
        self.L = np.random.default_rng(0).standard_normal((nrs, self.nv)) * 1e-3
        cfg = B.CONFIGS[JK_CFG]
        self.C3 = B.density_factor(m3.nbf, cfg["rank"], cfg["seed"])
        m4 = B.config_molecule(GRAD_CFG)
        self.o4 = O.Oracle(m4)
        self.o4.schwarz()
        C4 = B.density_factor(m4.nbf, B.CONFIGS[GRAD_CFG]["rank"], B.CONFIGS[GRAD_CFG]["seed"])
        self.D4 = C4 @ C4.T
        self.k = 0

    def step(self):
        t0 = time.time()
        self.O.cho_jk_blas(self.rs_a, self.rs_b, self.n, self.L, self.C3)
        t_jk_s = time.time() - t0
        t0 = time.time()
        _, nq = self.O.grad_sampled(self.o4, self.D4, CUTINT, CPU_SAMPLE_FACTOR, self.k)
        t_gr_s = time.time() - t0
        self.k += 1
        f_jk = self.M / self.nv
        return {"value": t_jk_s * f_jk + t_gr_s * CPU_SAMPLE_FACTOR, "unit": "s", "cores": self.threads,
                "kind": "port",
                "sample": f"J/K: CHO_LK_SCF through BLAS over {self.nv} of {self.M} vectors ({t_jk_s:.2f} s measured, "
                          f"x{f_jk:.1f}); gradient: every {CPU_SAMPLE_FACTOR}th of {nq} screened unique quartets "
                          f"({t_gr_s:.2f} s measured, x{CPU_SAMPLE_FACTOR})",
                "legs_s": {"jk": t_jk_s * f_jk, "grad": t_gr_s * CPU_SAMPLE_FACTOR},
                "measured_s": {"jk": t_jk_s, "grad": t_gr_s},
                "extrapolation": {"jk": f_jk, "grad": CPU_SAMPLE_FACTOR}}


def cpu_baseline(S=None, threads=None):
    """One step of the CPU sampler (CpuRef) for the GPU arm's line."""
    return CpuRef(M=S["cho"]["M"] if S else None, threads=threads).step()


def run_leg(args):
    """One leg alone, inside an NVTX range named after it (ncu --nvtx
    --nvtx-include "<leg>/" selects its kernels), timed with CUDA events:
      --leg eri  --cfg c2 --quartets N   seeded sample of the screened unique quartets
      --leg grad --cfg c4|small|medium   two-electron gradient (small/medium: 4/8 atoms of 4s3p2d)
      --leg jk   --natom N               Cholesky (ThrCom 1e-6) + J/K, N atoms of the 1500-bf mix
      --leg c5                           C5: Cholesky + mixed/FP64 J/K of 8 densities, CPU J/K sample"""
    import torch
    from openmolcas_b200 import basis as B
    from openmolcas_b200.molgpu import MolGpu, unique_quartets

    def timed(fn):
        ms = []
        for _ in range(args.reps):
            e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
            torch.cuda.nvtx.range_push(args.leg)
            e0.record()
            out = fn()
            e1.record()
            torch.cuda.nvtx.range_pop()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return out, ms

    if args.leg == "eri":
        cfg = args.cfg or ERI_CFG
        m = B.config_molecule(cfg)
        g = MolGpu(m)
        q = unique_quartets(len(m.shells), g.schwarz(), CUTINT)
        sel = q[np.sort(np.random.default_rng(0).choice(len(q), min(args.quartets, len(q)), replace=False))]
        out = torch.empty(int(g.quartet_offsets(sel)[-1]), dtype=torch.float64, device="cuda")
        _, ms = timed(lambda: g.eri_quartets(sel, out))
        print(f"eri {cfg}: {len(sel)} of {len(q)} quartets, last {ms[-1]:.2f} ms, {len(sel) / ms[-1] * 1e3:.3e} quartets/s")
    elif args.leg == "grad":
        cfg = args.cfg or GRAD_CFG
        if cfg in ("small", "medium"):
            na = 4 if cfg == "small" else 8
            m = B.make_molecule(f"{cfg}4s3p2d", na, [("4s3p2d", na)], 4)
            rank = 10 if cfg == "small" else 20
        else:
            m = B.config_molecule(cfg)
            rank = B.CONFIGS[cfg]["rank"] or 40
        g = MolGpu(m)
        Cn = B.density_factor(m.nbf, rank, 4)
        D = torch.from_numpy(Cn @ Cn.T).cuda()
        grad, ms = timed(lambda: g.drvg1(D, cutint=CUTINT))
        print(f"grad {cfg}: nbf {m.nbf}, last {ms[-1]:.1f} ms, |sum F| = {float(grad.sum(0).abs().max()):.2e}")
    elif args.leg == "c5":
        run_c5(timed)
    else:
        c3 = B.CONFIGS[JK_CFG]
        natom = args.natom
        if natom >= c3["natom"]:
            m = B.config_molecule(JK_CFG)
        else:
            mix = [(t, max(1, round(k * natom / c3["natom"]))) for t, k in c3["mix"]]
            mix[-1] = (mix[-1][0], natom - sum(k for _, k in mix[:-1]))
            m = B.make_molecule(f"jk{natom}", natom, mix, c3["seed"])
        g = MolGpu(m)
        info = g.cho_drv(thrcom=THRCOM)
        Cd = torch.from_numpy(B.density_factor(m.nbf, min(c3["rank"], m.nbf // 2), c3["seed"])).cuda()
        D = Cd @ Cd.t()
        res = {}
        for name in args.precision.split(","):
            prec = {"mixed": MolGpu.PREC_MIXED, "fp64": MolGpu.PREC_FP64}.get(name)
            if prec is None:
                prec = MolGpu.PREC_SLICED(int(name[1:]))
            g.cho_jk(Cd, precision=prec)
            torch.cuda.synchronize()
            (J, K), ms = timed(lambda: g.cho_jk(Cd, precision=prec))
            res[name] = (ms[-1], float(0.5 * (D * J).sum() - 0.25 * (D * K).sum()))
        line = f"jk {natom} atoms: nbf {m.nbf}, M {info['M']}"
        for name, (ms, E) in res.items():
            line += f", {name} {ms:.2f} ms (E {E:.10f})"
        print(line)
    return 0


def run_c5(timed):
    """The full-scale system (250 seeded atoms, 2s1p / 3s2p1d / 4s3p2d1f, 1815
    functions): the ERI Cholesky decomposition at ThrCom 1e-6, then J/K of 8
    random densities of uneven rank (50..300) in one batch through the mixed
    and the FP64 path, each density with its energy difference; the CPU
    restatement of the J/K
    (CHO_LK_SCF through BLAS) timed on a sample of the vectors for every
    density and scaled to all of them.  The gradient of this system is not
    run (about 10^3 s per density at the measured C4 rate).  One JSON line."""
    import torch
    from openmolcas_b200 import basis as B
    from openmolcas_b200.molgpu import MolGpu
    m = B.config_molecule("c5")
    g = MolGpu(m)
    torch.cuda.synchronize()
    t0 = time.time()
    info = g.cho_drv(thrcom=THRCOM)
    torch.cuda.synchronize()
    t_cd = time.time() - t0
    ranks = [int(round(r)) for r in np.linspace(50, 300, 8)]
    Cds = [torch.from_numpy(B.density_factor(m.nbf, rk, 5 + k)).cuda() for k, rk in enumerate(ranks)]
    dens = [{"rank": rk} for rk in ranks]
    times = {}
    for name, prec in (("mixed", MolGpu.PREC_MIXED), ("fp64", MolGpu.PREC_FP64)):
        # the 8 densities in one batch (every block of vectors unpacked once), after an untimed call
        g.cho_jk_batch(Cds, precision=prec)
        torch.cuda.synchronize()
        res, ms = timed(lambda: g.cho_jk_batch(Cds, precision=prec))
        times[name] = ms[-1] / 1e3
        for row, Cd, (J, K) in zip(dens, Cds, res):
            D = Cd @ Cd.t()
            row["E_" + name] = float(0.5 * (D * J).sum() - 0.25 * (D * K).sum())
        del res
    for row in dens:
        row["dE"] = row["E_mixed"] - row["E_fp64"]
    del g
    torch.cuda.empty_cache()
    # CPU restatement on a sample of the vectors (the cost does not depend on their values)
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    o5 = O.Oracle(m)
    o5.rs_compact(THRCOM)  # the AO pairs the vectors are stored over
    rs_a, rs_b, _ = o5.rs_list()
    nv = 8 * threads
    L = np.random.default_rng(0).standard_normal((rs_a.size, nv)) * 1e-3
    cpu = 0.0
    for k, rk in enumerate(ranks):
        Cm = B.density_factor(m.nbf, rk, 5 + k)
        t0 = time.time()
        O.cho_jk_blas(rs_a, rs_b, m.nbf, L, Cm)
        cpu += (time.time() - t0) * info["M"] / nv
    mixed, fp64 = times["mixed"], times["fp64"]
    print(json.dumps({"workload": f"c5: 250 atoms, {m.nbf} bf, ThrCom {THRCOM}, 8 densities of rank {ranks}",
                      "cholesky": {"seconds": t_cd, "M": info["M"], "npass": info["npass"]},
                      "jk_mixed_s": mixed, "jk_fp64_s": fp64, "speedup": fp64 / mixed,
                      "max_abs_dE": max(abs(r["dE"]) for r in dens), "densities": dens,
                      "cpu_baseline": {"jk_s": cpu, "cores": threads, "kind": "port",
                                       "sample": f"CHO_LK_SCF through BLAS over {nv} of {info['M']} vectors per "
                                                 f"density, x{info['M'] / nv:.1f}"}}))


def run_reference(args):
    import multiprocessing
    cores = multiprocessing.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(cores)
    vals = []
    cb = None
    ref = CpuRef(threads=cores)
    measured = {"jk": 0.0, "grad": 0.0}
    for k in range(args.warmup + args.steps):
        cb = ref.step()
        if k >= args.warmup:
            vals.append(cb["value"])
            for leg in measured:
                measured[leg] += cb["measured_s"][leg]
    v = float(np.mean(vals))
    cb["sample"] += f"; over the {args.steps} timed steps {measured['jk']:.1f} s (J/K) and {measured['grad']:.1f} s " \
                    f"(gradient) were measured"
    eri_ref = None
    try:  # ERI throughput of the CPU restatement on the same seeded quartet sample
        from oracle import oracle as O
        from openmolcas_b200 import basis as B
        from openmolcas_b200.molgpu import unique_quartets
        m2 = B.config_molecule(ERI_CFG)
        tm = O.Oracle(m2).schwarz()
        q = unique_quartets(len(m2.shells), tm, CUTINT)
        rng = np.random.default_rng(0)
        sel = q[np.sort(rng.choice(len(q), min(ERI_SAMPLE, len(q)), replace=False))]
        eri_ref = eri_cpu_baseline(sel, threads=cores)
    except Exception as e:  # the main metric stands without it
        eri_ref = {"unavailable": str(e)[:200]}
    res = {
        "metric": "J/K+grad seconds per step (J/K mixed @1500 bf + 2e gradient @460 bf)",
        "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded molecules)", "impl": "reference",
        "config": {"workload": f"J/K {JK_CFG} + gradient {GRAD_CFG} (CPU restatement of the reference path)"},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cb["cores"], "kind": "port", "sample": cb["sample"]},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "eri": eri_ref,
    }
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
