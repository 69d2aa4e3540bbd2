#!/usr/bin/env python
"""Benchmark of the TurboQuant encode-and-scan path on B200.

Workload (the HBM-bound encode + scan case): dim 768, bits_per_coord 8
(padded to D = 1024, 1036-byte codes), 10,000,000 rows drawn N(0,1) and
L2-normalised per row, encoded on the GPU into a device-resident corpus; a
step is distance_1_to_n for 64 independent normalised queries against it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is distance Gcodes/s over the whole job
(codes scored per second, all ranks), device-resident corpus; `e2e` is the
same metric through the public Python API with the corpus, the queries and the
distances in pinned host memory (copies inside the timed region);
`roofline` is the scan kernel's achieved HBM bandwidth against the measured
copy peak; `cpu_baseline` is the reference library (compiled from its own
sources into oracle/_ref, the x86-64-v4 build on an AVX-512 host) timed on
this host's cores on a bounded sample.

The same line carries the metric's other halves, each measured on its own
workload after the scan (skip with --no-extras): `cfg1` (100k x 128 4-bit
encode + distance_1_to_n), `mton` (4096 x 1M 768-d 4-bit, FP32 vs split-BF16),
`sym` (2048 x 2M 1536-d 4-bit symmetric, FP32 vs split-BF16) and `serve`
(20M x 384-d 4-bit corpus, exact top-10, p50/p99 and goodput at a few request
rates), each with its reference CPU slice and the clocks seen.

Under torchrun each rank scans its own 10M-code shard (weak scaling, no data
exchange); timing is on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "turboquant-space_b200", "python"))

METRIC = "distance Gcodes/s vs plain FP32 kernel at ≤1e-5 rel err; serving p99 ms at QPS"
DIM, BITS, QUERIES = 768, 8, 64
# DRAM bytes (read + write) per code of one scan launch, from the ncu capture of
# a 1M-code launch of the 768-d 8-bit corpus: 1.036057 GB read + 7.84 MB
# written.  Traffic grows with the code count, so the bench scales it per code.
SCAN_TRAFFIC_PER_CODE = (1.036057e9 + 7.835e6) / 1e6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def l2n(x):
    n = np.linalg.norm(x, axis=1, keepdims=True)
    n[n == 0] = 1.0
    return (x / n).astype(np.float32)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid):
        self.uuid = device_uuid
        self.proc = None

    def __enter__(self):
        try:
            cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                   "-lms", "200"]
            if self.uuid:
                cmd += ["-i", self.uuid]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def shard_seed(base, rank):
    """Seed of this rank's shard: each rank draws and scans its own codes."""
    return base + 7919 * rank


def max_over_ranks(value, dist, device=None):
    """The slowest rank's figure (timing is the max over ranks)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(codes_per_rank, queries, world, ms):
    """Whole-job distance Gcodes/s: every rank scored `queries` x its codes in `ms`."""
    return world * queries * codes_per_rank / (ms * 1e-3) / 1e9


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


REF_FLAGS = "-O3 -ffast-math -fno-finite-math-only -march={} -fopenmp"
_REF_MOD = None


def host_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            flags = set()
            for ln in f:
                if ln.startswith("flags"):
                    flags = set(ln.split(":", 1)[1].split())
                    break
        return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    except OSError:
        return False


def reference_module():
    """The reference's own pybind11 module, built from its sources (oracle/Makefile):
    the x86-64-v4 build on an AVX-512 host (the fixed stand-in for its default
    -march=native), else the x86-64-v3 wheel build.  Returns (module, flags)."""
    global _REF_MOD
    if _REF_MOD is None:
        import glob
        import importlib.util
        ref_dir = os.path.join(ROOT, "oracle", "_ref")
        cands = []
        if host_has_avx512():
            cands.append((os.path.join(ref_dir, "v4"), "x86-64-v4"))
        cands.append((ref_dir, "x86-64-v3"))
        last = None
        for d, arch in cands:
            so = sorted(glob.glob(os.path.join(d, "_turboquant*.so")))
            if not so:
                continue
            try:
                spec = importlib.util.spec_from_file_location("_turboquant", so[0])
                mod = importlib.util.module_from_spec(spec)
                spec.loader.exec_module(mod)
                _REF_MOD = (mod, REF_FLAGS.format(arch))
                break
            except Exception as e:  # e.g. an ISA the host lacks
                last = e
        if _REF_MOD is None:
            raise ImportError(f"reference build not found under oracle/_ref ({last})")
    return _REF_MOD


def cpu_space(dim, bits, cores):
    """(space, kind, build flags): the reference module, or without it the restatement."""
    try:
        mod, flags = reference_module()
        return mod.TurboQuantSpace(dim, bits_per_coord=bits, num_threads=cores), "reference", flags
    except Exception:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        return O.OracleSpace(dim, bits, num_threads=cores), "port", "restatement (tq_oracle.c)"


def cpu_scan(codes_host, queries, cores, kind_pref="reference"):
    """Time distance_1_to_n of the reference (or, without its build, the
    restatement) over `codes_host` for each query; returns (Gcodes/s, kind)."""
    n = codes_host.shape[0]
    sp, kind, flags = cpu_space(DIM, BITS, cores)
    sp.distance_1_to_n(queries[0], codes_host[: min(n, 10000)])  # warm the threads
    t0 = time.perf_counter()
    for q in queries:
        sp.distance_1_to_n(q, codes_host)
    dt = time.perf_counter() - t0
    return len(queries) * n / dt / 1e9, kind, flags


def code_geometry(dim, bits):
    """(padded dim D, code bytes) of the reference layout (space_turbo_quant.h:233-266)."""
    D = 4
    while D < dim:
        D *= 2
    return D, (D // 2 if bits <= 4 else D) + 12


def scan_kernel_name(dim, bits):
    """The staged 1->N scan kernel (tq_kernels.cu) that a dim / bits pair selects."""
    D, _ = code_geometry(dim, bits)
    if bits >= 5:
        return f"scant_kernel<ByteUnits<{D // 128}>,16,S> (staged 1->N scan, byte units)"
    if D == 128:
        return "scant_kernel<HalfNibbleUnits,16,S> (staged 1->N scan, half-warp per code)"
    return f"scant_kernel<NibbleUnits<{D // 256}>,16,S> (staged 1->N scan, nibble units)"


def scan_config(n, world):
    """The `config` of the 1->N scan workload, shared by both arms."""
    D, cs = code_geometry(DIM, BITS)
    gb = n * cs / 1e9
    return {"workload": f"distance_1_to_n x 64 queries over a device-resident corpus of "
                        f"{n / 1e6:g}M codes: dim {DIM}, bits {BITS} (D {D}, {cs} B/code)",
            "n_codes_per_gpu": n, "queries_per_step": QUERIES, "dim": DIM,
            "bits_per_coord": BITS, "code_bytes": cs,
            "l2": (f"corpus {gb:.2f} GB per GPU > 126 MB L2: no flush needed" if gb > 0.126
                   else f"corpus {gb:.3f} GB per GPU fits in the 126 MB L2"),
            "parallelism": f"{world} independent shards" if world > 1 else "1 GPU"}


def run_reference(args, rank):
    """--impl reference: the reference's CPU path on a bounded sample."""
    if rank != 0:
        return
    cores = cpu_cores()
    n_sample, q_sample = 1_000_000, 16
    rng = np.random.default_rng(2)
    X = np.concatenate([l2n(rng.standard_normal((250_000, DIM)).astype(np.float32))
                        for _ in range(n_sample // 250_000)])
    Q = l2n(np.random.default_rng(3).standard_normal((QUERIES, DIM)).astype(np.float32))[:q_sample]
    sp, kind, flags = cpu_space(DIM, BITS, cores)
    codes = sp.encode_batch(X)
    del X

    def step():
        for q in Q:
            sp.distance_1_to_n(q, codes)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    value = q_sample * n_sample / dt / 1e9
    sample = (f"each step {q_sample} of the 64 queries x {n_sample} of the corpus's codes "
              f"({DIM}-d, {BITS}-bit, normalised N(0,1) seed 2), distance_1_to_n, {cores} "
              f"OpenMP threads; codes/s is independent of the sample size for this per-code loop")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 6), "unit": "Gcodes/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": scan_config(args.n, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": round(value, 6), "unit": "Gcodes/s", "cores": cores,
                         "kind": kind, "build": flags, "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "Gcodes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


def mixture_rows(torch, gen, dev, n, dim, centres, std=0.3, chunk=1 << 18):
    """Rows of a Gaussian mixture (uniform weights over `centres`), L2-normalised."""
    out = torch.empty((n, dim), dtype=torch.float32, device=dev)
    k = centres.shape[0]
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        lab = torch.randint(0, k, (b - a,), generator=gen, device=dev)
        blk = centres.index_select(0, lab)
        blk.add_(torch.randn((b - a, dim), generator=gen, device=dev).mul_(std))
        nrm = blk.norm(dim=1, keepdim=True)
        nrm[nrm == 0] = 1.0
        out[a:b] = blk / nrm
    return out


def normal_rows(torch, gen, dev, n, dim, chunk=1 << 20):
    out = torch.empty((n, dim), dtype=torch.float32, device=dev)
    for a in range(0, n, chunk):
        blk = out[a:a + chunk]
        blk.normal_(generator=gen)
        nrm = blk.norm(dim=1, keepdim=True)
        nrm[nrm == 0] = 1.0
        blk.div_(nrm)
    return out


def bf16_peaks():
    """(burst, sustained) dense BF16 TFLOP/s of MEASURED_PEAKS.json, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops"]), float(p["bf16_tflops_sustained"]), "measured"
    except Exception:
        return 1590.0, 1400.0, "fallback"


def mton_result(args, sym, steps=10, cpu=True):
    """Dense M x N contractions, FP32 CUDA cores vs split-BF16 tcgen05.

    mton: 1,000,000 codes of normalised N(0,1) 768-d rows (4-bit), 4096
          normalised queries -> 4096 x 1,000,000 asymmetric distances.
    sym:  2048 x 2,000,000 codes of a 1024-centre Gaussian mixture at 1536-d
          (padded to 2048), 4-bit -> symmetric distances.
    Both forms are timed with CUDA events on their stream; the error of each is
    taken against the FP64 evaluation of the formula on 10,000 sampled pairs;
    the reference's CPU code is timed on a 128-row slice against 100,000 codes."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import turboquant as tq
    from turboquant._capi import check, lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = lib()
    stream = torch.cuda.Stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    gen = torch.Generator(device=dev)
    full_n = args.n == 10_000_000
    if sym:
        dim, bits, m, n = 1536, 4, 2048, 2_000_000 if full_n else args.n
        gen.manual_seed(6)
        centres = torch.randn((1024, dim), generator=gen, device=dev)
        Arows = mixture_rows(torch, gen, dev, m, dim, centres)
        gen.manual_seed(7)
        Brows = mixture_rows(torch, gen, dev, n, dim, centres)
    else:
        dim, bits, m, n = 768, 4, 4096, 1_000_000 if full_n else args.n
        gen.manual_seed(4)
        Brows = normal_rows(torch, gen, dev, n, dim)
        gen.manual_seed(5)
        Arows = normal_rows(torch, gen, dev, m, dim)
    space = tq.TurboQuantSpace(dim, bits_per_coord=bits, device=0)
    h = space._h
    cs, D = space.code_size_bytes(), space.padded_dim()
    codes = torch.empty((n, cs), dtype=torch.uint8, device=dev)
    check(L.tq_encode_batch_device(h, C.c_void_p(Brows.data_ptr()), n, C.c_void_p(codes.data_ptr()), sptr))
    if sym:
        acodes = torch.empty((m, cs), dtype=torch.uint8, device=dev)
        check(L.tq_encode_batch_device(h, C.c_void_p(Arows.data_ptr()), m, C.c_void_p(acodes.data_ptr()), sptr))
    stream.synchronize()
    Qh = Arows.cpu().numpy() if not sym else None
    del Brows
    out = torch.empty((m, n), dtype=torch.float32, device=dev)

    def call(prec):
        if sym:
            check(L.tq_distance_m_to_n_symmetric_device(h, C.c_void_p(acodes.data_ptr()), m,
                                                        C.c_void_p(codes.data_ptr()), n,
                                                        C.c_void_p(out.data_ptr()), prec, sptr))
        else:
            check(L.tq_distance_m_to_n_device(h, C.c_void_p(Arows.data_ptr()), m,
                                              C.c_void_p(codes.data_ptr()), n,
                                              C.c_void_p(out.data_ptr()), prec, sptr))

    flops = float(m) * n * (2 * D if sym else 4 * D)
    res = {}
    rng = np.random.default_rng(10)
    ii = rng.integers(0, m, 10_000)
    jj = rng.integers(0, n, 10_000)
    ch = codes.index_select(0, torch.from_numpy(jj).to(dev)).cpu().numpy()
    o = O.OracleSpace(dim, bits)
    if sym:
        ah = acodes.index_select(0, torch.from_numpy(ii).to(dev)).cpu().numpy()
        f64 = np.array([o.distance_symmetric_f64(ah[k], ch[k]) for k in range(10_000)])
        ma = np.frombuffer(ah[:, D // 2:D // 2 + 4].tobytes(), np.float32).astype(np.float64)
    else:
        f64 = np.array([o.distance_f64(Qh[i], ch[k]) for k, i in enumerate(ii)])
        ma = np.linalg.norm(Qh[ii].astype(np.float64), axis=1)
    mb = np.frombuffer(ch[:, cs - 12:cs - 8].tobytes(), np.float32).astype(np.float64)
    tscale = np.maximum(np.abs(f64), ma ** 2 + mb ** 2)
    flat = torch.from_numpy(ii * n + jj).to(dev)
    burst, sustained, pkind = bf16_peaks()
    legs = (("fp32", 0, max(1, steps // 5)), ("split_bf16", 1, max(3, steps)),
            ("split_bf16_decoded", 4, max(3, steps)))
    for name, prec, reps in legs:
        try:
            call(prec)
        except tq.TQError as e:
            # the decoded form refuses code tiles that do not fit in shared memory
            res[name] = {"not_supported": str(e)}
            continue
        stream.synchronize()
        got = out.view(-1).index_select(0, flat).cpu().numpy().astype(np.float64)
        err = float(np.max(np.abs(got - f64) / tscale))
        plain = float(np.max(np.abs(got - f64) / np.maximum(np.abs(f64), 1e-30)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            call(prec)
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = flops / (ms * 1e-3) / 1e12
        r = {"ms": round(ms, 3), "TFLOP_s_algorithmic": round(tf, 2),
             "Gdist_s": round(m * n / (ms * 1e-3) / 1e9, 3),
             "max_rel_err_vs_fp64": err, "max_plain_rel_err_vs_fp64": plain, "reps": reps}
        if name != "fp32":
            # issued tensor work: exact-sign asymmetric planes (or decoded tiles)
            # take 3 products over the D centroid columns and 2 over the D sign
            # columns; symmetric 3 over D
            issued = float(m) * n * 2 * (5 * D if not sym else 3 * D)
            r["TFLOP_s_issued"] = round(issued / (ms * 1e-3) / 1e12, 2)
            r["frac_issued_of_bf16_sustained"] = round(issued / (ms * 1e-3) / 1e12 / sustained, 4)
            r["frac_algorithmic_of_bf16_sustained"] = round(tf / sustained, 4)
            r["peak_bf16_sustained_tflops"] = sustained
            r["peak_kind"] = pkind
        res[name] = r
    del out
    cpu_base = None
    if cpu:
        cores = cpu_cores()
        sp, kind, rflags = cpu_space(dim, bits, cores)
        cb = codes[:100_000].cpu().numpy()
        if sym:
            ca = acodes[:128].cpu().numpy()
            sp.distance_m_to_n_symmetric(ca[:8], cb[:1000])
            t0 = time.perf_counter()
            sp.distance_m_to_n_symmetric(ca, cb)
        else:
            qa = np.ascontiguousarray(Qh[:128])
            sp.distance_m_to_n(qa[:8], cb[:1000])
            t0 = time.perf_counter()
            sp.distance_m_to_n(qa, cb)
        dt = time.perf_counter() - t0
        gd = 128 * 100_000 / dt / 1e9
        cpu_base = {"value": round(gd, 6), "unit": "Gdist/s", "cores": cores, "kind": kind,
                    "build": rflags, "full_config_s_extrapolated": round(m * n / (gd * 1e9), 1),
                    "sample": f"128 rows x 100,000 codes of this corpus, "
                              f"distance_m_to_n{'_symmetric' if sym else ''}"}
    return {
        "config": {"dim": dim, "padded_dim": D, "bits_per_coord": bits, "m": m, "n": n,
                   "flops_per_pair": 2 * D if sym else 4 * D,
                   "data": ("1024-centre Gaussian mixture, std 0.3, rows L2-normalised (seeds 6/7)"
                            if sym else "N(0,1) rows L2-normalised (seeds 4/5)"),
                   "error_sample": "10,000 (i, j) pairs, seed 10, vs the FP64 evaluation "
                                   "(max_rel_err: relative to max(|d|, |a|^2 + |b|^2))"},
        "results": res,
        "speedup_split_bf16_vs_fp32": round(res["fp32"]["ms"] / res["split_bf16"]["ms"], 2),
        "speedup_split_bf16_decoded_vs_fp32": (
            round(res["fp32"]["ms"] / res["split_bf16_decoded"]["ms"], 2)
            if "ms" in res["split_bf16_decoded"] else None),
        "target_speedup": 4.0,
        "cpu_baseline": cpu_base,
    }


def run_mton(args, sym):
    r = mton_result(args, sym, steps=args.steps, cpu=not args.no_cpu_baseline)
    print(json.dumps({"metric": METRIC, "workload": "sym" if sym else "mton", **r}), flush=True)


def run_symq(args):
    """QJL-corrected symmetric distances (light, full, full-prepared): 2048 row
    codes x 200,000 column codes of a 1024-centre Gaussian mixture at 1536-d
    (padded 2048), 4-bit, device-resident.  Each variant is timed on the GPU
    (CUDA events) in both precisions (FP32 CUDA cores, split-TF32 tensor
    cores) and checked against the FP64 evaluation of its formula on 2,000
    sampled pairs; the reference's own CPU code (oracle/_ref) is timed on a
    bounded sample (128 x 512 pairs) on the host cores."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import turboquant as tq
    from turboquant._capi import PRECISION, SYM_VARIANT, check, lib

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = lib()
    stream = torch.cuda.Stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    dim, bits, m = 1536, 4, 2048
    n = args.n if args.n != 10_000_000 else 200_000
    gen = torch.Generator(device=dev)
    gen.manual_seed(6)
    centres = torch.randn((1024, dim), generator=gen, device=dev)
    Arows = mixture_rows(torch, gen, dev, m, dim, centres)
    gen.manual_seed(7)
    Brows = mixture_rows(torch, gen, dev, n, dim, centres)
    space = tq.TurboQuantSpace(dim, bits_per_coord=bits, device=0)
    h = space._h
    cs, D = space.code_size_bytes(), space.padded_dim()
    acodes = torch.empty((m, cs), dtype=torch.uint8, device=dev)
    codes = torch.empty((n, cs), dtype=torch.uint8, device=dev)
    check(L.tq_encode_batch_device(h, C.c_void_p(Arows.data_ptr()), m, C.c_void_p(acodes.data_ptr()), sptr))
    check(L.tq_encode_batch_device(h, C.c_void_p(Brows.data_ptr()), n, C.c_void_p(codes.data_ptr()), sptr))
    stream.synchronize()
    del Arows, Brows
    out = torch.empty((m, n), dtype=torch.float32, device=dev)
    rng = np.random.default_rng(10)
    ii, jj = rng.integers(0, m, 2000), rng.integers(0, n, 2000)
    ah = acodes.index_select(0, torch.from_numpy(ii).to(dev)).cpu().numpy()
    ch = codes.index_select(0, torch.from_numpy(jj).to(dev)).cpu().numpy()
    o = O.OracleSpace(dim, bits)
    na = np.frombuffer(ah[:, cs - 12:cs - 8].tobytes(), np.float32).astype(np.float64)
    nb = np.frombuffer(ch[:, cs - 12:cs - 8].tobytes(), np.float32).astype(np.float64)
    flat = torch.from_numpy(ii * n + jj).to(dev)
    ref_mod = None
    try:
        ref_mod = reference_module()[0]
    except Exception:  # the reference build is optional
        ref_mod = None
    a_cpu, b_cpu = acodes[:128].cpu().numpy(), codes[:512].cpu().numpy()
    res = {}
    for variant in ("light", "full", "full_prepared"):
        v = SYM_VARIANT[variant]
        f64 = np.array([o.distance_symmetric_qjl_f64(ah[k], ch[k], variant) for k in range(2000)])
        k_total = D + (3 * D if variant != "light" else D)
        r = {}
        for prec in ("fp32", "split_tf32"):
            def call():
                check(L.tq_distance_m_to_n_symmetric_qjl_device(
                    h, C.c_void_p(acodes.data_ptr()), m, C.c_void_p(codes.data_ptr()), n,
                    C.c_void_p(out.data_ptr()), v, PRECISION[prec], sptr))

            call()
            stream.synchronize()
            got = out.view(-1).index_select(0, flat).cpu().numpy().astype(np.float64)
            err = float(np.max(np.abs(got - f64) / np.maximum(np.abs(f64), na ** 2 + nb ** 2)))
            reps = max(1, args.steps // 2) if prec == "fp32" else max(3, args.steps)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                call()
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1) / reps
            r[prec] = {"ms": round(ms, 3), "Gdist_s": round(m * n / (ms * 1e-3) / 1e9, 3),
                       "TFLOP_s_algorithmic": round(2.0 * k_total * m * n / (ms * 1e-3) / 1e12, 2),
                       "max_rel_err_vs_fp64": err, "reps": reps}
        r["speedup_split_tf32_vs_fp32"] = round(r["fp32"]["ms"] / r["split_tf32"]["ms"], 2)
        if ref_mod is not None:
            rs = ref_mod.TurboQuantSpace(dim, bits, num_threads=cpu_cores())
            fn = getattr(rs, f"distance_m_to_n_symmetric_{variant}")
            fn(a_cpu[:4], b_cpu[:4])
            t0 = time.perf_counter()
            fn(a_cpu, b_cpu)
            dt = time.perf_counter() - t0
            r["cpu_reference"] = {"Gdist_s": round(a_cpu.shape[0] * b_cpu.shape[0] / dt / 1e9, 6),
                                  "cores": cpu_cores(), "sample": "128 x 512 pairs of the same codes"}
        res[variant] = r
    print(json.dumps({
        "metric": METRIC, "workload": "symq",
        "config": {"dim": dim, "padded_dim": D, "bits_per_coord": bits, "m": m, "n": n,
                   "data": "1024-centre Gaussian mixture, std 0.3, rows L2-normalised (seeds 6/7)",
                   "error_sample": "2,000 (i, j) pairs, seed 10, vs the FP64 evaluation"},
        "results": res,
    }), flush=True)


def serve_result(args, rates, window, cpu=True, layout="planes"):
    """Serving over a device-resident corpus: 20,000,000 codes of a 1024-centre
    Gaussian mixture at dim 384 (padded 512), 4-bit; requests of m ~ U{1..256}
    queries from the same mixture ask for exact top-10; Poisson arrivals at each
    swept rate for one window; p50/p99 request latency (submit -> result on the
    host) and goodput (completed requests / window) per rate.  The CPU figure is
    the reference's distance_m_to_n + a stable argsort top-10 on a 128-row x
    100,000-code slice, as query rows per second over the whole corpus."""
    import torch
    import turboquant as tq

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dim, bits = 384, 4
    n = 20_000_000 if args.n == 10_000_000 else args.n
    gen = torch.Generator(device=dev)
    gen.manual_seed(8)
    centres = torch.randn((1024, dim), generator=gen, device=dev)
    space = tq.TurboQuantSpace(dim, bits_per_coord=bits, device=0)
    cs = space.code_size_bytes()
    codes = torch.empty((n, cs), dtype=torch.uint8, device=dev)
    chunk = 1 << 20
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        X = mixture_rows(torch, gen, dev, b - a, dim, centres)
        codes[a:b] = space.encode_batch(X)
    del X
    gen.manual_seed(9)
    pool = mixture_rows(torch, gen, dev, 262_144, dim, centres).cpu().numpy()
    cslice = codes[:100_000].cpu().numpy() if cpu else None
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    index = space.index(codes, layout=layout)
    build_s = time.perf_counter() - t0
    D_pad = space.padded_dim()
    index_bytes = n * (cs + (6 * D_pad + 8 if layout == "planes" else 16))
    del codes
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    max_rows, slots = getattr(args, "max_rows", 1024), getattr(args, "slots", 2)
    server = index.serve(k=10, max_rows=max_rows, slots=slots, kernel_variant=args.kernel_variant,
                         bound_scale=getattr(args, "bound_scale", 0.0))
    setup_s = time.perf_counter() - t0
    tuning = server.tuning(searched=True)
    rng = np.random.default_rng(9)
    results = []
    for rate in rates:
        server.reset_stats()
        reqs, refused = [], 0
        t_start = time.perf_counter()
        t_next = t_start
        off = 0
        while True:
            t_next += rng.exponential(1.0 / rate)
            if t_next - t_start > window:
                break
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            m = int(rng.integers(1, 257))
            if off + m > pool.shape[0]:
                off = 0
            try:
                reqs.append(server.submit(pool[off:off + m]))
            except tq.BusyError:
                refused += 1
            off += m
        offered_s = time.perf_counter() - t_start
        lat = []
        for r in reqs:
            r.wait()
            lat.append(r.latency_ms)
        drain_s = time.perf_counter() - t_start
        st = server.stats(latencies=False)
        lat = np.array(lat) if lat else np.array([np.nan])
        results.append({
            "rate_req_s": rate, "window_s": round(offered_s, 2), "offered": len(reqs) + refused,
            "admitted": len(reqs), "refused": refused,
            "goodput_req_s": round(len(reqs) / drain_s, 2),
            "rows_per_s": round(st["rows"] / drain_s, 1),
            "p50_ms": round(float(np.percentile(lat, 50)), 2),
            "p99_ms": round(float(np.percentile(lat, 99)), 2),
            "batches": st["batches"], "mean_rows_per_batch": round(st["rows"] / max(1, st["batches"]), 1),
            "exact_fallback_rows": st["fallback_rows"], "bound_violations": st["bound_violations"],
            "fallback_scan_rows": st["scan_pass_rows"], "fallback_list_rows": st["list_pass_rows"],
        })
    server.close()
    index.close()
    cpu_base = None
    if cpu:
        cores = cpu_cores()
        sp, kind, rflags = cpu_space(dim, bits, cores)
        q = np.ascontiguousarray(pool[:128])
        sp.distance_m_to_n(q[:8], cslice[:1000])
        t0 = time.perf_counter()
        d = sp.distance_m_to_n(q, cslice)
        np.argsort(d, axis=1, kind="stable")[:, :10]
        dt = time.perf_counter() - t0
        rows_s = 128 / (dt * n / cslice.shape[0])
        cpu_base = {"value": round(rows_s, 4), "unit": "query rows/s over the whole corpus",
                    "cores": cores, "kind": kind, "build": rflags,
                    "sample": "128 query rows x 100,000 codes: distance_m_to_n + stable argsort "
                              "top-10, scaled to the corpus size"}
    return {
        "config": {"dim": dim, "padded_dim": space.padded_dim(), "bits_per_coord": bits,
                   "n_codes": n, "k": 10, "request_rows": "U{1..256}", "arrivals": "Poisson",
                   "window_s": window, "max_batch_rows": max_rows, "slots": slots,
                   "kernel_variant": "autotuned" if args.kernel_variant < 0 else args.kernel_variant,
                   "top_k": "exact (tensor-pass candidates rescored with the reference's arithmetic)",
                   "bound_scale": getattr(args, "bound_scale", 0.0) or 1.0,
                   "index_layout": layout, "index_bytes": index_bytes,
                   "data": "1024-centre Gaussian mixture, std 0.3, rows L2-normalised (seeds 8/9)"},
        "index_build_s": round(build_s, 2), "server_setup_s": round(setup_s, 2), "tuning": tuning,
        "results": results, "cpu_baseline": cpu_base,
    }


def run_serve(args):
    rates = [float(r) for r in args.rates.split(",")]
    r = serve_result(args, rates, args.window, cpu=not args.no_cpu_baseline, layout=args.layout)
    print(json.dumps({"metric": METRIC, "workload": "serve", **r}), flush=True)


def cfg1_result(args):
    """The plain-method case: 100,000 x 128 N(0,1) rows (seed 0), 4-bit, one query
    (seed 1): encode_batch then distance_1_to_n, device-resident (CUDA events)
    and through the host API; codes against the reference's digest, distances
    against the checker; the reference's CPU path on the same full workload."""
    import hashlib
    import torch
    import turboquant as tq
    from turboquant._capi import check, lib
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    L = lib()
    stream = torch.cuda.Stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    X = np.random.default_rng(0).standard_normal((100_000, 128)).astype(np.float32)
    q = np.random.default_rng(1).standard_normal(128).astype(np.float32)
    space = tq.TurboQuantSpace(128, bits_per_coord=4, device=0)
    h = space._h
    cs = space.code_size_bytes()
    Xd, qd = torch.from_numpy(X).to(dev), torch.from_numpy(q).to(dev)
    codes = torch.empty((100_000, cs), dtype=torch.uint8, device=dev)
    out = torch.empty(100_000, dtype=torch.float32, device=dev)

    def enc():
        check(L.tq_encode_batch_device(h, C.c_void_p(Xd.data_ptr()), 100_000, C.c_void_p(codes.data_ptr()), sptr))

    def scan():
        check(L.tq_distance_1_to_n_device(h, C.c_void_p(qd.data_ptr()), C.c_void_p(codes.data_ptr()),
                                          100_000, C.c_void_p(out.data_ptr()), sptr))

    res = {}
    for name, fn in (("encode", enc), ("distance_1_to_n", scan)):
        for _ in range(5):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(100):
            fn()
        e1.record(stream)
        stream.synchronize()
        res[name] = {"us": round(e0.elapsed_time(e1) * 10.0, 2)}
    res["encode"]["Mvec_per_s"] = round(100_000 / res["encode"]["us"], 2)
    res["distance_1_to_n"]["Gcodes_per_s"] = round(100_000 / res["distance_1_to_n"]["us"] / 1e3, 3)
    ch = codes.cpu().numpy()
    digest_ok = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "digests.json")) as f:
            digest_ok = hashlib.sha256(ch.tobytes()).hexdigest() == json.load(f)["cfg1_codes_sha256"]
    except OSError:
        pass
    d = out.cpu().numpy()
    ref = O.OracleSpace(128, 4).distance_1_to_n(q, ch)
    meta = np.frombuffer(ch[:, cs - 12:cs - 8].tobytes(), np.float32).astype(np.float64)
    tscale = float(np.sum(q.astype(np.float64) ** 2)) + meta ** 2
    err = float(np.max(np.abs(d - ref) / np.maximum(np.abs(ref), tscale)))
    # through the host API (numpy in, numpy out: copies included)
    t0 = time.perf_counter()
    for _ in range(10):
        c2 = space.encode_batch(X)
        space.distance_1_to_n(q, c2)
    host_ms = (time.perf_counter() - t0) / 10 * 1e3
    cores = cpu_cores()
    sp, kind, rflags = cpu_space(128, 4, cores)
    sp.encode_batch(X[:1000])
    t0 = time.perf_counter()
    rc = sp.encode_batch(X)
    t1 = time.perf_counter()
    for _ in range(10):
        sp.distance_1_to_n(q, rc)
    t2 = time.perf_counter()
    return {
        "config": {"dim": 128, "bits_per_coord": 4, "n": 100_000, "code_bytes": cs,
                   "data": "N(0,1) rows (seed 0), query seed 1, not normalised"},
        "device": res, "host_api_ms_encode_plus_distance": round(host_ms, 3),
        "codes_match_reference_digest": digest_ok, "distance_max_rel_err_vs_checker": err,
        "cpu_baseline": {"encode_ms": round((t1 - t0) * 1e3, 3),
                         "distance_1_to_n_ms": round((t2 - t1) / 10 * 1e3, 3), "cores": cores,
                         "kind": kind, "build": rflags, "sample": "the full workload"},
    }


def extra(fn, uuid, *a):
    """One of the default run's extra workloads, with the clocks seen while it
    ran; an error is reported in its key instead of ending the run."""
    import torch
    try:
        with ClockSampler(uuid) as clk:
            r = fn(*a)
        r["clocks"] = clk.summary()
        return r
    except Exception as e:  # report, keep the headline line
        return {"error": f"{type(e).__name__}: {e}"}
    finally:
        torch.cuda.synchronize()
        torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--n", type=int, default=10_000_000, help="codes per GPU")
    ap.add_argument("--dim", type=int, default=768, help="scan: input dimension")
    ap.add_argument("--bits", type=int, default=8, help="scan: bits per coordinate")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="scan: skip the config-1, M x N (mton, sym) and serving keys")
    ap.add_argument("--extra-rates", default="20,60,1000",
                    help="scan: request rates (req/s) of the serving key")
    ap.add_argument("--extra-window", type=float, default=5.0,
                    help="scan: seconds per rate of the serving key")
    ap.add_argument("--rates", default="5,20,40,60,100,150,1000,50000",
                    help="serve: request rates (req/s) to sweep")
    ap.add_argument("--window", type=float, default=30.0, help="serve: seconds per rate")
    ap.add_argument("--max-rows", type=int, default=1024,
                    help="serve: query rows per batch (a request holds at most 256)")
    ap.add_argument("--slots", type=int, default=2, help="serve: batches in flight")
    ap.add_argument("--layout", choices=("planes", "codes"), default="planes",
                    help="serve: index layout (operand planes, or codes decoded in shared memory)")
    ap.add_argument("--kernel-variant", type=int, default=-1,
                    help="serve: top-k kernel variant (-1: autotuned per batch bucket; 0 .. 5: "
                         "the tile shapes of turboquant.variant_shapes())")
    ap.add_argument("--bound-scale", type=float, default=0.0,
                    help="serve: multiple of the certificate's error bound (0: the server's default, "
                         "1); larger values leave more rows to the exact fallback")
    ap.add_argument("--workload", choices=("scan", "mton", "sym", "symq", "serve"), default="scan",
                    help="scan (default): the 1->N scan benchmark; mton/sym: the dense M x N "
                         "contractions, FP32 vs split-BF16; symq: the QJL-corrected symmetric "
                         "distances; serve: the serving loop")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global DIM, BITS
    DIM, BITS = args.dim, args.bits
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "symq":
        run_symq(args)
        return
    if args.workload != "scan":
        run_mton(args, args.workload == "sym")
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    import turboquant as tq
    from turboquant._capi import check, lib

    L = lib()
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(dev)
    sptr = C.c_void_p(stream.cuda_stream)
    space = tq.TurboQuantSpace(DIM, bits_per_coord=BITS, device=local)
    h = space._h
    cs = space.code_size_bytes()
    D = space.padded_dim()
    n = args.n
    hbm_peak, peak_kind = peaks()

    # ---- corpus: N(0,1) rows, L2-normalised, on this GPU (untimed) ----------
    gen = torch.Generator(device=dev)
    gen.manual_seed(shard_seed(2, rank))
    X = torch.empty((n, DIM), dtype=torch.float32, device=dev)
    with torch.cuda.stream(stream):
        step_rows = 1 << 20
        for a in range(0, n, step_rows):
            blk = X[a:a + step_rows]
            blk.normal_(generator=gen)
            nrm = blk.norm(dim=1, keepdim=True)
            nrm[nrm == 0] = 1.0
            blk.div_(nrm)
    codes = torch.empty((n, cs), dtype=torch.uint8, device=dev)
    stream.synchronize()

    # ---- encode (bit-exact): timed separately -------------------------------
    def encode():
        check(L.tq_encode_batch_device(h, C.c_void_p(X.data_ptr()), n, C.c_void_p(codes.data_ptr()),
                                       sptr))

    encode()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    ev0.record(stream)
    for _ in range(reps):
        encode()
    ev1.record(stream)
    stream.synchronize()
    enc_ms = ev0.elapsed_time(ev1) / reps
    enc_bytes = n * (DIM * 4 + cs)

    # parity sample of the full-size encode against the CPU checker
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    rows = np.sort(np.random.default_rng(99).choice(n, size=min(n, 512), replace=False))
    ridx = torch.from_numpy(rows).to(dev)
    Xs = X.index_select(0, ridx).cpu().numpy()
    Cs = codes.index_select(0, ridx).cpu().numpy()
    enc_exact = bool(np.array_equal(O.OracleSpace(DIM, BITS).encode_batch(Xs), Cs))
    del X, ridx
    torch.cuda.empty_cache()

    # ---- queries and outputs --------------------------------------------------
    Qh = l2n(np.random.default_rng(shard_seed(3, rank)).standard_normal((QUERIES, DIM)).astype(np.float32))
    Qd = torch.from_numpy(Qh).to(dev)
    out = torch.empty((QUERIES, n), dtype=torch.float32, device=dev)
    qptr = [C.c_void_p(Qd[i].data_ptr()) for i in range(QUERIES)]
    optr = [C.c_void_p(out[i].data_ptr()) for i in range(QUERIES)]
    cptr = C.c_void_p(codes.data_ptr())

    def step():
        for i in range(QUERIES):
            check(L.tq_distance_1_to_n_device(h, qptr[i], cptr, n, optr[i], sptr))

    # distance parity sample: query 0 against 2048 codes, vs the checker
    step()
    stream.synchronize()
    csample = codes[:2048].cpu().numpy()
    dref = O.OracleSpace(DIM, BITS).distance_1_to_n(Qh[0], csample)
    meta = np.frombuffer(csample[:, cs - 12:cs - 8].tobytes(), np.float32).astype(np.float64)
    tscale = float(np.sum(Qh[0].astype(np.float64) ** 2)) + meta ** 2
    dgot = out[0, :2048].cpu().numpy()
    dist_err = float(np.max(np.abs(dgot - dref) / np.maximum(np.abs(dref), tscale)))
    dist_err_plain = float(np.max(np.abs(dgot - dref) / np.maximum(np.abs(dref), 1e-30)))

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- timed region: K steps of 64 distance_1_to_n calls --------------------
    for _ in range(args.warmup):
        step()
    stream.synchronize()
    barrier()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    with ClockSampler(uuid) as clk:
        torch.cuda.synchronize(dev)
        # the library's scan timer: CUDA events around each scan kernel launch
        # of the timed calls, on their stream
        check(L.tq_space_scan_timer(h, 1))
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        stream.synchronize()
        check(L.tq_space_scan_timer(h, 0))
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, dev)
    value = job_throughput(n, QUERIES, world, ms)
    t_ms, t_n = C.c_double(), C.c_uint64()
    check(L.tq_space_scan_timer_read(h, C.byref(t_ms), C.byref(t_n)))
    scan_ms = max_over_ranks(t_ms.value / max(1, t_n.value), dist, dev)

    # ---- the scan kernel alone: per-launch duration (prepared queries) --------
    qrot = torch.empty((QUERIES, D), dtype=torch.float32, device=dev)
    sq = torch.empty_like(qrot)
    nrm = torch.empty((QUERIES, 2), dtype=torch.float32, device=dev)
    check(L.tq_prepare_queries_device(h, C.c_void_p(Qd.data_ptr()), QUERIES, C.c_void_p(qrot.data_ptr()),
                                      C.c_void_p(sq.data_ptr()), C.c_void_p(nrm.data_ptr()), sptr))
    scan_args = [(C.c_void_p(qrot[i].data_ptr()), C.c_void_p(sq[i].data_ptr()),
                  C.c_void_p(nrm[i].data_ptr()), optr[i]) for i in range(QUERIES)]
    for a in scan_args[:4]:
        check(L.tq_distance_1_to_n_prepared_device(h, a[0], a[1], a[2], cptr, n, a[3], sptr))
    ev0.record(stream)
    for a in scan_args:
        check(L.tq_distance_1_to_n_prepared_device(h, a[0], a[1], a[2], cptr, n, a[3], sptr))
    ev1.record(stream)
    stream.synchronize()
    scan_ms_isolated = ev0.elapsed_time(ev1) / QUERIES
    scan_bytes = n * (cs + 4)
    achieved = scan_bytes / (scan_ms * 1e-3) / 1e9

    # ---- e2e: the public API with host buffers (rank-local) -------------------
    e2e = None
    if not args.no_e2e:
        codes_h = torch.empty((n, cs), dtype=torch.uint8, pin_memory=True)
        codes_h.copy_(codes)
        out_h = torch.empty((QUERIES, n), dtype=torch.float32, pin_memory=True)
        Q_h = torch.from_numpy(Qh).pin_memory()
        cn, on, qn = codes_h.numpy(), out_h.numpy(), Q_h.numpy()
        space.distance_m_to_n(qn, cn, out=on)  # warm-up
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            space.distance_m_to_n(qn, cn, out=on)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / args.e2e_steps, dist, dev)
        e2e = {"value": round(job_throughput(n, QUERIES, world, e2e_s * 1e3), 4), "unit": "Gcodes/s",
               "h2d_bytes_per_step": int(n * cs + QUERIES * DIM * 4),
               "d2h_bytes_per_step": int(QUERIES * n * 4),
               "ms_per_step": round(e2e_s * 1e3, 2),
               "call": "TurboQuantSpace.distance_m_to_n(queries, codes, out=...) on pinned host arrays"}
        del codes_h, out_h

    # ---- CPU baseline: the reference on this host's cores, bounded sample ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = cpu_cores()
        n_cpu = min(n, 1_000_000)
        ch = codes[:n_cpu].cpu().numpy()
        val, kind, flags = cpu_scan(ch, Qh[:16], cores)
        cpu = {"value": round(val, 6), "unit": "Gcodes/s", "cores": cores, "kind": kind,
               "build": flags, "sample": f"16 queries x {n_cpu} codes of this corpus, distance_1_to_n"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Gcodes/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (torch Philox N(0,1), rows L2-normalised; seeded per rank)",
            "config": scan_config(n, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                         "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "traffic": (int(round(SCAN_TRAFFIC_PER_CODE * n))
                                     if (DIM, BITS) == (768, 8) else None),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                           "1M-code launch, scaled per code",
                         "kernel": scan_kernel_name(DIM, BITS),
                         "bytes_per_launch": scan_bytes, "ms_per_launch": round(scan_ms, 4),
                         "launches_timed": int(t_n.value),
                         "ms_per_launch_source": "CUDA events around each scan kernel launch of the "
                                                 "timed region (the library's scan timer)",
                         "ms_per_launch_isolated": round(scan_ms_isolated, 4),
                         "peak_kind": peak_kind},
            "encode": {"ms": round(enc_ms, 3), "Mvec_per_s": round(n / enc_ms / 1e3, 2),
                       "GB_per_s": round(enc_bytes / enc_ms / 1e6, 1),
                       "frac_hbm": round(enc_bytes / enc_ms / 1e6 / hbm_peak, 4),
                       "bit_exact_sample_rows": len(rows), "bit_exact": enc_exact},
            "distance_check": {"max_rel_err_vs_checker": dist_err,
                               "max_plain_rel_err_vs_checker": dist_err_plain,
                               "rel_err_denominator": "max(|d_ref|, |q|^2 + |x|^2); plain: |d_ref|",
                               "codes_checked": 2048},
            "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": args.steps * QUERIES * 2,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_extras:
            # the metric's other halves on their own workloads, after the scan's
            # buffers are released
            del out, codes, Qd, qrot, sq, nrm, scan_args, optr, qptr, cptr
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            rates = [float(r) for r in args.extra_rates.split(",")]
            line["cfg1"] = extra(cfg1_result, uuid, args)
            line["mton"] = extra(mton_result, uuid, args, False, 10, not args.no_cpu_baseline)
            line["sym"] = extra(mton_result, uuid, args, True, 10, not args.no_cpu_baseline)
            line["serve"] = extra(serve_result, uuid, args, rates, args.extra_window,
                                  not args.no_cpu_baseline)
            # the same corpus in the codes layout (tiles decoded in shared memory): one rate
            line["serve_codes_layout"] = extra(serve_result, uuid, args, rates[-1:],
                                               args.extra_window, False, "codes")
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
