#!/usr/bin/env python
"""Benchmark: SLQ logdet probe*steps/s on B200 (mixed precision, batched).

Workload (one "step" = one SLQ logdet run over one block of probes on the
resident matrix): the sparse SPD correlation matrix of the headline
workload -- n = 262144 points uniform in [0,1]^2 (numpy PCG64 seed 1),
kernel exp(-r/0.005) zeroed below 0.05 -- with the diagonal shift 0.1 in place
of the specified 1e-3, which leaves the matrix indefinite (smallest Ritz
value -0.0548, logdet undefined); 48.07M nonzeros, FP32 values, int32
indices.  256 Rademacher probes (parity stream, seed 0), lanczos_degree 50,
full reorthogonalisation.  Inputs (matrix 385 MB, Krylov basis 13.4 GB) are
larger than L2 (126 MB), so no flush is needed between steps.

value      probe*Lanczos-steps per second, whole job, device-timed (CUDA
           events), matrix resident in HBM.
e2e        same metric through the public API from host scipy arrays: the
           CSR upload (host -> device) and the result readback are inside the
           timed region.
roofline   dominant kernel class: algorithmic bytes per launch / mean launch
           time (CUDA events inside the timed region), vs the measured HBM
           copy bandwidth; roofline.spmm the same for the SpMM, with the
           tensor-core work it issues on the block format.
cpu_baseline  the reference's own CPU SLQ (oracle/_ref, built from its
           sources) on the host cores, on a bounded sample of the workload.

--impl reference times that reference CPU implementation alone.
Multi-GPU: torchrun, one rank per GPU; each rank runs its own probes
(disjoint probe indices), no collective on the data path (weak scaling).
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("SLQ logdet probe·steps/s on 1 B200, mixed+batched vs plain "
          "FP64, at 1e-3 rel err")
# the function of the c2prime line: the reference's function code and the
# public entry point's name (traceinv: imate/traceinv/_slq_method.pyx:24)
FUNC_CODES = {"logdet": "log", "traceinv": "inv"}


def metric_of(args):
    return METRIC.replace("logdet", args.func)
UNIT = "probe*steps/s"
# FP64 oracle of the workload's logdet: sparse LU (scipy splu, MMD_AT_PLUS_A,
# symmetric mode) of the float64 matrix; tests/golden/make_c2_oracle.py
ORACLE_FILE = os.path.join(ROOT, "tests", "golden", "c2prime_oracle.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine",
                    choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--probes", type=int, default=256)
    ap.add_argument("--degree", type=int, default=50)
    ap.add_argument("--orthogonalize", type=int, default=-1)
    ap.add_argument("--shift", type=float, default=0.1)
    ap.add_argument("--fp64-probes", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="c2prime",
                    choices=["c2prime", "batched", "sweep", "gram-large",
                             "dense"],
                    help="c2prime: the headline line (default); batched: 64 "
                         "correlation matrices in one graph; sweep: 512-point "
                         "t-sweep by the surrogate; gram-large: logdet(X^T X "
                         "+ lambda I) of an 8388608 x 2097152 sparse X; "
                         "dense: logdet of a 16384 x 16384 dense correlation "
                         "matrix by the tensor-core operator")
    ap.add_argument("--batch-count", type=int, default=64)
    ap.add_argument("--spmm", default="block-tc",
                    choices=["auto", "csr", "row-group", "row-group-tma",
                             "row-group-tc", "block-tc"],
                    help="SpMM kernel of the device-resident run: the "
                         "tensor-core block kernel on the block format "
                         "(default), the built-in choice without that format "
                         "(auto) or a forced autotuner candidate; the e2e leg "
                         "always takes the public API's default path")
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--func", default="logdet", choices=sorted(FUNC_CODES),
                    help="function of the c2prime line (same kernels; "
                         "traceinv takes f = 1/x at the Ritz values)")
    ap.add_argument("--fp64-ref-probes", type=int, default=-1,
                    help="probes of the high-sample FP64 SLQ the c2prime "
                         "line states its error against (-1: 1024 for "
                         "traceinv, which has no direct FP64 oracle at full "
                         "size, 0 for logdet, whose oracle is sparse LU)")
    return ap.parse_args()


def build_matrix(args, dtype):
    from imate_b200.sample_matrices import correlation_matrix
    return correlation_matrix(args.n, scale=0.005, threshold=0.05,
                              shift=args.shift, seed=1, dtype=dtype)


def workload_config(args, nnz):
    return {
        "workload": "sparse SPD correlation matrix (exp(-r/0.005), cut 0.05, "
                    "diag shift %g), SLQ %s" % (args.shift, args.func),
        "n": args.n, "nnz": int(nnz), "value_dtype": "float32",
        "index_dtype": "int32", "probes_per_step": args.probes,
        "lanczos_degree": args.degree,
        "orthogonalize": args.orthogonalize, "rng": "parity",
        "l2": "inputs larger than L2 (matrix %.0f MB, basis %.1f GB)" % (
            nnz * 8e-6, (args.degree + 1) * args.n * args.probes * 4e-9),
        "spmm": args.spmm,
    }


def load_oracle(args):
    if args.func != "logdet":
        return None
    try:
        with open(ORACLE_FILE) as f:
            d = json.load(f)
        if d["n"] == args.n and abs(d["shift"] - args.shift) < 1e-15:
            return d["logdet"]
    except (OSError, KeyError, ValueError):
        pass
    return None


# ---------------------------------------------------------------------------
# reference CPU SLQ (oracle/_ref) -- CPU baseline and the reference arm
# ---------------------------------------------------------------------------

def reference_sample(A, args, probes, threads, seed=0):
    """Time the reference CPU estimator on `probes` probes; returns
    (probe*steps/s, seconds, kind)."""
    from oracle import ref
    if ref.available():
        r = ref.trace_estimator(A, FUNC_CODES[args.func],
                                min_num_samples=probes,
                                max_num_samples=probes, error_rtol=0.0,
                                lanczos_degree=args.degree,
                                orthogonalize=args.orthogonalize, seed=seed,
                                num_threads=threads)
        secs = r["alg_wall_time"]
        # the reference does not report per-sample Krylov sizes; breakdown
        # does not occur on this matrix, so every probe runs all steps
        return probes * args.degree / secs, secs, "reference"
    from oracle import oracle
    t = time.perf_counter()
    r = oracle.trace_estimator(A.astype(np.float64), FUNC_CODES[args.func],
                               min_num_samples=probes,
                               max_num_samples=probes, error_rtol=0.0,
                               lanczos_degree=args.degree,
                               orthogonalize=args.orthogonalize, seed=seed)
    secs = time.perf_counter() - t
    return float(np.sum(r["lanczos_sizes"][:probes])) / secs, secs, "port"


def reference_baseline(A, args, threads, min_secs=10.0, max_rounds=8):
    """The reference CPU SLQ timed over rounds of one probe per host thread
    (seeds 0, 1, ...) until at least ``min_secs`` of its own computation
    time: (probe*steps/s, probes, seconds, kind)."""
    probes = min(threads, 64)
    total_ps, total_s, rounds, kind = 0.0, 0.0, 0, "reference"
    while rounds < max_rounds and (rounds == 0 or total_s < min_secs):
        v, secs, kind = reference_sample(A, args, probes, threads, seed=rounds)
        total_ps += v * secs
        total_s += secs
        rounds += 1
    return total_ps / total_s, probes * rounds, total_s, kind


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    A = build_matrix(args, "float32")
    threads = cpu_threads()
    probes = threads  # one probe per host thread per step
    for _ in range(args.warmup):
        reference_sample(A, args, probes, threads)
    vals, secs = [], 0.0
    kind = "reference"
    for s in range(args.steps):
        v, t, kind = reference_sample(A, args, probes, threads, seed=s)
        vals.append(v)
        secs += t
    value = probes * args.degree * args.steps / secs
    line = {
        "impl": "reference", "metric": metric_of(args), "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(args, A.nnz),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": kind,
                         "sample": "%d probes x %d Lanczos steps per step, "
                                   "num_threads=%d" % (probes, args.degree,
                                                       threads)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    gpu_ref = reference_gpu_sample(A, args)
    if gpu_ref is not None:
        line["reference_gpu"] = gpu_ref
    print(json.dumps(line), flush=True)


def reference_gpu_sample(A, args, probes=8, path=None):
    """The reference's own GPU SLQ (cuSPARSE SpMV -- cuBLAS gemv for a dense
    ndarray -- and cuBLAS vector operations, one probe at a time;
    oracle/_ref/libimate_ref_gpu.so compiled from its sources for sm_100a)
    on a sample of the same workload, FP32 and FP64: probe*steps/s over its
    own computation time, and over the whole call (matrix upload included).
    None without a GPU or the library."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        from oracle import ref
        if not ref.gpu_available():
            return None
    except ImportError:
        return None
    out = {}
    for name, dt in (("f32", np.float32), ("f64", np.float64)):
        Ad = A.astype(dt)
        kw = dict(min_num_samples=probes, max_num_samples=probes,
                  error_rtol=0.0, lanczos_degree=args.degree,
                  orthogonalize=args.orthogonalize, seed=0)
        ref.gpu_trace_estimator(Ad, "log", **dict(kw, min_num_samples=1,
                                                  max_num_samples=1))
        t0 = time.perf_counter()
        r = ref.gpu_trace_estimator(Ad, "log", **kw)
        wall = time.perf_counter() - t0
        ps = probes * args.degree
        out[name] = {"value": ps / max(r["alg_wall_time"], 1e-9),
                     "unit": UNIT, "e2e": ps / wall, "probes": probes,
                     "alg_wall_s": r["alg_wall_time"], "wall_s": wall,
                     "estimate": float(r["trace"][0]),
                     "samples": [float(x) for x in r["samples"][:probes, 0]]}
        del Ad
    out["path"] = path or ("imate cu_trace_estimator (cuSPARSE SpMV, "
                           "cuBLAS), built from the reference sources for "
                           "sm_100a, 1 GPU")
    return out


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap")
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# engine arm
# ---------------------------------------------------------------------------

def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def tensor_peak():
    """Dense bf16 tensor throughput (TFLOP/s): the burst figure, as for a
    kernel timed alone."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def ncu_traffic(kind):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/*.txt or *.md lines 'traffic <kind> <bytes_per_launch>')."""
    pdir = os.path.join(ROOT, "profiles")
    try:
        for fn in sorted(os.listdir(pdir)):
            if not fn.endswith((".txt", ".md")):
                continue
            with open(os.path.join(pdir, fn)) as f:
                for line in f:
                    parts = line.split()
                    if len(parts) == 3 and parts[0] == "traffic" and \
                            parts[1] == kind:
                        return float(parts[2])
    except OSError:
        pass
    return None


def run_engine_arm(args):
    import torch
    import torch.distributed as dist
    import imate_b200 as ib
    from imate_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    fn = getattr(ib, args.func)
    A32 = build_matrix(args, "float32")
    # the tensor-core row-group SpMM serves 16-row groups only; the block
    # kernel needs the block format
    mopts = dict(group_rows=16 if args.spmm == "row-group-tc" else "auto",
                 blocks=args.spmm == "block-tc")
    Aop = ib.Matrix(A32, **mopts)
    dev_op = Aop.get_device_operator()  # one-time upload, outside the timed region
    if args.spmm not in ("auto", "block-tc"):
        from imate_b200.batch import tune_operator, set_variant
        cands, _ = tune_operator(dev_op, args.probes, reps=1)
        pick = [i for i, c in enumerate(cands) if c["kind"] == args.spmm]
        if not pick:
            raise SystemExit("SpMM kernel %s is not available for this operator"
                             % args.spmm)
        set_variant(dev_op, args.probes, pick[-1])
    eng = ib.EngineOptions(block_size=args.probes, rng="parity")
    kw = dict(method="slq", gpu=True, num_gpu_devices=1, return_info=True,
              min_num_samples=args.probes, max_num_samples=args.probes,
              error_rtol=0.0, lanczos_degree=args.degree,
              orthogonalize=args.orthogonalize, seed=0)

    def step(i, op=Aop):
        # disjoint probe indices per rank and step (parity stream offsets)
        eng.first_probe = (rank * (args.warmup + args.steps) + i) * args.probes
        return fn(op, engine=eng, **kw)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    _lib.profile_begin()
    ev0.record()
    probe_steps = 0
    launches = 0
    estimates = []
    samples = []
    for i in range(args.steps):
        tr, info = step(args.warmup + i)
        samples.append(info["convergence"]["samples"])
        probe_steps += int(np.sum(info["engine"]["lanczos_size"]
                                  [:args.probes]))
        launches += int(info["engine"]["gpu_launches"])
        estimates.append(float(tr))
    ev1.record()
    torch.cuda.synchronize()
    kstats = _lib.profile_end()
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1) * 1e-3
    if world > 1:
        t = torch.tensor([elapsed], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
        ps = torch.tensor([probe_steps], dtype=torch.float64, device="cuda")
        dist.all_reduce(ps, op=dist.ReduceOp.SUM)
        total_probe_steps = float(ps.item())
    else:
        total_probe_steps = float(probe_steps)
    value = total_probe_steps / elapsed

    # roofline of the dominant kernel class
    dom = max(kstats, key=lambda k: kstats[k][1])
    nl, ms, by = kstats[dom]
    achieved = (by / nl) / (ms / nl * 1e-3) / 1e9 if nl else 0.0
    peak, peak_kind = peaks()
    # the committed ncu figures belong to the default workload only
    default_wl = (args.n == 262144 and args.probes == 256 and args.degree == 50
                  and args.orthogonalize == -1 and args.spmm == "block-tc"
                  and abs(args.shift - 0.1) < 1e-15)
    traffic = ncu_traffic(dom) if default_wl else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_kind,
                "bytes_per_launch": by / nl if nl else 0.0,
                "ms_per_launch": ms / nl if nl else 0.0,
                "share_of_kernel_time": ms / max(1e-12, sum(
                    v[1] for v in kstats.values())),
                "kernels": {k: {"launches": v[0], "ms": v[1],
                                "GB/s": (v[2] / (v[1] * 1e-3) / 1e9)
                                if v[1] > 0 else None}
                            for k, v in kstats.items() if v[0]}}

    # the SpMM on its own: its algorithmic (CSR) bytes per launch against HBM,
    # and, on the block format, the tensor-core work it issues (three FP16
    # products per 16-column stage) against the useful 2 nnz b flops
    if kstats.get("spmm", (0,))[0]:
        nl_s, ms_s, by_s = kstats["spmm"]
        per = ms_s / nl_s * 1e-3
        spmm_line = {"bound": "hbm", "unit": "GB/s", "peak": peak,
                     "peak_source": peak_kind,
                     "achieved": (by_s / nl_s) / per / 1e9,
                     "frac": (by_s / nl_s) / per / 1e9 / peak,
                     "bytes_per_launch": by_s / nl_s,
                     "ms_per_launch": per * 1e3,
                     "traffic": ncu_traffic("spmm") if default_wl else None}
        nblk, nst = dev_op.blocks_info(False)
        if nst and args.spmm == "block-tc":
            tp, tp_kind = tensor_peak()
            useful = 2.0 * A32.nnz * args.probes
            issued = 3.0 * nst * 128 * 16 * args.probes * 2.0
            spmm_line["tensor"] = {
                "blocks": nblk, "stages": nst,
                "useful_tflops": useful / per / 1e12,
                "issued_tflops": issued / per / 1e12,
                "useful_over_issued": useful / issued,
                "peak": tp, "peak_source": tp_kind, "unit": "TFLOP/s",
                "issued_frac": issued / per / 1e12 / tp,
                "a_image_bytes": nst * 8192.0}
        if kstats.get("split", (0,))[0]:
            nl_x, ms_x, by_x = kstats["split"]
            spmm_line["split"] = {
                "kernel": "k_x16_split (FP16 parts of the first vector of each "
                          "probe block; the reorthogonalisation pass writes "
                          "the parts of the others)",
                "launches": nl_x, "products": nl_s,
                "ms_per_launch": ms_x / nl_x,
                "achieved_gbs": (by_x / nl_x) / (ms_x / nl_x * 1e-3) / 1e9}
        roofline["spmm"] = spmm_line

    line = {
        "metric": metric_of(args), "value": value, "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": workload_config(args, A32.nnz),
        "roofline": roofline, "gpu_launches": launches, "clocks": clk,
    }

    # accuracy vs the FP64 oracle
    oracle_val = load_oracle(args)
    est = float(np.mean(estimates))
    line["accuracy"] = {
        "estimate_mean": est,
        "fp64_oracle": oracle_val,
        "rel_err_vs_oracle": (abs(est - oracle_val) / abs(oracle_val)
                              if oracle_val else None),
        "probes_in_mean": args.probes * args.steps * world,
        "note": "precision error (mixed vs FP64 on identical probes) is in "
                "fp64_plain.rel_diff_same_probes",
    }
    s_mixed = np.concatenate([np.ravel(np.asarray(x, float)[:args.probes])
                              for x in samples])
    line["accuracy"]["standard_error"] = float(
        np.std(s_mixed, ddof=1) / np.sqrt(s_mixed.size)) \
        if s_mixed.size > 1 else None
    nref = args.fp64_ref_probes
    if nref < 0:
        nref = 1024 if args.func != "logdet" else 0
    if rank == 0 and nref > 0:
        # high-sample FP64 SLQ (FP64 operator and vectors, block width 256)
        # on probes 0 .. nref-1 of the parity stream: the full-size FP64
        # reference of a function without a direct FP64 oracle
        A64 = A32.astype(np.float64)
        Mref = ib.Matrix(A64)
        eref = ib.EngineOptions(block_size=256, rng="parity")
        t0 = time.perf_counter()
        tr_ref, info_ref = fn(Mref, engine=eref, **dict(
            kw, min_num_samples=nref, max_num_samples=nref))
        torch.cuda.synchronize()
        secs_ref = time.perf_counter() - t0
        sref = np.asarray(info_ref["convergence"]["samples"][:nref], float)
        se_ref = float(np.std(sref, ddof=1) / np.sqrt(nref))
        se_mix = line["accuracy"]["standard_error"] or 0.0
        diff = est - float(tr_ref)
        line["accuracy"]["fp64_high_sample"] = {
            "estimate": float(tr_ref), "probes": nref,
            "standard_error": se_ref, "seconds": secs_ref,
            "rel_standard_error": se_ref / abs(float(tr_ref)),
            "rel_diff_of_mixed_mean": abs(diff) / abs(float(tr_ref)),
            "z_of_mixed_mean": diff / max(np.hypot(se_ref, se_mix), 1e-300),
            "note": "different probes (mixed: the timed steps' probes; "
                    "FP64: probes 0..%d), so the difference is Monte-Carlo "
                    "error, z in units of the combined standard error"
                    % (nref - 1)}
        del Mref
        torch.cuda.empty_cache()

    if rank == 0 and args.fp64_probes > 0:
        # plain FP64 per-probe path (block width 1) on the same matrix
        A64 = A32.astype(np.float64)
        Aop64 = ib.Matrix(A64)
        Aop64.get_device_operator()
        e64 = ib.EngineOptions(block_size=1, rng="parity")
        nprb = args.fp64_probes
        kw64 = dict(kw, min_num_samples=nprb, max_num_samples=nprb)
        fn(Aop64, engine=e64, **dict(kw64, min_num_samples=1,
                                              max_num_samples=1))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        tr64, info64 = fn(Aop64, engine=e64, **kw64)
        e1.record()
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) * 1e-3
        ps64 = int(np.sum(info64["engine"]["lanczos_size"][:nprb]))
        # same probes in mixed precision
        e32 = ib.EngineOptions(block_size=min(args.probes, 256), rng="parity")
        tr32, info32 = fn(Aop, engine=e32, **kw64)
        s64 = np.asarray(info64["convergence"]["samples"][:nprb], float)
        s32 = np.asarray(info32["convergence"]["samples"][:nprb], float)
        v64 = ps64 / t64
        line["fp64_plain"] = {
            "value": v64, "unit": UNIT, "probes": nprb, "block_size": 1,
            "dtype": "f64", "speedup_mixed_batched": value / world / v64,
            "rel_diff_same_probes": float(np.max(np.abs(s32 - s64) /
                                                 np.abs(s64))),
            "rel_diff_same_probes_path": "8 probes, block width 8 (row-group "
                                         "SpMM)",
        }
        if args.spmm == "block-tc" and args.probes in (128, 256):
            # the bench's own path (block SpMM at b = 128 / 256) against the
            # FP64 engine on the same probes
            kwb = dict(kw, min_num_samples=args.probes,
                       max_num_samples=args.probes)
            eb = ib.EngineOptions(block_size=args.probes, rng="parity")
            _, ib64 = fn(Aop64, engine=eb, **kwb)
            _, ib32 = fn(Aop, engine=eb, **kwb)
            t64 = np.asarray(ib64["convergence"]["samples"][:args.probes],
                             float)
            t32 = np.asarray(ib32["convergence"]["samples"][:args.probes],
                             float)
            line["fp64_plain"]["rel_diff_same_probes_block_spmm"] = float(
                np.max(np.abs(t32 - t64) / np.abs(t64)))
            line["fp64_plain"]["mean_rel_diff_same_probes_block_spmm"] = \
                float(np.mean((t32 - t64) / np.abs(t64)))
        del Aop64
        torch.cuda.empty_cache()

    if rank == 0:
        # end to end through the public API from host arrays
        if not args.no_e2e:
            h2d = A32.data.nbytes + A32.indices.nbytes + A32.indptr.nbytes
            # one untimed call first: its device allocations (formats,
            # workspace) then come from the allocator's cache, as in a
            # process that has called before
            eng.first_probe = 0
            fn(A32, engine=eng, **kw)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e_ps = 0
            nsteps = max(1, min(args.steps, 3))
            for i in range(nsteps):
                # the drop-in call on the scipy matrix: every step uploads
                # it and builds its device formats (default options:
                # blocks='auto' gives this float32 matrix the block format)
                eng.first_probe = i * args.probes
                tr, info = fn(A32, engine=eng, **kw)
                e_ps += int(np.sum(info["engine"]["lanczos_size"]
                                   [:args.probes]))
            torch.cuda.synchronize()
            te = time.perf_counter() - t0
            line["e2e"] = {"value": e_ps / te, "unit": UNIT,
                           "h2d_bytes_per_step": int(h2d),
                           "d2h_bytes_per_step": int(args.probes * 8 * 2),
                           "steps": nsteps,
                           "path": "imate_b200.%s(scipy CSR on host), "
                                   "default options (block format)"
                                   % args.func}

        if not args.no_cpu_baseline:
            threads = cpu_threads()
            v, probes, secs, kind = reference_baseline(A32, args, threads)
            line["cpu_baseline"] = {
                "value": v, "unit": UNIT, "cores": threads, "kind": kind,
                "sample": "%d probes x %d steps, FP32, full reorth, %.1f s"
                          % (probes, args.degree, secs)}
        print(json.dumps(line), flush=True)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# other workloads (one JSON line each; not the headline line)
# ---------------------------------------------------------------------------

def _timed(fn, steps):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    out = [fn(i) for i in range(steps)]
    e1.record()
    torch.cuda.synchronize()
    return out, e0.elapsed_time(e1) * 1e-3


def run_batched(args):
    """64 sparse SPD correlation matrices (sizes log-uniform 2^10..2^17 and
    length scales U(0.002, 0.05) from PCG64 seed 2; points from seed 1000+i;
    kernel cut 0.05; diagonal shift --shift), built on the device, FP32;
    512 probes each, lanczos_degree 40, no reorthogonalisation; one batch
    plan (one CUDA graph, autotuned SpMM and block width per matrix).  A
    step is one launch of the plan over all matrices."""
    import torch
    import imate_b200 as ib
    from imate_b200.batch import BatchPlan
    from imate_b200.sample_matrices import (correlation_matrix_device,
                                            batched_correlation_sizes)
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    probes = 512 if args.probes == 256 else args.probes
    degree = 40 if args.degree == 50 else args.degree
    sizes, scales = batched_correlation_sizes(args.batch_count, seed=2)
    mats, mats64, nnz = [], [], []
    t0 = time.perf_counter()
    for i, (n, sc) in enumerate(zip(sizes, scales)):
        ip, ind, dat, _ = correlation_matrix_device(
            int(n), scale=float(sc), threshold=0.05, shift=args.shift,
            seed=1000 + i, dtype="float32")
        mats.append(ib.DeviceMatrix(ip, ind, dat, (int(n), int(n))))
        nnz.append(int(ind.numel()))
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    ests = [dict(func="logdet", A=M, min_num_samples=probes,
                 max_num_samples=probes, error_rtol=0.0,
                 lanczos_degree=degree, orthogonalize=0, seed=i)
            for i, M in enumerate(mats)]
    t0 = time.perf_counter()
    plan = BatchPlan(ests, autotune=True, num_gpu_devices=1)
    plan_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        plan.run()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    outs, elapsed = _timed(lambda i: plan.run(), args.steps)
    clk = clocks.stop()
    ps = sum(int(np.sum(info["engine"]["lanczos_size"])) for res in outs
             for _, info in res)
    value = ps / elapsed
    widths = [t["width"] for t in plan.tuning]
    kinds = {}
    for t in plan.tuning:
        rep = t["report"][t["width"]]["direct"]
        k = rep["candidates"][rep["chosen"]]["kind"]
        kinds[k] = kinds.get(k, 0) + 1
    # algorithmic bytes of the whole graph per step: per matrix and
    # Lanczos step, the SpMM of every block plus the update pass
    by = 0.0
    flops = 0.0
    for n, z, w in zip(sizes, nnz, widths):
        blocks = -(-probes // w)
        spmm = z * 8.0 + (n + 1) * 4.0 + 2.0 * n * w * 4.0
        upd = 4.0 * n * w * 4.0
        by += degree * blocks * (spmm + upd)
        flops += degree * 2.0 * z * probes
    achieved = by * args.steps / elapsed / 1e9
    peak, peak_kind = peaks()
    # plain FP64 per-probe path (block width 1) on three of the matrices
    order = np.argsort(sizes)
    pick = [int(order[len(order) // 4]), int(order[len(order) // 2]),
            int(order[-1])]
    ps64, t64 = 0, 0.0
    for i in pick:
        ip, ind, dat, _ = correlation_matrix_device(
            int(sizes[i]), scale=float(scales[i]), threshold=0.05,
            shift=args.shift, seed=1000 + i, dtype="float64")
        M64 = ib.DeviceMatrix(ip, ind, dat, (int(sizes[i]),) * 2,
                              group_rows=0)
        kw64 = dict(method="slq", gpu=True, num_gpu_devices=1, return_info=True,
                    min_num_samples=4, max_num_samples=4, error_rtol=0.0,
                    lanczos_degree=degree, orthogonalize=0, seed=i,
                    engine=ib.EngineOptions(block_size=1))
        ib.logdet(M64, **dict(kw64, min_num_samples=1, max_num_samples=1))
        (res,), t = _timed(lambda k: ib.logdet(M64, **kw64), 1)
        ps64 += int(np.sum(res[1]["engine"]["lanczos_size"]))
        t64 += t
        del M64
    v64 = ps64 / t64
    line = {
        "workload_kind": "batched", "metric": "batched SLQ logdet "
        "probe*steps/s (64 matrices, one graph launch)", "value": value,
        "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "%d sparse SPD correlation matrices, one "
                               "batch plan" % len(mats),
                   "total_rows": int(np.sum(sizes)), "total_nnz": int(sum(nnz)),
                   "max_nnz_per_row": float(max(z / n for z, n in
                                                zip(nnz, sizes))),
                   "probes_per_matrix": probes, "lanczos_degree": degree,
                   "orthogonalize": 0, "diag_shift": args.shift,
                   "l2": "inputs larger than L2 (matrices %.1f GB)"
                         % (sum(nnz) * 8 / 1e9)},
        "graph": {"kernels": plan.graph_kernels, "nodes": plan.graph_nodes,
                  "build_s": build_s, "plan_s": plan_s,
                  "widths": {str(w): widths.count(w) for w in sorted(
                      set(widths))},
                  "spmm_kernels": kinds},
        "roofline": {"bound": "hbm", "kernel": "whole graph (SpMM + update "
                     "passes)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "spmm_fp32_tflops": flops * args.steps / elapsed / 1e12},
        "gpu_launches": plan.graph_kernels * args.steps, "clocks": clk,
        "fp64_plain": {"value": v64, "unit": UNIT, "probes": 4 * len(pick),
                       "block_size": 1, "matrices": [int(sizes[i])
                                                     for i in pick],
                       "speedup_mixed_batched": value / v64},
    }
    print(json.dumps(line), flush=True)


def run_sweep(args):
    """t-sweep of logdet(A + tI) and traceinv(A + tI) over 512 log-spaced t
    in [1e-4, 1e2] on the benchmark matrix (FP32): the surrogate (trained
    on 32 SLQ points, gated on 16 held-out points, SLQ fallback) against
    per-t SLQ and against one shift-relation SLQ run over all 512 t."""
    import torch
    import imate_b200 as ib
    from imate_b200.surrogate import SweepSurrogate
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    A32 = build_matrix(args, "float32")
    t_grid = np.logspace(-4, 2, 512)
    opts = dict(min_num_samples=args.probes, max_num_samples=args.probes,
                num_gpu_devices=1,
                error_rtol=0.0, lanczos_degree=args.degree,
                orthogonalize=args.orthogonalize, seed=0)
    funcs = {"log": ib.logdet, "inv": ib.traceinv}
    Aop = ib.AffineMatrixFunction(A32)
    Aop.get_device_operator()
    out = {}
    for func, f in funcs.items():
        S = SweepSurrogate(A32, func=func, t_min=1e-4, t_max=1e2,
                           num_train=32, checks_per_interval=4, rtol=1e-3,
                           **opts)
        S.Aop = Aop  # share the resident operator
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.fit()
        torch.cuda.synchronize()
        fit_s = time.perf_counter() - t0
        vals = None
        reps = max(3, args.steps)
        t0 = time.perf_counter()
        for _ in range(reps):
            vals = S(t_grid)
        torch.cuda.synchronize()
        answer_s = (time.perf_counter() - t0) / reps
        fallback = int(np.sum(S.last_fallback))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        shift_vals = f(Aop, method="slq", gpu=True, parameters=t_grid, **opts)
        torch.cuda.synchronize()
        shift_s = time.perf_counter() - t0
        k = 3
        t0 = time.perf_counter()
        for t in t_grid[::len(t_grid) // k][:k]:
            f(Aop, method="slq", gpu=True, parameters=float(t), **opts)
        torch.cuda.synchronize()
        per_t_s = (time.perf_counter() - t0) / k
        # relative error judged as the held-out gate judges it: against
        # max(|value|, rtol_floor * mean |value|), since logdet(A + tI)
        # crosses zero inside the sweep
        floor = S.rtol_floor * float(np.mean(np.abs(shift_vals)))
        err = np.abs(vals - shift_vals) / np.maximum(np.abs(shift_vals),
                                                     floor)
        out[func] = {
            "fit_s": fit_s, "answer_512_s": answer_s,
            "per_t_slq_s": per_t_s, "per_t_slq_512_s": 512 * per_t_s,
            "shift_relation_slq_512_s": shift_s,
            "speedup_vs_per_t": 512 * per_t_s / answer_s,
            "speedup_vs_per_t_incl_fit": 512 * per_t_s / (answer_s + fit_s),
            "speedup_vs_shift_relation": shift_s / answer_s,
            "fallback_points": fallback,
            "held_out_max_rel_err": float(np.max(S.check_error)),
            "max_rel_diff_vs_shift_relation_slq": float(np.max(err)),
            "points_over_1e-3_vs_shift_relation_slq": int(np.sum(err >
                                                                 1e-3)),
            "train_timings": dict(S.timings),
        }
    line = {
        "workload_kind": "sweep", "metric": "512-point t-sweep answer time, "
        "surrogate vs per-t SLQ", "value": out["log"]["speedup_vs_per_t"],
        "unit": "x faster than per-t SLQ (logdet)", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": dict(workload_config(args, A32.nnz),
                       sweep="512 t log-spaced over [1e-4, 1e2]",
                       per_t_note="per-t SLQ time = mean of 3 single-t "
                                  "runs x 512"),
        "sweeps": out,
    }
    print(json.dumps(line), flush=True)


def run_gram_large(args):
    """logdet(X^T X + lambda I), lambda = 1e-2, X 8388608 x 2097152 sparse
    (16 nonzeros per column at uniform rows, N(0,1) values, PCG64 seed 4),
    FP32 CSC; Lanczos on the normal operator, lanczos_degree 60, 1024
    probes in blocks of --block, no reorthogonalisation."""
    import torch
    import imate_b200 as ib
    from imate_b200.sample_matrices import sparse_gram_design
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t0 = time.perf_counter()
    X = sparse_gram_design(8388608, 2097152, 16, seed=4)
    build_s = time.perf_counter() - t0
    probes = 1024 if args.probes == 256 else args.probes
    degree = 60 if args.degree == 50 else args.degree
    G = ib.GramAffineMatrixFunction(X)
    G.get_device_operator(need_transpose=True)
    kw = dict(method="slq", gpu=True, num_gpu_devices=1, return_info=True, parameters=1e-2,
              min_num_samples=probes, max_num_samples=probes,
              error_rtol=0.0, lanczos_degree=degree, orthogonalize=0, seed=0)
    eng = ib.EngineOptions(block_size=args.block)
    for _ in range(args.warmup):
        ib.logdet(G, engine=eng, **kw)
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    from imate_b200 import _lib
    _lib.profile_begin()
    outs, elapsed = _timed(lambda i: ib.logdet(G, engine=eng, **kw),
                           args.steps)
    kstats = _lib.profile_end()
    clk = clocks.stop()
    ps = sum(int(np.sum(info["engine"]["lanczos_size"])) for _, info in outs)
    value = ps / elapsed
    nl, ms, by = kstats["spmm"]
    achieved = (by / nl) / (ms / nl * 1e-3) / 1e9 if nl else 0.0
    peak, peak_kind = peaks()
    # plain FP64 per-probe path on 4 probes, and the same probes mixed
    G64 = ib.GramAffineMatrixFunction(X.astype(np.float64))
    kw64 = dict(kw, min_num_samples=4, max_num_samples=4)
    ib.logdet(G64, engine=ib.EngineOptions(block_size=1),
              **dict(kw64, min_num_samples=1, max_num_samples=1))
    (r64,), t64 = _timed(lambda i: ib.logdet(
        G64, engine=ib.EngineOptions(block_size=1), **kw64), 1)
    r32 = ib.logdet(G, engine=ib.EngineOptions(block_size=4), **kw64)
    s64 = np.asarray(r64[1]["convergence"]["samples"][:4], float)
    s32 = np.asarray(r32[1]["convergence"]["samples"][:4], float)
    v64 = int(np.sum(r64[1]["engine"]["lanczos_size"])) / t64
    est = float(np.mean([tr for tr, _ in outs]))
    line = {
        "workload_kind": "gram-large", "metric": "Gram-form SLQ logdet "
        "probe*steps/s (normal operator X^T X + lambda I)", "value": value,
        "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "logdet(X^T X + 1e-2 I), X 8388608 x 2097152,"
                               " 16 nnz/col, CSC FP32", "nnz": int(X.nnz),
                   "probes": probes, "block_size": args.block,
                   "lanczos_degree": degree, "orthogonalize": 0,
                   "host_build_s": build_s,
                   "l2": "inputs larger than L2 (basis blocks > 2 GB)"},
        "roofline": {"bound": "hbm", "kernel": "spmm", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": peak_kind,
                     "note": "algorithmic bytes count each X value once; the "
                             "random rows make every nonzero gather a "
                             "b-wide row of the other operand"},
        "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in
                    kstats.items() if v[0]},
        "estimate": est, "estimate_error": float(np.mean(
            [info["error"]["absolute_error"] for _, info in outs])),
        "clocks": clk,
        "fp64_plain": {"value": v64, "unit": UNIT, "probes": 4,
                       "block_size": 1, "speedup_mixed_batched": value / v64,
                       "rel_diff_same_probes": float(np.max(
                           np.abs(s32 - s64) / np.abs(s64)))},
    }
    print(json.dumps(line), flush=True)


def run_dense(args):
    """logdet of a dense SPD exponential-kernel correlation matrix: n = 16384
    points uniform in the unit square (PCG64 seed 1), scale 0.02, every pair
    kept, diagonal shift --shift; FP32 row-major on the host.  256 probes,
    lanczos_degree 50, full reorthogonalisation.  The operator is the
    tensor-core dense product (3-term TF32 split, FP32 accumulation)."""
    import torch
    import imate_b200 as ib
    from imate_b200 import _lib
    from imate_b200.sample_matrices import dense_correlation_matrix
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    n = 16384 if args.n == 262144 else args.n
    t0 = time.perf_counter()
    A32 = dense_correlation_matrix(n, scale=0.02, shift=args.shift, seed=1,
                                   dtype="float32", device="cuda")
    build_s = time.perf_counter() - t0
    # FP64 oracle: dense Cholesky of the stored (float32) matrix in float64
    L = torch.linalg.cholesky(torch.from_numpy(A32).to("cuda",
                                                        torch.float64))
    exact = float(2.0 * torch.log(torch.diagonal(L)).sum())
    del L
    torch.cuda.empty_cache()

    Aop = ib.Matrix(A32)
    Aop.get_device_operator()  # upload + TF32 split, outside the timing
    eng = ib.EngineOptions(block_size=args.probes, rng="parity")
    kw = dict(method="slq", gpu=True, num_gpu_devices=1, return_info=True,
              min_num_samples=args.probes, max_num_samples=args.probes,
              error_rtol=0.0, lanczos_degree=args.degree,
              orthogonalize=args.orthogonalize, seed=0)

    def step(i):
        eng.first_probe = i * args.probes
        return ib.logdet(Aop, engine=eng, **kw)

    for i in range(args.warmup):
        step(i)
    clocks = ClockSampler(local)
    clocks.start()
    _lib.profile_begin()
    outs, elapsed = _timed(lambda i: step(args.warmup + i), args.steps)
    kstats = _lib.profile_end()
    clk = clocks.stop()
    ps = sum(int(np.sum(info["engine"]["lanczos_size"][:args.probes]))
             for _, info in outs)
    launches = sum(int(info["engine"]["gpu_launches"]) for _, info in outs)
    value = ps / elapsed
    est = float(np.mean([float(tr) for tr, _ in outs]))

    # tensor roofline of the dense product: useful 2 n^2 b flops per call,
    # issued as three TF32 products; TF32 runs at half the bf16 rate
    nl, ms, _ = kstats["spmm"]
    per_call = ms / nl * 1e-3 if nl else float("nan")
    useful = 2.0 * n * n * args.probes / per_call / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            bf16 = float(json.load(f)["bf16_tflops"])
        src = "measured bf16 burst / 2"
    except (OSError, KeyError, ValueError):
        bf16, src = 1590.0, "fallback bf16 burst / 2"
    tf32_peak = bf16 / 2.0
    # DRAM bytes per product from the committed ncu capture at n = 8192
    # (traffic there equals the algorithmic bytes: A parts once, probe parts
    # and Y once), scaled by the algorithmic bytes of this size
    t8 = ncu_traffic("dense") if args.probes == 256 else None
    alg = lambda m: 8.0 * m * m + 12.0 * m * args.probes  # noqa: E731
    traffic = t8 * alg(n) / alg(8192) if t8 else None
    line = {
        "workload_kind": "dense", "metric": "dense SLQ logdet probe*steps/s "
        "(tensor-core operator)", "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "dense SPD exponential-kernel correlation "
                               "matrix (scale 0.02, diag shift %g), SLQ "
                               "logdet" % args.shift, "n": n,
                   "probes_per_step": args.probes,
                   "lanczos_degree": args.degree,
                   "orthogonalize": args.orthogonalize, "rng": "parity",
                   "host_build_s": build_s,
                   "l2": "inputs larger than L2 (split matrix %.1f GB)"
                         % (8.0 * n * n / 1e9)},
        "roofline": {"bound": "tensor", "kernel": "k_dense_tc (+ probe "
                     "split)", "achieved": 3.0 * useful, "peak": tf32_peak,
                     "unit": "TFLOP/s", "frac": 3.0 * useful / tf32_peak,
                     "traffic": traffic, "peak_source": src,
                     "traffic_note": "DRAM bytes per product: ncu at n = "
                                     "8192 scaled by algorithmic bytes",
                     "algorithmic_bytes_per_call": alg(n),
                     "useful_tflops": useful, "ms_per_call": per_call * 1e3,
                     "calls": nl,
                     "share_of_kernel_time": ms / max(1e-12, sum(
                         v[1] for v in kstats.values()))},
        "kernels": {k: {"launches": v[0], "ms": v[1]} for k, v in
                    kstats.items() if v[0]},
        "gpu_launches": launches, "clocks": clk,
        "accuracy": {"estimate_mean": est, "fp64_cholesky": exact,
                     "rel_err_vs_oracle": abs(est - exact) / abs(exact),
                     "probes_in_mean": args.probes * args.steps},
    }
    if not args.no_e2e:
        h2d = A32.nbytes
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_ps = 0
        nsteps = max(1, min(args.steps, 3))
        for i in range(nsteps):
            fresh = ib.Matrix(A32)
            eng.first_probe = i * args.probes
            tr, info = ib.logdet(fresh, engine=eng, **kw)
            e_ps += int(np.sum(info["engine"]["lanczos_size"][:args.probes]))
            del fresh
        torch.cuda.synchronize()
        te = time.perf_counter() - t0
        line["e2e"] = {"value": e_ps / te, "unit": UNIT,
                       "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(args.probes * 8 * 2),
                       "steps": nsteps,
                       "path": "imate_b200.logdet(numpy float32 array)"}
    del Aop
    torch.cuda.empty_cache()
    if args.fp64_probes > 0:
        nprb = args.fp64_probes
        gpu_ref = reference_gpu_sample(
            A32, args, probes=nprb,
            path="imate cu_trace_estimator on cuDenseMatrix (cuBLAS gemv), "
                 "built from the reference sources for sm_100a, 1 GPU")
        if gpu_ref is not None:
            # the same probes through this engine (parity stream, seed 0)
            e8 = ib.EngineOptions(block_size=nprb, rng="parity")
            _, info8 = ib.logdet(ib.Matrix(A32), engine=e8, **dict(
                kw, min_num_samples=nprb, max_num_samples=nprb))
            mine = np.asarray(info8["convergence"]["samples"][:nprb], float)
            s64 = np.asarray(gpu_ref["f64"]["samples"], float)
            gpu_ref["rel_diff_same_probes_vs_f64"] = float(
                np.max(np.abs(mine - s64) / np.abs(s64)))
            gpu_ref["speedup_vs_f64"] = value / gpu_ref["f64"]["value"]
            gpu_ref["speedup_vs_f32"] = value / gpu_ref["f32"]["value"]
            line["reference_gpu"] = gpu_ref
    if not args.no_cpu_baseline:
        threads = cpu_threads()
        v, probes, secs, kind = reference_baseline(A32, args, threads)
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": "%d probes x %d steps, FP32 dense, full reorth, %.1f s"
                      % (probes, args.degree, secs)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.workload != "c2prime":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference CPU path is timed on the "
                              "headline workload only"}), flush=True)
            return
        {"batched": run_batched, "sweep": run_sweep,
         "gram-large": run_gram_large, "dense": run_dense}[args.workload](args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_engine_arm(args)


if __name__ == "__main__":
    main()
