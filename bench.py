"""Benchmark: C = A*A on the 27-point stencil over a 96^3 grid (884,736 rows,
23.4M nonzeros), learned-binned SpGEMM vs the plain two-pass method on one
B200, through the library's C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full C = A*A (validation off, C allocated and released by the
library), inputs resident in HBM.  Timed with CUDA events on the stream the
library launches on, L2 flushed between steps; under torchrun every rank runs
its own replica and the slowest rank's time counts (weak scaling).  Rank 0
prints one JSON line.

--impl reference times the reference arm on the host cores: the reference
has no CPU SpMSpM path, so the arm is the CPU restatement of its arithmetic
(oracle/spgemm_oracle.c, OpenMP, canonical FP32 order) on a bounded row
sample of the same workload.
"""
from __future__ import annotations

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

METRIC = "SpGEMM GFLOP/s & ms per C=A·A, learned-binned vs plain 2-pass on same B200"
WORKLOAD = "C=A*A, A = 27-point 3D stencil on a 96^3 grid (884,736 rows), FP32 N(0,1), diag 26+sum|row|"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def csr_bytes(rows, nnz, rp_bytes=4):
    return nnz * 8 + (rows + 1) * rp_bytes


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return PEAKS_FALLBACK["hbm_gbs"], "fallback"


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` on this workload, from the committed
    ncu summary (profiles/traffic.txt: `<kernel> <workload> <bytes>`)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel and parts[1] == "stencil96":
                    return float(parts[2])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (one `nvidia-smi -lms 20` process for the whole region)."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._proc = None

    def __enter__(self):
        # one synchronous query first: nvidia-smi's first start-up is slow and
        # must not land inside the timed region
        subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=clocks.sm", "--format=csv"],
                       capture_output=True, timeout=60)
        try:
            self._proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                           "--format=csv,noheader,nounits", "-lms", "20"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.1)  # first sample before the region starts
        except OSError:
            self._proc = None
        return self

    def __exit__(self, *a):
        if self._proc is None:
            return
        time.sleep(0.05)  # one more sample after the region
        self._proc.terminate()
        try:
            out, _ = self._proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self._proc.kill()
            out, _ = self._proc.communicate()
        for line in out.splitlines():
            if line.strip():
                self.samples.append([x.strip() for x in line.split(",")])

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 4 + i and s[4 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_sample(A, target_s: float, threads: int | None = None):
    """Times the oracle (FP32 canonical Gustavson, OpenMP) on leading rows of A*A,
    sized to about target_s seconds.  Returns (GFLOP/s, dict)."""
    from oracle import oracle
    from rtspmspm_b200 import gen

    if threads:
        oracle.set_threads(threads)
    cores = oracle.num_threads()
    prod = gen.row_products(A, A)
    cum = np.cumsum(prod)
    # calibrate on ~0.5% of the work, then size the sample
    r1 = int(np.searchsorted(cum, cum[-1] * 0.005)) + 1
    t = time.perf_counter()
    oracle.baseline_rows(A, A, 0, r1)
    dt = max(time.perf_counter() - t, 1e-4)
    rate = float(cum[r1 - 1]) / dt
    want = min(float(cum[-1]), rate * target_s)
    r2 = int(np.searchsorted(cum, want)) + 1
    r2 = min(r2, A.rows)
    # a workload shorter than the target is run whole, pass after pass,
    # until the target time is filled
    passes = 0
    t = time.perf_counter()
    while True:
        oracle.baseline_rows(A, A, 0, r2)
        passes += 1
        dt = time.perf_counter() - t
        if r2 < A.rows or dt >= target_s:
            break
    work = float(cum[r2 - 1]) * passes
    return 2.0 * work / dt / 1e9, {"cores": cores, "rows": r2, "products": int(work), "seconds": dt,
                                   "passes": passes}


def scipy_sample(A, target_s: float):
    """scipy.sparse A[:r] @ A (single-threaded SMMP, FP32 CSR) on the leading
    rows of the product, sized to about target_s seconds: a second CPU
    reference beside the oracle.  Returns (GFLOP/s, rows, seconds) or None."""
    try:
        import scipy.sparse as sp
    except ImportError:
        return None
    from rtspmspm_b200 import gen

    S = sp.csr_matrix((A.val, A.col_idx, A.row_ptr), shape=(A.rows, A.cols))
    cum = np.cumsum(gen.row_products(A, A))
    r1 = int(np.searchsorted(cum, cum[-1] * 0.002)) + 1
    t = time.perf_counter()
    S[:r1] @ S
    rate = float(cum[r1 - 1]) / max(time.perf_counter() - t, 1e-4)
    r2 = min(A.rows, int(np.searchsorted(cum, min(float(cum[-1]), rate * target_s))) + 1)
    t = time.perf_counter()
    S[:r2] @ S
    dt = time.perf_counter() - t
    return 2.0 * float(cum[r2 - 1]) / dt / 1e9, r2, dt


def parity_sample(A, c_rp, c_col, c_val, lo: int, hi: int) -> dict:
    """Rows lo..hi-1 of the engine's C = A*A (host arrays) against the oracle
    (the checker): structure, bit equality with the FP32 canonical oracle,
    the error relative to sum|a*b| and the error against the FP64 twin."""
    from oracle import oracle
    from rtspmspm_b200.gen import Csr

    s0, s1 = int(A.row_ptr[lo]), int(A.row_ptr[hi])
    sub = Csr(hi - lo, A.cols, np.asarray(A.row_ptr[lo:hi + 1], np.int64) - s0, A.col_idx[s0:s1], A.val[s0:s1])
    R = oracle.spgemm(sub, A)
    c0, c1 = int(c_rp[lo]), int(c_rp[hi])
    rp = np.asarray(c_rp[lo:hi + 1], np.int64) - c0
    col, val = np.asarray(c_col[c0:c1]), np.asarray(c_val[c0:c1], np.float32)
    same = bool(np.array_equal(rp, R.row_ptr) and np.array_equal(col, R.col_idx))
    out = {"rows": f"{lo}..{hi - 1}", "nnz": int(c1 - c0), "structure_exact": same}
    if same:
        v = val.astype(np.float64)
        rel = np.abs(v - R.val.astype(np.float64)) / np.maximum(R.bound, np.finfo(np.float64).tiny)
        e64 = np.abs(v - R.val64)
        out.update({"bit_exact_fp32": bool(np.array_equal(val.view(np.uint32), R.val.view(np.uint32))),
                    "max_rel_err_vs_sum_abs": float(rel.max()) if rel.size else 0.0,
                    "max_abs_err_fp64": float(e64.max()) if e64.size else 0.0,
                    "mean_abs_err_fp64": float(e64.mean()) if e64.size else 0.0})
    return out


def sample_text(info, what: str) -> str:
    head = f"{info['passes']} passes over all" if info["passes"] > 1 else "leading"
    return f"{head} {info['rows']} rows of {what} ({info['products']} products, {info['seconds']:.1f} s)"


def workload_config(A, products: int, nnz_c: int, world: int) -> dict:
    """The `config` object of both arms: the workload and how it is timed."""
    return {"workload": WORKLOAD, "rows": A.rows, "nnz_a": A.nnz, "products": products, "nnz_c": nnz_c,
            "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) before every step",
            "index": "int32 CSR"}


def reference_arm(args, A):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle
    from rtspmspm_b200 import gen

    products = int(gen.row_products(A, A).sum())
    nnz_c = int(oracle.row_nnz(A, A).sum())
    per_step = max(2.0, min(20.0, 60.0 / max(1, args.steps + args.warmup)))
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        v, info = cpu_sample(A, per_step)
        if i >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    sample = f"{sample_text(info, 'the stencil-96 C=A*A')} per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(info["seconds"] / info["passes"] * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(A, products, nnz_c, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": round(value, 4), "unit": "GFLOP/s", "cores": info["cores"], "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def timed_median(fn, k, flush, stream):
    """Median CUDA-event time (ms) of k calls of fn on `stream`, L2 flushed
    (256 MB write) before each."""
    import torch

    ts = []
    for _ in range(k):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def measure_single(eng, A, algos, warmup, steps, flush, stream, index_bits=32, use_tuning=False):
    """Per-method timings of C = A*A on device-resident A (validation off):
    median ms, GFLOP/s, and the stage breakdown, prediction and heavy-row
    counts of one extra call with stage timing on (the context's tuning when
    use_tuning, else the defaults)."""
    from rtspmspm_b200 import DeviceCsr, _lib, gen

    dA = DeviceCsr.from_host(A, index_bits=index_bits)
    products = int(gen.row_products(A, A).sum())
    sa = dA.struct()
    out = {"rows": A.rows, "nnz_a": A.nnz, "products": products}
    for algo in algos:
        o = eng.opts(algo=algo, skip_validation=True, stage_timing=False, use_tuning=use_tuning)
        for _ in range(warmup):
            c = _lib.SpgCsr()
            eng.multiply_raw(sa, sa, o, c, _lib.SpgReport())
            eng.free_raw(c)
        holder = {}

        def step():
            c = _lib.SpgCsr()
            rep = _lib.SpgReport()
            eng.multiply_raw(sa, sa, o, c, rep)
            holder["rep"] = rep
            eng.free_raw(c)

        ms = timed_median(step, steps, flush, stream)
        c = _lib.SpgCsr()
        rep = _lib.SpgReport()
        eng.multiply_raw(sa, sa, eng.opts(algo=algo, skip_validation=True, stage_timing=True, use_tuning=use_tuning),
                         c, rep)
        eng.free_raw(c)
        r = rep.as_dict()
        out[algo] = {"ms": round(ms, 3), "gflops": round(2 * products / ms / 1e6, 2), "nnz_c": r["nnz_c"],
                     "stages_ms": {k: round(v, 3) for k, v in r["stages_ms"].items()},
                     "rows_predicted": r["rows_predicted"], "rows_overflow": r["rows_overflow"],
                     "rows_heavy": r["rows_heavy"], "kernel_launches": holder["rep"].kernel_launches,
                     "small_path": r["small_path"]}
        if algo == "learned":
            out[algo]["misprediction_rate"] = round(r["rows_overflow"] / max(1, r["rows_predicted"]), 6)
    if "plain" in out and "learned" in out:
        out["speedup_learned_vs_plain"] = round(out["plain"]["ms"] / out["learned"]["ms"], 4)
    del dA
    return out


CUSPARSE_ALGS = (("ALG1", 1), ("ALG2", 2), ("ALG3", 0))


def measure_cusparse(eng, sa, products, warmup, steps, flush, stream):
    """cuSPARSE SpGEMM on the same GPU, each algorithm (ALG2/ALG3 with chunk
    fraction 0.01 as the reference's driver) with its own warm-up and median:
    a reported reference point, not a gate."""
    from rtspmspm_b200 import _lib

    res = {}
    for name, code in CUSPARSE_ALGS:
        o = eng.opts(algo="cusparse", skip_validation=True, cusparse_alg=code)
        try:
            for _ in range(warmup):
                c = _lib.SpgCsr()
                eng.multiply_raw(sa, sa, o, c, _lib.SpgReport())
                eng.free_raw(c)

            def step():
                c = _lib.SpgCsr()
                eng.multiply_raw(sa, sa, o, c, _lib.SpgReport())
                eng.free_raw(c)

            ms = timed_median(step, steps, flush, stream)
            res[name] = {"ms": round(ms, 3), "gflops": round(2 * products / ms / 1e6, 3)}
        except Exception as ex:  # an algorithm can run out of memory on large products
            res[name] = {"error": str(ex)[:160]}
    ok = {k: v for k, v in res.items() if "ms" in v}
    if ok:
        res["fastest"] = min(ok, key=lambda k: ok[k]["ms"])
    res["timing"] = f"median of {steps} after {warmup} warm-up calls, each algorithm"
    return res


def measure_batch(eng, pairs, warmup, steps, flush, stream, tune=True, modes=None):
    """Batched uneven products: median ms per call of spg_multiply_batched
    (graph replay and plain stream launches; tuned and default settings)."""
    from rtspmspm_b200 import DeviceCsr, gen

    dA = [DeviceCsr.from_host(a) for a, _ in pairs]
    dB = [DeviceCsr.from_host(b) for _, b in pairs]
    products = sum(int(gen.row_products(a, b).sum()) for a, b in pairs)
    out = {"products": int(products), "count": len(pairs), "rows": int(sum(a.rows for a, _ in pairs))}
    if tune:
        t = time.perf_counter()
        eng.tune(dA[:min(64, len(dA))], dB[:min(64, len(dB))], None)
        out["tune_s"] = round(time.perf_counter() - t, 2)
        out["tuning"] = eng.get_tuning()
    for graph, tuned, algo in modes or ((True, True, "plain"), (False, True, "plain"), (True, False, "plain"),
                                        (True, False, "learned")):
        if tuned and not tune:
            continue
        for _ in range(warmup):
            eng.multiply_batched(dA, dB, use_graph=graph, use_tuning=tuned, skip_validation=True, algo=algo)
        holder = {}

        def step():
            res, rep = eng.multiply_batched(dA, dB, use_graph=graph, use_tuning=tuned, skip_validation=True,
                                            algo=algo)
            holder["rep"] = rep

        ms = timed_median(step, steps, flush, stream)
        key = ("graph" if graph else "stream") + ("_tuned" if tuned else "_default") + \
            ("_learned" if algo == "learned" else "")
        rep = holder["rep"]
        out[key] = {"ms": round(ms, 3), "gflops": round(2 * products / ms / 1e6, 2), "nnz_c": rep["nnz_c"],
                    "kernel_launches": rep["kernel_launches"], "rows_predicted": rep.get("rows_predicted", 0),
                    "rows_overflow": rep.get("rows_overflow", 0), "products_individual": rep.get("rows_heavy", 0)}
    del dA, dB
    return out


def other_workload(args) -> int:
    """Per-method timings for the other configurations (1 GPU):
    rmat20 = C=A*A on R-MAT scale 20 (a=.57, b=c=.19, edge factor 16, seed 0);
    er4096 = C=A*A on the 4,096^2 Erdos-Renyi Poisson(8) matrix (seed 0);
    batch512 = 512 independent uneven products (seed 1) replayed from a CUDA
    graph; coo = COO -> CSR on the GPU of 2^26 random entries."""
    import torch

    from rtspmspm_b200 import DeviceCsr, Engine, gen

    eng = Engine(0, use_torch_stream=True)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {"workload": args.workload, "steps": args.steps, "warmup": args.warmup}
    if args.workload == "coo":
        # COO -> CSR on the GPU: 2^26 random entries over 2^22 x 2^22, device-resident
        n, dim = 1 << 26, 1 << 22
        g = torch.Generator(device="cuda").manual_seed(3)
        r = torch.randint(0, dim, (n,), device="cuda", dtype=torch.int32, generator=g)
        c = torch.randint(0, dim, (n,), device="cuda", dtype=torch.int32, generator=g)
        v = torch.rand(n, device="cuda", generator=g)
        holder = {}

        def step():
            C = eng.coo_to_csr(dim, dim, r, c, v)
            holder["nnz"] = C.nnz
            C.free()

        for _ in range(args.warmup):
            step()
        ms = timed_median(step, args.steps, flush, stream)
        out.update({"entries": n, "nnz_c": holder["nnz"], "ms": round(ms, 3),
                    "entries_per_s": round(n / (ms * 1e-3), 1)})
        print(json.dumps(out), flush=True)
        eng.close()
        return 0
    # --profile: one method only, default settings (short runs under ncu)
    only = [args.profile] if args.profile else ["plain", "learned"]
    if args.workload == "batch512":
        modes = [(True, False, m) for m in only] if args.profile else None
        out.update(measure_batch(eng, gen.batch_uneven(count=args.batch_count, seed=1), args.warmup, args.steps,
                                 flush, stream, tune=not args.profile, modes=modes))
    else:
        A = gen.rmat(args.rmat_scale, 16, seed=0) if args.workload == "rmat20" else gen.erdos_renyi(4096, 4096, 8.0, 0)
        out.update(measure_single(eng, A, only, args.warmup, args.steps, flush, stream))
        if args.workload == "er4096" and not args.profile:
            dA = DeviceCsr.from_host(A)
            out["cusparse"] = measure_cusparse(eng, dA.struct(), out["products"], args.warmup, args.steps, flush,
                                               stream)
        if args.workload == "rmat20" and not args.no_cpu and not args.profile:
            v, info = cpu_sample(A, args.cpu_seconds)
            out["cpu_baseline"] = {"value": round(v, 4), "unit": "GFLOP/s", "cores": info["cores"], "kind": "port",
                                   "sample": sample_text(info, "the same C=A*A")}
    print(json.dumps(out), flush=True)
    eng.close()
    return 0


def extra_workloads(args, eng, flush, stream) -> dict:
    """The other configurations, measured in the same run as the headline so
    that its line records them (1 GPU only): R-MAT scale 20 and ER 4096
    (plain vs learned), and the 512 uneven products (graph replay)."""
    from rtspmspm_b200 import gen

    out = {}
    t = time.perf_counter()
    E = gen.erdos_renyi(4096, 4096, 8.0, 0)
    out["er4096"] = measure_single(eng, E, ["plain", "learned"], 3, 20, flush, stream)
    # the same product through the binned pipeline (small-product path off)
    saved = eng.get_tuning()
    eng.set_tuning(small_rows=-1)
    out["er4096"]["binned"] = measure_single(eng, E, ["plain", "learned"], 3, 20, flush, stream, use_tuning=True)
    eng.set_tuning(**saved)
    del E
    pairs = gen.batch_uneven(count=512, seed=1)
    out["batch512"] = measure_batch(eng, pairs, 3, max(3, min(args.steps, 10)), flush, stream,
                                    modes=((True, True, "plain"), (True, False, "plain"), (True, False, "learned")))
    b = out["batch512"]
    if "graph_default" in b and "graph_default_learned" in b:
        b["speedup_learned_vs_plain"] = round(b["graph_default"]["ms"] / b["graph_default_learned"]["ms"], 4)
    del pairs
    A = gen.rmat(20, 16, seed=0)
    out["rmat20"] = measure_single(eng, A, ["plain", "learned"], 1, 3, flush, stream)
    out["wall_s"] = round(time.perf_counter() - t, 1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=96)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the R-MAT-20 / ER-4096 / batch-512 timings that ride on the headline line")
    ap.add_argument("--profile", choices=["plain", "learned"], default=None,
                    help="only W warm-up + K steps of one method (short runs under ncu)")
    ap.add_argument("--workload", choices=["stencil96", "rmat20", "er4096", "batch512", "coo"], default="stencil96",
                    help="other configurations: one JSON line of per-method timings (not the headline)")
    ap.add_argument("--rmat-scale", type=int, default=20, help="scale of --workload rmat20 (smaller for profiling)")
    ap.add_argument("--batch-count", type=int, default=512, help="products of --workload batch512")
    ap.add_argument("--e2e-blocks", type=int, default=8,
                    help="row blocks of the end-to-end call (device-to-host copy overlapped with the product)")
    args = ap.parse_args()
    if args.workload != "stencil96":
        return other_workload(args)
    args.warmup = max(args.warmup, 3)

    from rtspmspm_b200 import gen

    A = gen.stencil27(args.grid, seed=0)
    if args.impl == "reference":
        return reference_arm(args, A)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from rtspmspm_b200 import DeviceCsr, Engine, HostCsr, _lib

    eng = Engine(local, use_torch_stream=True)
    stream = torch.cuda.current_stream()
    dA = DeviceCsr.from_host(A, device=local, index_bits=32)
    products = int(gen.row_products(A, A).sum())
    flops = 2.0 * products
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sa = dA.struct()

    def run_steps(algo: str, k: int, stage_timing=False):
        """k timed steps; returns (ms per step, last report, launches per step)."""
        o = eng.opts(algo=algo, skip_validation=True, stage_timing=stage_timing)
        rep = _lib.SpgReport()
        total = 0.0
        launches = 0
        stages = {}
        for _ in range(k):
            flush.zero_()
            c = _lib.SpgCsr()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.multiply_raw(sa, sa, o, c, rep)
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
            launches += rep.kernel_launches
            for i, nm in enumerate(_lib.STAGES):
                stages[nm] = stages.get(nm, 0.0) + rep.ms_stage[i]
            nnz_c = rep.nnz_c
            eng.free_raw(c)
        return total / k, rep, launches / k, {s: v / k for s, v in stages.items() if v}, nnz_c

    if args.profile:
        run_steps(args.profile, args.warmup)
        ms, rep, _, _, nnz_c = run_steps(args.profile, args.steps)
        if rank == 0:
            print(json.dumps({"profile": args.profile, "grid": args.grid, "ms_per_step": round(ms, 4),
                              "gflops": round(flops / ms / 1e6, 3), "nnz_c": nnz_c}), flush=True)
        eng.close()
        return 0

    # warm-up (also loads the predictor)
    for algo in ("learned", "plain"):
        run_steps(algo, args.warmup)

    with ClockSampler(local) as clk:
        barrier()
        ms_learned, rep_l, launches_l, _, nnz_c = run_steps("learned", args.steps)
        ms_learned = max_over_ranks(ms_learned)
        ms_plain, rep_p, launches_p, _, _ = run_steps("plain", args.steps)
        ms_plain = max_over_ranks(ms_plain)
    clocks = clk.summary()
    # per-stage breakdown (separate, untimed-for-headline runs)
    _, rep_ls, _, stages_l, _ = run_steps("learned", 2, stage_timing=True)
    _, rep_ps, _, stages_p, _ = run_steps("plain", 2, stage_timing=True)

    # cuSPARSE SpGEMM on the same GPU (ALG1, ALG2 and ALG3, the reference
    # driver's choice): a reported reference point
    cus = measure_cusparse(eng, sa, products, 3, 10, flush, stream)

    # value-only recompute (structure of C kept, new values): the cuSPARSE
    # reuse flow of the reference's driver
    reuse = {}
    try:
        c = _lib.SpgCsr()
        eng.multiply_raw(sa, sa, eng.opts(algo="plain", skip_validation=True), c, _lib.SpgReport())
        o_r = eng.opts(algo="plain", skip_validation=True)
        rr = _lib.SpgReport()
        for _ in range(args.warmup):
            eng.multiply_reuse_raw(sa, sa, o_r, c, rr)
        ts = []
        for _ in range(args.steps):
            flush.zero_()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.multiply_reuse_raw(sa, sa, o_r, c, rr)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        eng.free_raw(c)
        ms_r = max_over_ranks(statistics.mean(ts))
        reuse = {"ms": round(ms_r, 4), "gflops": round(flops / ms_r / 1e6, 3)}
    except Exception as ex:  # reported, not gated
        reuse = {"error": str(ex)[:200]}

    # end to end through the public API: pinned host inputs -> C in pinned
    # host memory, the download overlapped with the product in row blocks
    hA = HostCsr(A, index_bits=32, pinned=True)
    sh = hA.struct()
    o_e2e = eng.opts(algo="learned", skip_validation=True)
    h2d = hA.nnz * 8 + (A.rows + 1) * 4  # A = B: one upload
    host_c = [torch.empty(A.rows + 1, dtype=torch.int32, pin_memory=True),
              torch.empty(nnz_c, dtype=torch.int32, pin_memory=True),
              torch.empty(nnz_c, dtype=torch.float32, pin_memory=True)]
    hc = eng._host_out(host_c[0], host_c[1], host_c[2], 32)
    e2e_ms = []
    for i in range(2 + args.steps):
        rep = _lib.SpgReport()
        hc.nnz = 0
        flush.zero_()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.multiply_into_host_raw(sh, sh, hc, args.e2e_blocks, o_e2e, rep)
        e1.record(stream)
        e1.synchronize()
        if i >= 2:
            e2e_ms.append(e0.elapsed_time(e1))
    d2h = (A.rows + 1) * 4 + int(hc.nnz) * 8
    e2e_ms_step = max_over_ranks(statistics.mean(e2e_ms))

    # roofline of the dominant kernel (numeric stage of the learned path)
    bytes_alg = csr_bytes(A.rows, A.nnz) * 2 + csr_bytes(A.rows, nnz_c)
    t_num = stages_l.get("numeric", 0.0)
    peak, peak_kind = load_peaks()
    achieved = bytes_alg / (t_num * 1e-3) / 1e9 if t_num else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                "traffic": traffic_from_profiles("k_num_warp_learned"),
                "kernel": "numeric stage (k_num_warp_learned)", "peak_kind": peak_kind,
                "algorithmic_bytes": int(bytes_alg), "kernel_ms": round(t_num, 4),
                "whole_call_frac": round(bytes_alg / (ms_learned * 1e-3) / 1e9 / peak, 4)}

    cpu = None
    cpu_scipy = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, info = cpu_sample(A, args.cpu_seconds)
        cpu = {"value": round(v, 4), "unit": "GFLOP/s", "cores": info["cores"], "kind": "port",
               "sample": sample_text(info, "the same C=A*A")}
        mid = A.rows // 2
        parity = parity_sample(A, host_c[0].numpy(), host_c[1].numpy(), host_c[2].numpy(), mid,
                               min(A.rows, mid + 4096))
        sc = scipy_sample(A, 5.0)
        if sc is not None:
            cpu_scipy = {"value": round(sc[0], 4), "unit": "GFLOP/s", "threads": 1,
                         "sample": f"scipy.sparse A[:{sc[1]}] @ A ({sc[2]:.1f} s)"}

    # the other configurations, so that this line records them (1 GPU)
    extra = None
    if world == 1 and not args.no_extra:
        extra = extra_workloads(args, eng, flush, stream)

    value = world * flops / (ms_learned * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_learned, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(A, products, nnz_c, world),
        "plain": {"ms": round(ms_plain, 4), "gflops": round(world * flops / (ms_plain * 1e-3) / 1e9, 3),
                  "stages_ms": {k: round(v, 4) for k, v in stages_p.items()}},
        "learned": {"ms": round(ms_learned, 4), "stages_ms": {k: round(v, 4) for k, v in stages_l.items()},
                    "rows_predicted": rep_ls.rows_predicted, "rows_overflow": rep_ls.rows_overflow,
                    "misprediction_rate": round(rep_ls.rows_overflow / max(1, rep_ls.rows_predicted), 6)},
        "speedup_learned_vs_plain": round(ms_plain / ms_learned, 4),
        "cusparse": cus,
        "reuse": reuse,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "cpu_scipy": cpu_scipy,
        "parity_sample": parity,
        "e2e": {"value": round(world * flops / (e2e_ms_step * 1e-3) / 1e9, 3), "unit": "GFLOP/s",
                "ms_per_step": round(e2e_ms_step, 4), "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "call": f"spg_multiply_into_host, {args.e2e_blocks} row blocks"},
        "gpu_launches": int(round(launches_l * args.steps)),
        "clocks": clocks,
        "other_workloads": extra,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
