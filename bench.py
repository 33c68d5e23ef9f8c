#!/usr/bin/env python
"""Benchmark of the B200 exact linear-algebra path (one JSON line on stdout).

Workload (one "step"): dense gemm over Z/65521 (Modular<uint32>) at
8192 x 8192 x 8192, C <- A*B + C, entries uniform in [0, p), seeded
synthetic inputs already resident in HBM (3 x 256 MiB, larger than L2, so no
flush is needed between steps).  Metric: Z/p operations per second
(2*M*N*K per step), reported in Gop/s; results are bit-exact (the GPU tests
check them against the CPU oracle).

Also reported on the same line:
  e2e           the same metric through the host-pointer C ABI
                (lela_cuda_gemm_zp_u32) with pinned host buffers: every step
                copies A, B, C to the device and C back;
  plain_gpu     the CUDA-core delayed-reduction gemm on the same GPU;
  roofline      the tensor-core kernel's int8 tensor throughput against the
                int8 peak measured in this run (cuBLASLt int8 gemm);
  cpu_baseline  LELA's own CPU gemm (oracle/_ref) on a bounded row slice,
                all host threads.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one process per GPU) every rank runs an independent
replica of the workload ("replicas only": a single gemm is not sharded) and
value = total operations of all ranks / the slowest rank's time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Z/p gemm Gop/s at 8192^3 (Modular<uint32>, p=65521), bit-exact"
P = 65521
N = 8192


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fl", action="store_true")
    ap.add_argument("--fl-only", action="store_true",
                    help="run only the Faugere-Lachartre line (profiling aid)")
    ap.add_argument("--fl-m", type=int, default=20000)
    ap.add_argument("--fl-count", type=int, default=3)
    ap.add_argument("--no-gf2", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-fl", type=int, default=12)
    ap.add_argument("--batch-dense", type=int, default=48)
    ap.add_argument("--gf2-n", type=int, default=16384)
    ap.add_argument("--gf2-ech-n", type=int, default=32768)
    ap.add_argument("--gf2-ech-rank", type=int, default=30000)
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = []
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(self.device):
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        load = [r for r in rows if r["power"] > 300] or rows
        return {"sm_mhz": statistics.median(r["sm"] for r in load),
                "sm_max_mhz": max(r["smax"] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows), "samples_under_load": len(load)}


# --------------------------------------------------------------- helpers
def max_over_ranks(torch, value, dev, world):
    """The slowest rank's time: MAX all-reduce over the process group (NCCL
    on GPUs; gloo in the CPU tests), identity on one rank."""
    if world <= 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_gops(world, ops_per_step, steps, ms_max):
    """Whole-job throughput: every rank runs `steps` replicas of the step;
    total operations over the slowest rank's time."""
    return world * ops_per_step * steps / (ms_max / 1e3) / 1e9


def int8_peak_tops(torch, dev):
    """Dense int8 tensor-core peak measured here: cuBLASLt int8 gemm
    (torch._int_mm) at 8192^3, best of 5, CUDA events."""
    try:
        a = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device=dev)
        b = torch.randint(-128, 127, (8192, 8192), dtype=torch.int8, device=dev).t()
        for _ in range(3):
            torch._int_mm(a, b)
        best = None
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        del a, b
        return 2 * 8192 ** 3 / best / 1e12, "cuBLASLt int8 gemm 8192^3 (torch._int_mm), best of 5"
    except Exception as ex:  # fall back to twice the measured dense bf16 peak
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
            return 2 * peaks["bf16_tflops"], "2 x measured bf16 dense (int8 gemm unavailable: %s)" % ex
        except Exception:
            return 2 * 1590.0, "2 x fallback bf16 1.59 PFLOP/s"


def cpu_baseline(n, threads):
    """LELA's own CPU gemm on a bounded sample: rows 0..r-1 of the n^3
    workload, ZpModule gemm row-sliced over all host threads."""
    import oracle
    from lela_b200 import gen
    rows = max(64, 8 * threads)
    A = gen.dense_zp(101, rows, n, P)
    B = gen.dense_zp(102, n, n, P)
    C = gen.dense_zp(103, rows, n, P)
    if oracle.have_ref():
        fn, kind = (lambda: oracle.ref_gemm_zp(P, A, B, C, 1, 1, threads=threads)), "reference"
    else:
        fn, kind = (lambda: oracle.gemm_zp(P, A, B, C, 1, 1, threads=threads)), "port"
    t0 = time.perf_counter()
    fn()
    t = time.perf_counter() - t0
    return {"value": round(2 * rows * n * n / t / 1e9, 4), "unit": "Gop/s", "cores": threads,
            "kind": kind,
            "sample": "rows 0-%d of the %d^3 gemm (%dx%dx%d), LELA ZpModule gemm row-sliced over %d threads, %.1f s"
                      % (rows - 1, n, rows, n, n, threads, t)}


# ----------------------------------------------------- Faugere-Lachartre
FL_DENSITY = 0.025


def run_fl(args, cm, stream, torch, dev, rank):
    """FaugereLachartre::echelonize (reduced) on F4-shaped matrices over
    Z/65521: m rows, n = 1.2 m columns, 75% pivot rows, row density 2.5%,
    5% of the non-pivot rows dependent.  The CSR input and the dense output
    stay on the device; each matrix is timed with CUDA events on the
    module's stream (host orchestration between kernels included).  Also
    timed: the plain per-matrix pipeline (same algorithm with every gemm on
    the CUDA-core kernel)."""
    import types
    from lela_b200 import gen
    m = args.fl_m
    res = {"workload": "FL reduced echelon form, F4-shaped, p=65521, m=%d, n=%d, density %.3f, %d matrices"
                       % (m, int(1.2 * m), FL_DENSITY, args.fl_count),
           "unit": "ms/matrix"}
    mats = []
    for s in range(args.fl_count):
        X = gen.f4_matrix(1000 + 17 * rank + s, m, P, density=FL_DENSITY)
        T = types.SimpleNamespace(
            m=X.m, n=X.n, nnz=X.nnz,
            rowptr=torch.from_numpy(X.rowptr.view(np.int64)).to(dev),
            colidx=torch.from_numpy(X.colidx.view(np.int32)).to(dev),
            vals=torch.from_numpy(X.vals.view(np.int32)).to(dev))
        mats.append(T)
    R = torch.empty((m, int(1.2 * m)), dtype=torch.int32, device=dev)

    def timed(T):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, rk, det = cm.fl_echelonize(P, T, True, False, R=R)
        e1.record(stream)
        cm.synchronize()
        return e0.elapsed_time(e1), rk, det

    cm.fl_echelonize(P, mats[0], True, False, R=R)  # warm-up
    cm.synchronize()
    times, ranks = [], []
    for T in mats:
        t, rk, _ = timed(T)
        times.append(t)
        ranks.append(rk)
    # phase breakdown from one more, untimed run with per-launch events on
    # (the events themselves cost host time, so the timed runs go without)
    cm.profile_reset()
    cm.profile(True)
    timed(mats[0])
    phases = {k.replace("fl_phase_", ""): round(cm.profile_read(k)[0], 2)
              for k in ("fl_phase_trsm", "fl_phase_schur", "fl_phase_echelon", "fl_phase_reduce")}
    cm.profile(False)
    res.update({"ms_per_matrix": round(sum(times) / len(times), 2), "ms_each": [round(t, 2) for t in times],
                "ranks": ranks, "phase_ms": phases, "nnz": [T.nnz for T in mats]})
    if not args.no_plain:
        cm.set_gemm_kernel(1)
        t, rk, _ = timed(mats[0])
        cm.set_gemm_kernel(0)
        res["plain_ms_per_matrix"] = round(t, 2)
        res["speedup_vs_plain"] = round(t / times[0], 2)
    del R
    return res


def run_gf2(args, cm, stream, torch, dev):
    """GF(2) workloads: packed gemm 16384^3 with Bernoulli(1/2) bits on both
    kernels (int8-expanded tensor cores, bit-packed four-Russians), and the
    echelon form of a 32768 x 32768 matrix of planted rank 30000 (product of
    random 32768 x 30000 and 30000 x 32768 factors, formed on the device with
    the GF(2) gemm).  Inputs resident in HBM."""
    n = args.gf2_n
    w = n // 64
    res = {"gemm_workload": "GF(2) gemm %d^3, Bernoulli(1/2), packed words" % n, "unit": "ms"}
    g = torch.Generator(device=dev)
    g.manual_seed(7)

    def rnd(rows, cols_words):
        return torch.randint(-2 ** 63, 2 ** 63 - 1, (rows, cols_words), dtype=torch.int64,
                             device=dev, generator=g)

    A, B, C = rnd(n, w), rnd(n, w), torch.zeros((n, w), dtype=torch.int64, device=dev)
    for kernel, name in ((1, "tc"), (2, "m4rm")):
        cm.set_gf2_kernel(kernel)
        cm.gemm_gf2(A, B, C, n, n, 1, 0)
        cm.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record(stream)
        for _ in range(reps):
            cm.gemm_gf2(A, B, C, n, n, 1, 0)
        e1.record(stream)
        cm.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res["gemm_%s_ms" % name] = round(ms, 3)
        res["gemm_%s_Tbitop_s" % name] = round(2.0 * n ** 3 / (ms / 1e3) / 1e12, 1)
    cm.set_gf2_kernel(0)
    del A, B, C
    # planted-rank echelon
    m, r = args.gf2_ech_n, args.gf2_ech_rank
    mw, rw = m // 64, (r + 63) // 64
    F1 = rnd(m, rw)
    if r % 64:
        F1[:, -1] &= (1 << (r % 64)) - 1
    F2 = rnd(r, mw)
    D = torch.zeros((m, mw), dtype=torch.int64, device=dev)
    cm.gemm_gf2(F1, F2, D, m, r, 1, 0)
    del F1, F2
    cm.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _, rank = cm.echelonize_gf2(D, m)
    e1.record(stream)
    cm.synchronize()
    res.update({"echelon_workload": "GF(2) echelon %d x %d, planted rank %d" % (m, m, r),
                "echelon_ms": round(e0.elapsed_time(e1), 2), "echelon_rank": rank})
    del D
    return res


def run_batch(args, cm, stream, torch, dev):
    """Batched workload (scaled to minutes): F4-shaped FL matrices with m
    log-uniform in [2000, 8000] plus dense Z/p echelon blocks of sizes
    log-uniform in [64, 4096], p in {251, 65521, 2^31-1}.
    * ours: the FL matrices through the batched entry point (8 worker
      streams, tensor-core gemms) and the dense blocks through one batched
      call whose kernel per block is chosen by the MLP cost model, trained
      first on autotuner timings of a separate set of blocks (small blocks in
      one persistent graph launch, the others over worker streams);
    * plain: the per-matrix pipeline -- one matrix per call, one at a time on
      one stream, with every gemm on the CUDA-core kernel and every dense
      block through the panel pipeline."""
    import types
    from lela_b200 import gen
    from lela_b200 import selector as sel
    rng = np.random.default_rng(11)
    primes = [251, 65521, 2147483647]
    fl_items = []
    for i in range(args.batch_fl):
        m = int(2 ** rng.uniform(math.log2(2000), math.log2(8000)))
        X = gen.f4_matrix(3000 + i, m, P, density=FL_DENSITY)
        fl_items.append(types.SimpleNamespace(
            m=X.m, n=X.n, rowptr=torch.from_numpy(X.rowptr.view(np.int64)).to(dev),
            colidx=torch.from_numpy(X.colidx.view(np.int32)).to(dev),
            vals=torch.from_numpy(X.vals.view(np.int32)).to(dev)))
    dense = []
    for i in range(args.batch_dense):
        s = int(2 ** rng.uniform(6, 12))
        p = int(rng.choice(primes))
        dense.append((torch.from_numpy(gen.dense_zp(4000 + i, s, s, p).view(np.int32)).to(dev), p))
    Rs = [torch.empty((X.m, X.n), dtype=torch.int32, device=dev) for X in fl_items]
    work = [torch.empty_like(A) for A, _ in dense]

    # cost model from autotuner timings on separate blocks
    t0 = time.perf_counter()
    tuner = sel.Autotuner(cm, reps=2)
    for i in range(24):
        s = int(2 ** rng.uniform(6, 12))
        tuner.tune_echelon(s, s, int(rng.choice(primes)), seed=9000 + i)
    X, y = sel.records_to_xy(tuner.records)
    model = sel.CostModel(cm, seed=1)
    model.fit(X, y, epochs=600)
    choose = sel.Selector(model)
    kernels = [choose.choose("echelon", A.shape[0], A.shape[1], 0, 1.0, p.bit_length(), A.shape[0])
               for A, p in dense]
    tune_s = time.perf_counter() - t0

    # the dense blocks go through a second handle from a second host thread,
    # concurrently with the FL batch (a handle serves one thread at a time)
    from lela_b200 import CudaModule
    cm_dense = CudaModule(torch.cuda.current_device())

    def ours():
        for w, (A, _) in zip(work, dense):
            w.copy_(A)
        torch.cuda.synchronize()  # the copies are done before another stream reads them
        failed = []

        def dense_part():
            try:
                cm_dense.echelonize_batch(work, [p for _, p in dense], kernels)
            except BaseException as e:  # re-raised on the calling thread
                failed.append(e)

        th = threading.Thread(target=dense_part)
        th.start()
        try:
            cm.fl_echelonize_batch(fl_items, [P] * len(fl_items), Rs, True, nworkers=8)
        finally:
            th.join()
        if failed:
            raise failed[0]

    def plain():
        for w, (A, _) in zip(work, dense):
            w.copy_(A)
        cm.set_gemm_kernel(1)
        try:
            for X, R in zip(fl_items, Rs):
                cm.fl_echelonize(P, X, True, False, R=R)
            for w, (_, p) in zip(work, dense):
                cm.echelonize_batch([w], [p], [3])
        finally:
            cm.set_gemm_kernel(0)

    def timed(fn):
        torch.cuda.synchronize()
        cm.synchronize()
        t = time.perf_counter()
        fn()
        cm.synchronize()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3

    ours()
    t_ours = min(timed(ours) for _ in range(4))
    plain()
    t_plain = timed(plain)
    return {"workload": "%d F4 matrices (m log-uniform 2000-8000, p=65521) + %d dense echelon blocks "
                        "(64-4096, p in {251, 65521, 2^31-1})" % (len(fl_items), len(dense)),
            "unit": "ms/batch", "ms": round(t_ours, 1), "plain_ms": round(t_plain, 1),
            "speedup_vs_plain": round(t_plain / t_ours, 2),
            "selector": {"kernels": {str(k): kernels.count(k) for k in sorted(set(kernels))},
                         "tuning_and_training_s": round(tune_s, 1),
                         "names": {str(k): sel.KERNEL_NAMES[("echelon", k)] for k in (1, 2, 3)}},
            "timing": "host wall clock around the synchronised batch (includes host orchestration)"}


def fl_cpu_baseline(m_target):
    """LELA's own FaugereLachartre (oracle/_ref) on the same matrix family at
    m = 1000 and 2000, single-threaded (LELA has no threading), fitted as
    c*m^3 and extrapolated; labelled as such."""
    import oracle
    from lela_b200 import gen
    if not oracle.have_ref():
        return {"unavailable": "oracle/_ref not built"}
    pts = []
    for m in (1000, 2000):
        X = gen.f4_matrix(500 + m, m, P, density=FL_DENSITY)
        t0 = time.perf_counter()
        oracle.ref_fl_echelonize_zp(P, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
        pts.append((m, time.perf_counter() - t0))
    c = pts[-1][1] / pts[-1][0] ** 3
    return {"kind": "reference", "cores": 1, "measured_s": {str(m): round(t, 3) for m, t in pts},
            "extrapolated_ms_per_matrix": round(c * m_target ** 3 * 1e3, 1),
            "extrapolation": "c*m^3 with c from the m=2000 run, at m=%d" % m_target}


# ------------------------------------------------------------ reference
def run_reference(args):
    """LELA's own CPU gemm (oracle/_ref; the C restatement if LELA was not
    built) on the bench's workload, all host threads, each step a row slice
    of the 8192^3 gemm sized so that warm-up + steps take about two minutes."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from lela_b200 import gen
    threads = os.cpu_count() or 1
    n = args.n
    B = gen.dense_zp(102, n, n, P)
    kind = "reference" if oracle.have_ref() else "port"

    def run(rows):
        A = gen.dense_zp(101, rows, n, P)
        C = gen.dense_zp(103, rows, n, P)
        t0 = time.perf_counter()
        if kind == "reference":
            oracle.ref_gemm_zp(P, A, B, C, 1, 1, threads=threads)
        else:
            oracle.gemm_zp(P, A, B, C, 1, 1, threads=threads)
        return time.perf_counter() - t0

    t1 = run(threads)  # calibration: one row per thread
    budget = 120.0 / max(1, args.steps + args.warmup)
    rows = threads * max(1, int(budget / max(t1, 1e-3)))
    for _ in range(args.warmup):
        run(rows)
    tot = 0.0
    for _ in range(args.steps):
        tot += run(rows)
    t = tot / args.steps
    v = 2 * rows * n * n / t / 1e9
    line = {"metric": METRIC, "value": round(v, 4), "unit": "Gop/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 (u64 accumulate)", "data": "synthetic",
            "config": {"workload": "gemm Z/65521 %d^3 C<-A*B+C" % n, "p": P, "m": n, "n": n, "k": n,
                       "parallelism": "host threads (row slices)"},
            "cpu_baseline": {"value": round(v, 4), "unit": "Gop/s", "cores": threads, "kind": kind,
                             "sample": "rows 0-%d of the %d^3 gemm per step (LELA ZpModule gemm, row-sliced)"
                                       % (rows - 1, n)},
            "e2e": {"value": round(v, 4), "unit": "Gop/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours
def run_ours(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    from lela_b200 import gen, CudaModule

    n = args.n
    cm = CudaModule(local)
    stream = torch.cuda.Stream(device=dev)
    cm.set_stream(stream)

    A = gen.dense_zp(11 + rank, n, n, P)
    B = gen.dense_zp(12 + rank, n, n, P)
    C = gen.dense_zp(13 + rank, n, n, P)
    dA = torch.from_numpy(A.view(np.int32)).to(dev)
    dB = torch.from_numpy(B.view(np.int32)).to(dev)
    dC = torch.from_numpy(C.view(np.int32)).to(dev)
    torch.cuda.synchronize()

    peak, peak_src = int8_peak_tops(torch, dev)

    def step():
        cm.gemm(P, 1, dA, dB, 1, dC)

    for _ in range(max(args.warmup, 3)):
        step()
    cm.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    cm.profile_reset()
    cm.profile(True)
    launches0 = cm.launch_count
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    cm.synchronize()
    torch.cuda.synchronize()
    launches = cm.launch_count - launches0
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    tc_ms, tc_n = cm.profile_read("zp_gemm_tc")
    sp_ms, sp_n = cm.profile_read("zp_split")
    cm.profile(False)

    ms_max = max_over_ranks(torch, ms, dev, world)
    ops_step = 2.0 * n ** 3
    value = whole_job_gops(world, ops_step, args.steps, ms_max)

    # dominant kernel roofline: int8 tensor ops actually required
    L = 2
    tc_avg = tc_ms / max(tc_n, 1)
    achieved = L * L * 2.0 * n ** 3 / (tc_avg / 1e3) / 1e12
    roofline = {"bound": "tensor", "kernel": "zp_gemm_tc_kernel<2>", "achieved": round(achieved, 1),
                "peak": round(peak, 1), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                "traffic": None,
                "ops_per_launch": "4 limb products x 2*8192^3 int8 multiply-adds = %.3e" % (L * L * 2.0 * n ** 3),
                "kernel_ms_avg": round(tc_avg, 4), "split_ms_avg": round(sp_ms / max(sp_n, 1), 4),
                "peak_source": peak_src + " (measured in this run)"}

    out = {"metric": METRIC, "value": round(value, 2), "unit": "Gop/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "u32 (u8 limbs, s32 tensor accumulate)", "data": "synthetic",
           "config": {"workload": "gemm Z/65521 %d^3 C<-A*B+C" % n, "p": P, "m": n, "n": n, "k": n,
                      "limbs": L, "parallelism": "replicas" if world > 1 else "single GPU",
                      "l2": "inputs 3 x %d MiB > L2 (no flush)" % (n * n * 4 >> 20)},
           "roofline": roofline, "clocks": clk, "gpu_launches": int(launches)}

    # plain CUDA-core gemm on the same GPU (the "plain GPU form")
    if not args.no_plain:
        cm.set_gemm_kernel(1)
        cm.gemm(P, 1, dA, dB, 1, dC)
        cm.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        reps = 2
        for _ in range(reps):
            cm.gemm(P, 1, dA, dB, 1, dC)
        f1.record(stream)
        cm.synchronize()
        pms = f0.elapsed_time(f1) / reps
        cm.set_gemm_kernel(0)
        out["plain_gpu"] = {"value": round(ops_step / (pms / 1e3) / 1e9, 2), "unit": "Gop/s",
                            "ms_per_step": round(pms, 3), "kernel": "zp_gemm_plain_kernel"}
        out["speedup_vs_plain"] = round(out["value"] / world / out["plain_gpu"]["value"], 2)

    del dA, dB, dC
    torch.cuda.empty_cache()

    # end to end through the host-pointer C ABI, pinned host buffers
    if not args.no_e2e:
        pin = lambda x: torch.from_numpy(x.view(np.int32)).pin_memory().numpy().view(np.uint32)
        hA, hB, hC = pin(A), pin(B), pin(C)
        cm.gemm(P, 1, hA, hB, 1, hC)
        steps = max(1, min(args.steps, 5))
        if world > 1:
            torch.distributed.barrier()
        t0 = time.perf_counter()
        for _ in range(steps):
            cm.gemm(P, 1, hA, hB, 1, hC)
        te = max_over_ranks(torch, (time.perf_counter() - t0) / steps, dev, world)
        out["e2e"] = {"value": round(world * ops_step / te / 1e9, 2), "unit": "Gop/s",
                      "h2d_bytes_per_step": 3 * n * n * 4, "d2h_bytes_per_step": n * n * 4,
                      "ms_per_step": round(te * 1e3, 3),
                      "api": "lela_cuda_gemm_zp_u32 (host pointers, pinned)"}

    if not args.no_fl:
        out["fl"] = run_fl(args, cm, stream, torch, dev, rank)
    if not args.no_gf2:
        out["gf2"] = run_gf2(args, cm, stream, torch, dev)
    if not args.no_batch:
        out["batch"] = run_batch(args, cm, stream, torch, dev)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(n, os.cpu_count() or 1)
        if not args.no_fl:
            out["fl"]["cpu_lela"] = fl_cpu_baseline(args.fl_m)

    cm.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_fl_only(args):
    """Only the Faugere-Lachartre line (for kernel launch lists and
    profiles): one process, one GPU; prints its JSON object."""
    import torch
    from lela_b200 import CudaModule
    dev = torch.device("cuda", 0)
    cm = CudaModule(0)
    stream = torch.cuda.Stream(device=dev)
    cm.set_stream(stream)
    print(json.dumps(run_fl(args, cm, stream, torch, dev, 0)))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.fl_only:
        run_fl_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
