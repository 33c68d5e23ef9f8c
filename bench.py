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
# DRAM bytes of one launch of the tensor-core gemm at 8192^3, p = 65521 (two
# limbs, wide tiles), from an ncu capture of
# `python bench.py --gemm-only 8192,8192,8192 --steps 3 --warmup 2`:
# dram__bytes_read.sum 1315.0 MB + dram__bytes_write.sum 261.4 MB.
TC_TRAFFIC_8192 = 1315042304 + 261354496
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
    ap.add_argument("--gf2-only", action="store_true",
                    help="run only the GF(2) gemm and echelon line (profiling aid)")
    ap.add_argument("--gemm-only", metavar="M,N,K",
                    help="time only a Z/p gemm of this shape on the tensor cores (profiling aid)")
    ap.add_argument("--echelon-only", type=int, metavar="N", default=0,
                    help="only a dense N x N row-echelon form over Z/65521 (for launch lists)")
    ap.add_argument("--gemm-p", type=int, default=P)
    ap.add_argument("--gemm-tile", type=int, default=0,
                    help="tile variant for --gemm-only: 0 auto, 1 wide, 2 two accumulator buffers")
    ap.add_argument("--fl-m", type=int, default=20000)
    ap.add_argument("--fl-count", type=int, default=3)
    ap.add_argument("--fl-big", type=int, default=120000,
                    help="rows of the one large FL matrix (CSR output; 0 = skip)")
    ap.add_argument("--no-fl-check", action="store_true",
                    help="skip the reduced-echelon certificate of the last timed FL matrix")
    ap.add_argument("--no-dense", action="store_true",
                    help="skip the p = 2^31-1 gemm, trsm and dense echelon lines")
    ap.add_argument("--no-gf2", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-fl", type=int, default=16)
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


class NvmlClockSampler:
    """SM clock, power and clock-event reasons of this process's GPU read
    through NVML every 5 ms from a thread (read-only queries), so that even
    a timed region of a few tens of milliseconds gets samples.  The GPU is
    found by its UUID; raises when NVML or the UUID is unavailable."""

    def __init__(self, torch, dev):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
        self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid.encode() if isinstance(uuid, str) else uuid)
        self.smax = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        self.rows = []
        self.stop_ev = threading.Event()
        self.th = threading.Thread(target=self._run, daemon=True)
        self.th.start()

    def _run(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                self.rows.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                  nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0,
                                  nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except Exception:
                pass
            time.sleep(0.005)

    def stop(self):
        self.stop_ev.set()
        self.th.join(timeout=2)
        nv = self.nv
        names = ((nv.nvmlClocksEventReasonHwSlowdown, "hw_slowdown"),
                 (nv.nvmlClocksEventReasonHwThermalSlowdown, "hw_thermal_slowdown"),
                 (nv.nvmlClocksEventReasonSwThermalSlowdown, "sw_thermal_slowdown"),
                 (nv.nvmlClocksEventReasonSwPowerCap, "sw_power_cap"))
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["unsampled"]}
        reasons = sorted({name for _, _, r in self.rows for bit, name in names if r & bit})
        return {"sm_mhz": statistics.median(s for s, _, _ in self.rows), "sm_max_mhz": self.smax,
                "reasons": reasons, "samples": len(self.rows),
                "power_w_max": round(max(w for _, w, _ in self.rows), 1), "source": "NVML, 5 ms"}


def clock_sampler(torch, dev, index):
    try:
        return NvmlClockSampler(torch, dev)
    except Exception:
        return ClockSampler(index)


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


def _hbm_peak():
    """HBM copy bandwidth measured on this pool (MEASURED_PEAKS.json), else
    the stated fallback."""
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent)"


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class CpuGemmSampler:
    """LELA's own CPU gemm (oracle/_ref, else the C restatement) on row
    slices of the n^3 workload: rows 0..r-1 of A and C against all of B,
    row-sliced over `threads` host threads (row slices are independent, so
    the result equals a single call's).  Shared by the cpu_baseline leg and
    the reference arm, so both sample the same way."""

    def __init__(self, n, threads):
        import oracle
        from lela_b200 import gen
        self.oracle, self.gen, self.n, self.threads = oracle, gen, n, threads
        self.B = gen.dense_zp(102, n, n, P)
        self.kind = "reference" if oracle.have_ref() else "port"

    def run(self, rows):
        A = self.gen.dense_zp(101, rows, self.n, P)
        C = self.gen.dense_zp(103, rows, self.n, P)
        t0 = time.perf_counter()
        if self.kind == "reference":
            self.oracle.ref_gemm_zp(P, A, self.B, C, 1, 1, threads=self.threads)
        else:
            self.oracle.gemm_zp(P, A, self.B, C, 1, 1, threads=self.threads)
        return time.perf_counter() - t0

    def rows_for(self, seconds):
        """Rows (a multiple of the thread count) that take about `seconds`."""
        t1 = self.run(self.threads)  # calibration: one row per thread
        return self.threads * max(1, int(seconds / max(t1, 1e-3)))


def cpu_baseline(n, threads):
    """LELA's own CPU gemm on a bounded sample of the n^3 workload (about
    12 s of work), all host threads."""
    s = CpuGemmSampler(n, threads)
    rows = s.rows_for(12.0)
    t = s.run(rows)
    return {"value": round(2 * rows * n * n / t / 1e9, 4), "unit": "Gop/s", "cores": threads,
            "kind": s.kind, "cpu": cpu_model(),
            "sample": "rows 0-%d of the %d^3 gemm (%dx%dx%d), LELA ZpModule gemm row-sliced over %d threads, %.1f s"
                      % (rows - 1, n, rows, n, n, threads, t)}


# ----------------------------------------------------- Faugere-Lachartre
FL_DENSITY = 0.025


def fl_structure(X):
    """Pivot structure of an F4 matrix as FaugereLachartre splits it
    (setup_splicer, faugere-lachartre.tcc:47-146): pivot rows/columns and the
    off-diagonal nonzeros of the pivot block A."""
    heads = X.colidx[X.rowptr[:-1].astype(np.int64)].astype(np.int64)
    piv = np.concatenate([[True], heads[1:] > heads[:-1]])
    is_pc = np.zeros(X.n, dtype=bool)
    is_pc[heads[piv]] = True
    rows = np.repeat(np.arange(X.m), np.diff(X.rowptr).astype(np.int64))
    in_a = piv[rows] & is_pc[X.colidx.astype(np.int64)]
    npiv = int(piv.sum())
    return npiv, int(in_a.sum()) - npiv


def fl_algorithmic_ops(m, n, npiv, nnz_off_a, rank):
    """Z/p operations of one reduced FL echelonization (multiply and add
    counted separately): the sparse triangular solve 2 nnz_off(A) (n - npiv),
    the Schur complement 2 (m - npiv) npiv (n - npiv), the echelon form of D
    (mres x nres, rank r) 2 (mres nres r - (mres + nres) r^2 / 2 + r^3 / 3),
    and the back-substitution r^2 (nres - r) + 2 npiv r (nres - r)."""
    mres, nres, r = m - npiv, n - npiv, rank - npiv
    parts = {"trsm": 2.0 * nnz_off_a * nres, "schur": 2.0 * mres * npiv * nres,
             "echelon": 2.0 * (mres * nres * r - (mres + nres) * r * r / 2.0 + r ** 3 / 3.0),
             "reduce": float(r) * r * (nres - r) + 2.0 * npiv * r * (nres - r)}
    return parts


def run_fl(args, cm, stream, torch, dev, rank, zp_peak=None):
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
        npiv, nnz_off = fl_structure(X)
        T = types.SimpleNamespace(
            m=X.m, n=X.n, nnz=X.nnz, host=X, npiv=npiv, nnz_off=nnz_off,
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
    # roofline of the whole matrix and of its phases: algorithmic Z/p
    # operations over the time, against the two-limb Z/p peak (int8 peak / 4)
    ops = [fl_algorithmic_ops(T.m, T.n, T.npiv, T.nnz_off, rk) for T, rk in zip(mats, ranks)]
    tot = [sum(o.values()) for o in ops]
    res["algorithmic_ops"] = {k: "%.3e" % ops[0][k] for k in ops[0]}
    res["Zp_Top_s"] = round(sum(tot) / (sum(times) / 1e3) / 1e12, 2)
    if zp_peak:
        res["roofline"] = {"bound": "tensor", "peak_Zp_Top_s": round(zp_peak, 1),
                           "frac": round(res["Zp_Top_s"] / zp_peak, 4),
                           "phase_frac": {k: round(ops[0][k] / (phases[k] / 1e3) / 1e12 / zp_peak, 4)
                                          for k in phases if phases[k] > 0},
                           "counting": "fl_algorithmic_ops (trsm counted on the sparse A)"}
    if not args.no_fl_check:
        # R holds the output of the last run, the profiled one of matrix 0
        from lela_b200 import certify
        T = mats[0]
        err = certify.rref_certificate(torch, P, T.host, R[:T.m], ranks[0])
        res["checked"] = err is None
        res["check"] = ("reduced-echelon certificate of matrix 0 (echelon structure exact; "
                        "row space by 2 random projections, error <= p^-2)"
                        + ("" if err is None else ": FAILED " + err))
    if not args.no_plain:
        cm.set_gemm_kernel(1)
        t, rk, _ = timed(mats[0])
        cm.set_gemm_kernel(0)
        res["plain_ms_per_matrix"] = round(t, 2)
        res["speedup_vs_plain"] = round(t / times[0], 2)
    del R
    return res


def _event_ms(torch, stream, fn, reps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_dense(args, cm, stream, torch, dev, int8_peak):
    """The other dense workloads, inputs resident in HBM, CUDA events on the
    module's stream:
    * gemm 8192^3 at p = 2^31 - 1 (four limbs: 16 limb products per output);
    * trsm with the 8192 x 8192 unit-lower L (uniform off-diagonal entries)
      and an 8192 x 4096 right-hand side, at p = 65521 and 2^31 - 1;
    * the row-echelon form of a dense 8192 x 8192 matrix over Z/65521.
    Each with its roofline: algorithmic Z/p operations per second against
    the Z/p peak of its limb count (the int8 peak measured in this run /
    limbs^2)."""
    from lela_b200 import gen
    n = 8192
    out = {}
    p31 = 2147483647
    dA = torch.from_numpy(gen.dense_zp(21, n, n, p31).view(np.int32)).to(dev)
    dB = torch.from_numpy(gen.dense_zp(22, n, n, p31).view(np.int32)).to(dev)
    dC = torch.from_numpy(gen.dense_zp(23, n, n, p31).view(np.int32)).to(dev)
    cm.gemm(p31, 1, dA, dB, 1, dC)
    cm.profile_reset()
    cm.profile(True)
    ms = _event_ms(torch, stream, lambda: cm.gemm(p31, 1, dA, dB, 1, dC), 5)
    tc_ms, tc_n = cm.profile_read("zp_gemm_tc")
    cm.profile(False)
    cm.synchronize()
    kern = tc_ms / max(tc_n, 1)
    zp = 2.0 * n ** 3 / (ms / 1e3) / 1e12
    out["gemm_p31"] = {"workload": "gemm Z/2147483647 8192^3 C<-A*B+C", "ms": round(ms, 3),
                       "Gop_s": round(zp * 1e3, 1), "limbs": 4,
                       "roofline": {"bound": "tensor", "kernel": "zp_gemm_tc_kernel<4>",
                                    "kernel_ms": round(kern, 3),
                                    "achieved_int8_Tops": round(16 * 2.0 * n ** 3 / (kern / 1e3) / 1e12, 1),
                                    "peak_int8_Tops": round(int8_peak, 1),
                                    "frac": round(16 * 2.0 * n ** 3 / (kern / 1e3) / 1e12 / int8_peak, 4)}}
    del dA, dB, dC
    # trsm, both moduli
    out["trsm"] = {}
    for p, L in ((65521, 2), (p31, 4)):
        Lm = torch.from_numpy(gen.unit_lower_zp(31, n, p).view(np.int32)).to(dev)
        B0 = torch.from_numpy(gen.dense_zp(32, n, n // 2, p).view(np.int32)).to(dev)
        B = B0.clone()
        cm.trsm(p, 1, Lm, B, False, True)
        times = []
        for _ in range(3):
            B.copy_(B0)
            times.append(_event_ms(torch, stream, lambda: cm.trsm(p, 1, Lm, B, False, True), 1))
        ms = min(times)
        ops = float(n) * n * (n // 2)
        peak = int8_peak / (L * L)
        out["trsm"][str(p)] = {"workload": "trsm 8192x8192 unit-lower, 8192x4096 RHS, p=%d" % p,
                               "ms": round(ms, 3), "Zp_Top_s": round(ops / (ms / 1e3) / 1e12, 2),
                               "roofline": {"bound": "tensor", "peak_Zp_Top_s": round(peak, 1),
                                            "frac": round(ops / (ms / 1e3) / 1e12 / peak, 4),
                                            "counting": "m^2 n Z/p operations (triangle, multiply and add)"}}
        del Lm, B0, B
    # dense echelon form
    E0 = torch.from_numpy(gen.dense_zp(33, n, n, P).view(np.int32)).to(dev)
    E = E0.clone()
    cm.echelonize(P, E)
    times, rk = [], None
    for _ in range(3):
        E.copy_(E0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, rk, _ = cm.echelonize(P, E)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = min(times)
    r = rk
    ops = 2.0 * (n * n * r - (n + n) * r * r / 2.0 + r ** 3 / 3.0)
    out["echelon"] = {"workload": "row-echelon form, dense 8192x8192 over Z/65521 (LELA pivot rule)",
                      "ms": round(ms, 3), "rank": rk, "Zp_Top_s": round(ops / (ms / 1e3) / 1e12, 2),
                      "roofline": {"bound": "tensor", "peak_Zp_Top_s": round(int8_peak / 4, 1),
                                   "frac": round(ops / (ms / 1e3) / 1e12 / (int8_peak / 4), 4),
                                   "counting": "2 (m n r - (m + n) r^2 / 2 + r^3 / 3)"}}
    del E0, E
    torch.cuda.empty_cache()
    return out


def run_fl_big(args, torch, dev, zp_peak=None):
    """One F4 matrix at the top of the FL family's range (m = args.fl_big,
    n = 1.2 m, density 2.5 %, p = 65521), generated on the device
    (gen.f4_matrix_torch), echelonized (reduced) with the result as CSR rows
    -- no dense m x n array, which would be 69 GB at m = 120000.  A warm-up
    run (device buffers grow to size), then one timed run (CUDA events on
    the handle's stream), then the reduced-echelon certificate of its
    result.  Runs on its own handle, closed afterwards."""
    from lela_b200 import CudaModule, certify, gen
    m = args.fl_big
    res = {"workload": "FL reduced echelon form, CSR output, F4-shaped, p=65521, m=%d, n=%d, density %.3f"
                       % (m, int(1.2 * m), FL_DENSITY), "unit": "ms/matrix"}
    cm = CudaModule(torch.cuda.current_device())
    try:
        stream = torch.cuda.Stream(device=dev)
        cm.set_stream(stream)
        t0 = time.perf_counter()
        X = gen.f4_matrix_torch(7000, m, P, dev, density=FL_DENSITY)
        torch.cuda.synchronize()
        res["generation_s"] = round(time.perf_counter() - t0, 1)
        res["nnz"] = X.nnz
        torch.cuda.empty_cache()
        R, rk, det = cm.fl_echelonize_csr(P, X, True, False)
        cap = int(R.colidx.numel())
        del R
        torch.cuda.empty_cache()
        cm.profile_reset()
        cm.profile(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        R, rk, det = cm.fl_echelonize_csr(P, X, True, False, cap=cap)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        phases = {k.replace("fl_phase_", ""): round(cm.profile_read(k)[0], 1)
                  for k in ("fl_phase_trsm", "fl_phase_schur", "fl_phase_echelon", "fl_phase_reduce")}
        cm.profile(False)
        res.update({"ms": round(ms, 1), "rank": rk, "R_nnz": int(R.colidx.numel()),
                    "phase_ms_profiled": phases,
                    "timing": "CUDA events around one call (after a warm-up call); phases from the same "
                              "call's per-launch events"})
        err = certify.rref_certificate_csr(torch, P, X, R, rk)
        res["checked"] = err is None
        res["check"] = "reduced-echelon certificate (CSR form; 2 random projections)" + \
                       ("" if err is None else ": FAILED " + err)
        del R, X
    except Exception as ex:  # reported in the line, the other workloads still run
        res["error"] = "%s: %s" % (type(ex).__name__, ex)
    finally:
        cm.close()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    return res


def run_gf2(args, cm, stream, torch, dev, int8_peak=None):
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
    if int8_peak:
        # one int8 multiply-add per bit product on the tensor cores; the
        # packed operands and result are 3 n^2 / 8 bytes (HBM fraction of the
        # algorithmic bytes against the copy bandwidth, for reference)
        hbm = _hbm_peak()
        res["roofline"] = {"bound": "tensor", "frac_tc": round(res["gemm_tc_Tbitop_s"] / int8_peak, 4),
                           "peak_int8_Tops": round(int8_peak, 1),
                           "hbm_frac_tc": round(3 * n * n / 8 / (res["gemm_tc_ms"] / 1e3) / 1e9 / hbm[0], 5),
                           "hbm_frac_m4rm": round(3 * n * n / 8 / (res["gemm_m4rm_ms"] / 1e3) / 1e9 / hbm[0], 5),
                           "hbm_peak_GBs": hbm[0], "hbm_peak_source": hbm[1]}
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
    ems = e0.elapsed_time(e1)
    ops = 2.0 * (m * m * rank - (m + m) * rank * rank / 2.0 + rank ** 3 / 3.0)
    res.update({"echelon_workload": "GF(2) echelon %d x %d, planted rank %d" % (m, m, r),
                "echelon_ms": round(ems, 2), "echelon_rank": rank,
                "echelon_Tbitop_s": round(ops / (ems / 1e3) / 1e12, 1)})
    if int8_peak:
        res["echelon_frac_tc"] = round(ops / (ems / 1e3) / 1e12 / int8_peak, 4)
    del D
    return res


def run_batch(args, cm, stream, torch, dev):
    """Batched workload: F4 matrices of the FL family (m uniform in
    [20000, 24000], n = 1.2 m, density 2.5 %, p = 65521; the vectorised
    generator gen.f4_matrix_fast) plus dense Z/p echelon blocks of sizes
    log-uniform in [64, 4096], p in {251, 65521, 2^31-1}.
    * ours: the FL matrices through the batched entry point (8 worker
      streams, tensor-core gemms) and the dense blocks through one batched
      call whose kernel and tile variant per block are chosen by the MLP
      cost model, trained first on autotuner timings of a separate set of
      blocks (small blocks in one persistent graph launch, the others over
      worker streams); both batches are stream-ordered on CUDA streams and
      timed by CUDA events around them;
    * per-matrix tensor cores: the same matrices and blocks one call at a
      time on one stream, tensor-core gemms (the batching gain alone);
    * plain: the per-matrix pipeline with every gemm on the CUDA-core kernel
      and every dense block through the panel pipeline with CUDA-core
      updates.
    The selector's regret is measured on this batch's own dense blocks
    (every candidate timed)."""
    import types
    from lela_b200 import gen
    from lela_b200 import selector as sel
    rng = np.random.default_rng(11)
    primes = [251, 65521, 2147483647]
    fl_items = []
    t_gen = time.perf_counter()
    for i in range(args.batch_fl):
        m = int(rng.integers(20000, 24001))
        X = gen.f4_matrix_fast(3000 + i, m, P, density=FL_DENSITY)
        fl_items.append(types.SimpleNamespace(
            m=X.m, n=X.n, rowptr=torch.from_numpy(X.rowptr.view(np.int64)).to(dev),
            colidx=torch.from_numpy(X.colidx.view(np.int32)).to(dev),
            vals=torch.from_numpy(X.vals.view(np.int32)).to(dev)))
    t_gen = time.perf_counter() - t_gen
    dense = []
    for i in range(args.batch_dense):
        s_ = int(2 ** rng.uniform(6, 12))
        p = int(rng.choice(primes))
        dense.append((torch.from_numpy(gen.dense_zp(4000 + i, s_, s_, p).view(np.int32)).to(dev), p, s_, 4000 + i))
    Rs = [torch.empty((X.m, X.n), dtype=torch.int32, device=dev) for X in fl_items]
    work = [torch.empty_like(A) for A, _, _, _ in dense]

    # cost model from autotuner timings on separate blocks
    t0 = time.perf_counter()
    tuner = sel.Autotuner(cm, reps=2)
    for i in range(32):
        s_ = int(2 ** rng.uniform(6, 12))
        tuner.tune_echelon(s_, s_, int(rng.choice(primes)), seed=9000 + i)
    X_, y_ = sel.records_to_xy(tuner.records)
    model = sel.CostModel(cm, seed=1)
    model.fit(X_, y_, epochs=800)
    choose = sel.Selector(model)
    kernels = [choose.choose("echelon", s_, s_, 0, 1.0, p.bit_length(), s_) for _, p, s_, _ in dense]
    tune_s = time.perf_counter() - t0
    # the selector's regret on this batch's blocks: every candidate timed
    exhaustive = sel.Autotuner(cm, reps=2)
    for _, p, s_, seed in dense:
        exhaustive.tune_echelon(s_, s_, p, seed=seed)
    res_sel = sel.evaluate(choose, sel.group_blocks(exhaustive.records))

    from lela_b200 import CudaModule
    cm_dense = CudaModule(torch.cuda.current_device())
    s2 = torch.cuda.Stream(device=dev)
    cm_dense.set_stream(s2)

    def ours():
        for w, (A, _, _, _) in zip(work, dense):
            w.copy_(A)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s2.wait_event(e0)
        failed = []

        def dense_part():
            try:
                cm_dense.echelonize_batch(work, [p for _, p, _, _ in dense], kernels)
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
        stream.wait_stream(s2)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def one_at_a_time(gemm_kernel, dense_kernel):
        for w, (A, _, _, _) in zip(work, dense):
            w.copy_(A)
        torch.cuda.synchronize()
        cm.set_gemm_kernel(gemm_kernel)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        try:
            e0.record(stream)
            for X, R in zip(fl_items, Rs):
                cm.fl_echelonize(P, X, True, False, R=R)
            for w, (_, p, _, _) in zip(work, dense):
                cm.echelonize_batch([w], [p], [dense_kernel])
            e1.record(stream)
            torch.cuda.synchronize()
        finally:
            cm.set_gemm_kernel(0)
        return e0.elapsed_time(e1)

    ours()
    t_ours = min(ours() for _ in range(3))
    t_tc = one_at_a_time(0, 2)
    t_plain = one_at_a_time(1, 3)
    cm_dense.close()
    ms_ = [X.m for X in fl_items]
    return {"workload": "%d F4 matrices (m uniform 20000-24000, n = 1.2 m, density 2.5%%, p=65521) + %d dense "
                        "echelon blocks (64-4096 log-uniform, p in {251, 65521, 2^31-1})"
                        % (len(fl_items), len(dense)),
            "unit": "ms/batch", "ms": round(t_ours, 1),
            "per_matrix_tc_ms": round(t_tc, 1), "batching_gain": round(t_tc / t_ours, 2),
            "plain_ms": round(t_plain, 1), "speedup_vs_plain": round(t_plain / t_ours, 2),
            "fl_m": ms_, "generation_s": round(t_gen, 1),
            "selector": {"kernels": {sel.KERNEL_NAMES[("echelon", k)]: kernels.count(k) for k in sorted(set(kernels))},
                         "tuning_and_training_s": round(tune_s, 1),
                         "regret_on_batch": round(res_sel["regret"], 4),
                         "gain_vs_default_on_batch": round(res_sel["gain_vs_default"], 4),
                         "exhaustive_ms": round(res_sel["exhaustive_ms"], 2),
                         "selector_ms": round(res_sel["selector_ms"], 2)},
            "timing": "CUDA events on the handle's stream around the stream-ordered batch calls (the FL "
                      "workers and the dense blocks' second stream joined to it); best of 3"}


def fl_cpu_baseline(m_target):
    """LELA's own FaugereLachartre (oracle/_ref) on the same matrix family at
    m = 1000, 2000 and 3000, single-threaded (LELA has no threading), fitted
    as c*m^3 by least squares over the three points and extrapolated to the
    bench's size; labelled as such.  (LELA needs about 40 s at m = 4000 and
    9 min at m = 8000 on one core of this build's CPU, which is why the
    bench stops at 3000.)"""
    import oracle
    from lela_b200 import gen
    if not oracle.have_ref():
        return {"unavailable": "oracle/_ref not built"}
    pts = []
    for m in (1000, 2000, 3000):
        X = gen.f4_matrix(500 + m, m, P, density=FL_DENSITY)
        t0 = time.perf_counter()
        oracle.ref_fl_echelonize_zp(P, X.m, X.n, X.rowptr, X.colidx, X.vals, 1, 0)
        pts.append((m, time.perf_counter() - t0))
    x = np.array([float(m) ** 3 for m, _ in pts])
    y = np.array([t for _, t in pts])
    c = float((x * y).sum() / (x * x).sum())
    rel = [round(float(t / (c * xx)), 3) for t, xx in zip(y, x)]
    return {"kind": "reference", "cores": 1, "cpu": cpu_model(),
            "measured_s": {str(m): round(t, 3) for m, t in pts},
            "fit": "t = c m^3, least squares over the measured points, c = %.3e s; measured / fit = %s" % (c, rel),
            "extrapolated_ms_per_matrix": round(c * m_target ** 3 * 1e3, 1),
            "extrapolation": "fitted c*m^3 at m=%d (extrapolated, not measured)" % m_target}


# ------------------------------------------------------------ reference
def run_reference(args):
    """LELA's own CPU gemm (oracle/_ref; the C restatement if LELA was not
    built) on the bench's workload, all host threads, each step a row slice
    of the 8192^3 gemm sized so that warm-up + steps take about two minutes."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = args.n
    sampler = CpuGemmSampler(n, threads)
    kind, run = sampler.kind, sampler.run
    budget = 120.0 / max(1, args.steps + args.warmup)
    rows = sampler.rows_for(budget)
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
                             "cpu": cpu_model(),
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
    # the largest FL matrix first, before the other workloads hold device memory
    fl_big = run_fl_big(args, torch, dev) if (args.fl_big and not args.no_fl) else None
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

    clocks = clock_sampler(torch, dev, local)
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
    roofline = {"bound": "tensor", "kernel": "zp_gemm_tc_kernel<2, 0, 0> (two limbs, wide tiles)",
                "achieved": round(achieved, 1),
                "peak": round(peak, 1), "unit": "TFLOP/s", "frac": round(achieved / peak, 4),
                "traffic": TC_TRAFFIC_8192 if n == 8192 else None,
                "traffic_unit": "bytes per launch",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                                  "kernel at 8192^3 (one pass, --clock-control none), 1315 + 261 MB; "
                                  "algorithmic bytes 805 MB (limb planes 268 MB, C read and written)",
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

    if not args.no_dense:
        out["dense"] = run_dense(args, cm, stream, torch, dev, peak)
    if not args.no_fl:
        out["fl"] = run_fl(args, cm, stream, torch, dev, rank, zp_peak=peak / 4)
        if fl_big is not None:
            out["fl"]["large"] = fl_big
    if not args.no_gf2:
        out["gf2"] = run_gf2(args, cm, stream, torch, dev, peak)
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
    print(json.dumps(run_fl(args, cm, stream, torch, dev, 0, zp_peak=int8_peak_tops(torch, dev)[0] / 4)))


def run_gf2_only(args):
    """Only the GF(2) line (for kernel launch lists): one process, one GPU;
    prints its JSON object."""
    import torch
    from lela_b200 import CudaModule
    dev = torch.device("cuda", 0)
    cm = CudaModule(0)
    stream = torch.cuda.Stream(device=dev)
    cm.set_stream(stream)
    print(json.dumps(run_gf2(args, cm, stream, torch, dev, int8_peak_tops(torch, dev)[0])))
    cm.close()


def run_gemm_only(args):
    """One Z/p gemm shape C <- C - A*B (the update form of the triangular
    solve and the elimination) on the tensor-core kernel, inputs resident:
    `steps` launches after `warmup`, CUDA events; prints one JSON object
    (for kernel launch lists and profiles of a given shape)."""
    import torch
    from lela_b200 import CudaModule, gen
    m, n, k = (int(x) for x in args.gemm_only.split(","))
    p = args.gemm_p
    dev = torch.device("cuda", 0)
    cm = CudaModule(0)
    stream = torch.cuda.Stream(device=dev)
    cm.set_stream(stream)
    cm.set_gemm_kernel(2)
    cm.set_gemm_tile(args.gemm_tile)
    t = lambda x: torch.from_numpy(x.view(np.int32)).to(dev)
    dA, dB, dC = t(gen.dense_zp(1, m, k, p)), t(gen.dense_zp(2, k, n, p)), t(gen.dense_zp(3, m, n, p))
    for _ in range(max(1, args.warmup)):
        cm.gemm(p, p - 1, dA, dB, 1, dC)
    cm.synchronize()
    cm.profile_reset()
    cm.profile(True)
    ms = _event_ms(torch, stream, lambda: cm.gemm(p, p - 1, dA, dB, 1, dC), args.steps)
    kms, kn = cm.profile_read("zp_gemm_tc")
    cm.profile(False)
    L = 1 if p <= 256 else (2 if p <= 65536 else 4)
    kavg = kms / max(kn, 1)
    print(json.dumps({"workload": "gemm C <- C - A*B, %dx%dx%d, p=%d" % (m, n, k, p), "tile": args.gemm_tile,
                      "ms_per_gemm": round(ms, 4), "kernel_ms": round(kavg, 4),
                      "int8_Tops": round(L * L * 2.0 * m * n * k / (kavg / 1e3) / 1e12, 1),
                      "c_GBs": round(8.0 * m * n / (kavg / 1e3) / 1e9, 1)}))
    cm.close()


def run_echelon_only(args):
    """One dense N x N row-echelon form over Z/65521 (the dense echelon line
    at another size): a warm-up call, then `steps` calls timed by CUDA events
    on the module's stream; prints one JSON object."""
    import torch
    from lela_b200 import CudaModule, gen
    n = args.echelon_only
    dev = torch.device("cuda", 0)
    cm = CudaModule(0)
    stream = torch.cuda.Stream(device=dev)
    cm.set_stream(stream)
    E0 = torch.from_numpy(gen.dense_zp(33, n, n, P).view(np.int32)).to(dev)
    E = E0.clone()
    _, rk, _ = cm.echelonize(P, E)
    times = []
    for _ in range(max(1, args.steps)):
        E.copy_(E0)
        times.append(_event_ms(torch, stream, lambda: cm.echelonize(P, E), 1))
    print(json.dumps({"workload": "row-echelon form, dense %dx%d over Z/65521" % (n, n),
                      "ms": round(min(times), 3), "rank": rk}))
    cm.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.gemm_only:
        run_gemm_only(args)
    elif args.fl_only:
        run_fl_only(args)
    elif args.gf2_only:
        run_gf2_only(args)
    elif args.echelon_only:
        run_echelon_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
