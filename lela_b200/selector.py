"""Autotuner and learned kernel selector.

Several kernels compute the same exact result for a block (Z/p gemm on the
tensor cores, with wide tiles or with tiles of two accumulator buffers, or
on CUDA cores, plain or small-K; GF(2) gemm int8-expanded on the tensor
cores or bit-packed four-Russians; a dense echelon block in one CTA's shared
memory or through the panel pipeline with tensor-core updates of either
tile variant or CUDA-core updates).  Which is fastest depends on the block.

* ``Autotuner`` times every candidate (kernel and tile variant) on a block
  (exhaustive search) and records ``{op, features, kernel, ms}`` lines
  (JSONL).
* ``CostModel`` is a fully connected FP32 network (14 -> 64 -> 64 -> 1,
  ReLU) that predicts log time from the block features and a description
  of the candidate (operation, kernel family, tile variant).  It is trained
  on the GPU by the library's own forward / backward / Adam kernels
  (``lela_cuda_mlp_*``) from the autotuner's records.
* ``Selector`` picks the candidate with the smallest predicted time, and
  falls back to exhaustive tuning when no model is loaded.

The choice never changes a result: every candidate is bit-exact.
"""
import ctypes
import json
import math
import time

import numpy as np

from . import api

# Candidates per operation: kernel id -> (kernel family, tile variant).
# Families: "plain" (CUDA-core delayed-reduction products), "small" (a
# CUDA-core kernel for small work: the small-K gemm, bit-packed
# four-Russians, the one-CTA shared-memory echelon), "tc" (tensor cores).
# Tiles (tensor cores): "wide" (one accumulator buffer for two and four
# limbs) or "double" (two buffers, the epilogue overlapping the next tile).
# The ids are the ones the library takes: lela_cuda_set_gemm_kernel /
# set_gemm_tile for gemm, lela_cuda_set_gf2_kernel, and the per-block
# kernel of lela_cuda_echelon_zp_u32_batch.
KERNELS = {
    "gemm": {1: ("plain", None), 2: ("tc", "wide"), 3: ("small", None), 4: ("tc", "double")},
    "gf2_gemm": {1: ("tc", "wide"), 2: ("small", None)},
    "echelon": {1: ("small", None), 2: ("tc", "wide"), 3: ("plain", None), 4: ("tc", "double")},
}
KERNEL_NAMES = {("gemm", 1): "zp CUDA-core (plain)", ("gemm", 2): "zp tensor-core, wide tiles",
                ("gemm", 3): "zp CUDA-core small-K", ("gemm", 4): "zp tensor-core, double-buffered tiles",
                ("gf2_gemm", 1): "gf2 tensor-core", ("gf2_gemm", 2): "gf2 four-Russians",
                ("echelon", 1): "echelon shared-memory batch",
                ("echelon", 2): "echelon panels, TC updates (wide tiles)",
                ("echelon", 3): "echelon panels, CUDA-core updates",
                ("echelon", 4): "echelon panels, TC updates (double-buffered tiles)"}
DEFAULT = {"gemm": 2, "gf2_gemm": 1, "echelon": 2}   # the choice without a model
OPS = ("gemm", "gf2_gemm", "echelon")
FAMILIES = ("plain", "small", "tc")
NFEAT = 6 + len(OPS) + len(FAMILIES) + 2


def candidates(op, m, n, k, pbits=16):
    """Kernel ids worth timing for this block (four-limb moduli have one
    tensor-core tile variant; the shared-memory echelon kernel takes blocks
    of at most 200 KB)."""
    if op == "gemm":
        return [1, 2, 3] + ([4] if pbits <= 16 else [])
    if op == "gf2_gemm":
        return [1, 2]
    if op == "echelon":
        c = [2, 3] + ([4] if pbits <= 16 else [])
        if m * n * 4 <= 200 * 1024:
            c.insert(0, 1)
        return c
    raise ValueError(op)


def features(op, kernel, m, n, k, density, pbits, pivots):
    """Numeric block features (m, n, k, density, bits of p, pivot count,
    log-scaled), then the candidate: one-hot operation, one-hot kernel
    family, and the tile variant (wide, double) of a tensor-core kernel."""
    lg = lambda v: math.log2(max(1.0, float(v))) / 16.0
    f = [lg(m), lg(n), lg(k), float(density), float(pbits) / 32.0, lg(pivots)]
    fam, tile = KERNELS[op][kernel]
    f += [1.0 if op == o else 0.0 for o in OPS]
    f += [1.0 if fam == x else 0.0 for x in FAMILIES]
    f += [1.0 if tile == "wide" else 0.0, 1.0 if tile == "double" else 0.0]
    return f


class CostModel:
    """The network's parameters on the GPU and its training loop."""

    def __init__(self, cm, seed=0, device="cuda"):
        import torch
        self.cm, self.torch = cm, torch
        L = cm.L
        L.lela_cuda_mlp_param_count.argtypes = [ctypes.c_int]
        L.lela_cuda_mlp_param_count.restype = ctypes.c_size_t
        P, S = ctypes.c_void_p, ctypes.c_size_t
        L.lela_cuda_mlp_forward.argtypes = [P, P, ctypes.c_int, P, S, P]
        L.lela_cuda_mlp_grad.argtypes = [P, P, ctypes.c_int, P, P, S, P, P]
        L.lela_cuda_mlp_adam.argtypes = [P, P, P, P, P, S, ctypes.c_int, ctypes.c_float]
        self.np = int(L.lela_cuda_mlp_param_count(NFEAT))
        g = np.random.default_rng(seed)
        H = 64
        parts = [g.normal(0, math.sqrt(2.0 / NFEAT), NFEAT * H), np.zeros(H),
                 g.normal(0, math.sqrt(2.0 / H), H * H), np.zeros(H),
                 g.normal(0, math.sqrt(1.0 / H), H), np.zeros(1)]
        self.params = torch.tensor(np.concatenate(parts), dtype=torch.float32, device=device)
        assert self.params.numel() == self.np
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step_no = 0
        self.mu = 0.0
        self.sd = 1.0

    def _p(self, t):
        return ctypes.c_void_p(t.data_ptr())

    def predict(self, X):
        """Predicted log time for feature rows X (numpy n x NFEAT)."""
        torch = self.torch
        Xt = torch.tensor(np.asarray(X, dtype=np.float32), device=self.params.device)
        out = torch.empty(Xt.shape[0], dtype=torch.float32, device=self.params.device)
        st = self.cm.L.lela_cuda_mlp_forward(self.cm.h, self._p(self.params), NFEAT, self._p(Xt),
                                             Xt.shape[0], self._p(out))
        self.cm._raise(st)
        self.cm.synchronize()
        return out.cpu().numpy() * self.sd + self.mu

    def gradient(self, X, y):
        """(loss, grad) of the mean squared error on standardised targets."""
        torch = self.torch
        Xt = torch.tensor(np.asarray(X, dtype=np.float32), device=self.params.device)
        yt = torch.tensor(np.asarray(y, dtype=np.float32), device=self.params.device)
        st = self.cm.L.lela_cuda_mlp_grad(self.cm.h, self._p(self.params), NFEAT, self._p(Xt),
                                          self._p(yt), Xt.shape[0], self._p(self.grad),
                                          self._p(self.loss))
        self.cm._raise(st)
        self.cm.synchronize()
        return float(self.loss.item()), self.grad.cpu().numpy()

    def fit(self, X, y, epochs=400, lr=3e-3):
        """Full-batch Adam on log times (standardised); returns the loss curve."""
        torch = self.torch
        y = np.asarray(y, dtype=np.float64)
        self.mu, self.sd = float(y.mean()), float(y.std() or 1.0)
        Xt = torch.tensor(np.asarray(X, dtype=np.float32), device=self.params.device)
        yt = torch.tensor(((y - self.mu) / self.sd).astype(np.float32), device=self.params.device)
        L, h = self.cm.L, self.cm.h
        losses = []
        for _ in range(epochs):
            st = L.lela_cuda_mlp_grad(h, self._p(self.params), NFEAT, self._p(Xt), self._p(yt),
                                      Xt.shape[0], self._p(self.grad), self._p(self.loss))
            self.cm._raise(st)
            self.step_no += 1
            st = L.lela_cuda_mlp_adam(h, self._p(self.params), self._p(self.grad), self._p(self.m),
                                      self._p(self.v), self.np, self.step_no, ctypes.c_float(lr))
            self.cm._raise(st)
            losses.append(self.loss.clone())
        self.cm.synchronize()
        return [float(x.item()) for x in losses[:: max(1, len(losses) // 50)]]

    def state(self):
        return {"params": self.params.cpu().numpy().tolist(), "mu": self.mu, "sd": self.sd}


class Autotuner:
    """Exhaustive timing of every candidate kernel on a block (CUDA events on
    the module's stream, best of `reps` after one warm-up)."""

    def __init__(self, cm, reps=3):
        import torch
        self.cm, self.torch, self.reps = cm, torch, reps
        self.records = []

    def _time(self, fn):
        torch = self.torch
        s = torch.cuda.Stream()
        self.cm.set_stream(s)
        try:
            fn()
            self.cm.synchronize()
            best = float("inf")
            for _ in range(self.reps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(s)
                fn()
                e1.record(s)
                self.cm.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best
        finally:
            self.cm.set_stream(None)

    def tune_gemm(self, m, n, k, p, seed=0):
        from . import gen
        torch = self.torch
        t = lambda x: torch.from_numpy(x.view(np.int32)).cuda()
        A, B, C = t(gen.dense_zp(seed, m, k, p)), t(gen.dense_zp(seed + 1, k, n, p)), t(gen.dense_zp(seed + 2, m, n, p))
        out = {}
        for kern in candidates("gemm", m, n, k, p.bit_length()):
            set_gemm_choice(self.cm, kern)
            out[kern] = self._time(lambda: self.cm.gemm(p, 1, A, B, 1, C))
        set_gemm_choice(self.cm, 0)
        return self._record("gemm", m, n, k, 1.0, p.bit_length(), 0, out)

    def tune_gf2_gemm(self, m, n, k, seed=0):
        torch = self.torch
        r = lambda a, b: torch.randint(-2 ** 62, 2 ** 62, (a, (b + 63) // 64), dtype=torch.int64, device="cuda")
        A, B, C = r(m, k), r(k, n), r(m, n)
        if k % 64:
            A[:, -1] &= (1 << (k % 64)) - 1
        if n % 64:
            B[:, -1] &= (1 << (n % 64)) - 1
            C[:, -1] &= (1 << (n % 64)) - 1
        out = {}
        for kern in candidates("gf2_gemm", m, n, k):
            self.cm.set_gf2_kernel(kern)
            out[kern] = self._time(lambda: self.cm.gemm_gf2(A, B, C, n, k, 1, 1))
        self.cm.set_gf2_kernel(0)
        return self._record("gf2_gemm", m, n, k, 0.5, 1, 0, out)

    def tune_echelon(self, m, n, p, seed=0):
        from . import gen
        torch = self.torch
        src = torch.from_numpy(gen.dense_zp(seed, m, n, p).view(np.int32)).cuda()
        work = torch.empty_like(src)
        out = {}
        for kern in candidates("echelon", m, n, 0, p.bit_length()):
            def run():
                work.copy_(src)
                self.cm.echelonize_batch([work], [p], kernels=[kern])
            out[kern] = self._time(run)
        return self._record("echelon", m, n, 0, 1.0, p.bit_length(), min(m, n), out)

    def _record(self, op, m, n, k, density, pbits, pivots, out):
        for kern, ms in out.items():
            self.records.append({"op": op, "m": m, "n": n, "k": k, "density": density,
                                 "pbits": pbits, "pivots": pivots, "kernel": kern, "ms": ms})
        return out

    def dump(self, path):
        with open(path, "w") as f:
            for r in self.records:
                f.write(json.dumps(r) + "\n")


def records_to_xy(records):
    X = [features(r["op"], r["kernel"], r["m"], r["n"], r["k"], r["density"], r["pbits"], r["pivots"])
         for r in records]
    y = [math.log(max(r["ms"], 1e-4)) for r in records]
    return np.array(X, dtype=np.float32), np.array(y)


def group_blocks(records):
    """{block key: {kernel: ms}} from autotuner records."""
    blocks = {}
    for r in records:
        key = (r["op"], r["m"], r["n"], r["k"], r["density"], r["pbits"], r["pivots"])
        blocks.setdefault(key, {})[r["kernel"]] = r["ms"]
    return blocks


def set_gemm_choice(cm, kern):
    """Apply a gemm kernel id of KERNELS (0: the library's automatic
    choice) to a module handle."""
    kernel, tile = {0: (0, 0), 1: (1, 0), 2: (2, 1), 3: (3, 0), 4: (2, 2)}[kern]
    cm.set_gemm_kernel(kernel)
    cm.set_gemm_tile(tile)


class Selector:
    """Pick a kernel per block: the cost model's argmin, else exhaustive."""

    def __init__(self, model=None, tuner=None):
        self.model, self.tuner = model, tuner

    def choose(self, op, m, n, k, density, pbits, pivots):
        cands = candidates(op, m, n, k, pbits)
        if self.model is None:
            return DEFAULT[op]
        X = [features(op, c, m, n, k, density, pbits, pivots) for c in cands]
        pred = self.model.predict(X)
        return cands[int(np.argmin(pred))]


def evaluate(selector, blocks):
    """Total time of the selector's choices, of the best choices (exhaustive
    tuning) and of the default choices (no model) over measured blocks."""
    t_sel = t_best = t_def = 0.0
    for (op, m, n, k, density, pbits, pivots), times in blocks.items():
        c = selector.choose(op, m, n, k, density, pbits, pivots)
        t_sel += times[c]
        t_best += min(times.values())
        t_def += times[DEFAULT[op]]
    return {"selector_ms": t_sel, "exhaustive_ms": t_best, "default_ms": t_def,
            "regret": t_sel / t_best - 1.0, "gain_vs_default": t_def / t_sel}
