"""Golden digests of LELA's FaugereLachartre at F4-matrix sizes the GPU
tests check bit-exactly (tests/golden/fl_large.json).

    python tests/golden/make_fl_large.py            # m = 4000 (4 modes), 8000 (reduced)

Needs oracle/_ref/liblela_ref.so (LELA's own CPU code, `make -C oracle ref`).
Each case is one matrix of the F4 family (lela_b200.gen.f4_matrix, p = 65521,
n = 1.2 m, row density 2.5 %, 75 % pivot rows, 5 % of the non-pivot rows
dependent), echelonized by LELA's FaugereLachartre<Modular<uint32>>::
echelonize (faugere-lachartre.tcc:735-917) in the given mode.  Stored: the
generator arguments, SHA-256 digests of the CSR input and of LELA's dense
output R, rank and det.  LELA needs about 40 s (m = 4000) and 5 min
(m = 8000) per matrix on one core, so the cases run in parallel processes.
"""
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

P = 65521
DENSITY = 0.025
CASES = [(4000, 41, 1, 0), (4000, 41, 0, 0), (4000, 41, 1, 1), (4000, 41, 0, 1),
         (8000, 83, 1, 0)]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def input_sha(X):
    h = hashlib.sha256()
    for a in (X.rowptr, X.colidx, X.vals):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def one(case):
    import oracle
    from lela_b200 import gen
    m, seed, red, od = case
    X = gen.f4_matrix(seed, m, P, density=DENSITY)
    t0 = time.time()
    r = oracle.ref_fl_echelonize_zp(P, X.m, X.n, X.rowptr, X.colidx, X.vals, red, od)
    t = time.time() - t0
    assert r["status"] == 0, r["status"]
    return {"m": m, "n": X.n, "seed": seed, "p": P, "density": DENSITY, "reduced": red,
            "only_D": od, "input_sha": input_sha(X), "R_sha": sha(r["R"]),
            "rank": int(r["rank"]), "det": int(r["det"]), "lela_s": round(t, 1)}


def main():
    import oracle
    assert oracle.have_ref(), "build oracle/_ref first (make -C oracle ref)"
    with mp.get_context("spawn").Pool(len(CASES)) as pool:
        rows = pool.map(one, CASES)
    out = {"generator": "lela_b200.gen.f4_matrix(seed, m, p, density=density)",
           "computed_by": "LELA FaugereLachartre<Modular<uint32>>::echelonize (oracle/_ref)",
           "cases": rows}
    with open(os.path.join(HERE, "fl_large.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
