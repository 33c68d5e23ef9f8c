"""Access to the committed golden fixtures (tests/golden/lela_golden.*),
computed by LELA's own CPU code (tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_cache = {}


def data():
    if "npz" not in _cache:
        _cache["npz"] = dict(np.load(os.path.join(HERE, "lela_golden.npz")))
        _cache["json"] = json.load(open(os.path.join(HERE, "lela_golden.json")))
    return _cache["npz"], _cache["json"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def gemm_cases():
    z, man = data()
    for pre in man["gemm_small"]:
        p, a, b = (int(x) for x in z[pre + "meta"])
        yield pre, p, a, b, z[pre + "A"], z[pre + "B"], z[pre + "C"], z[pre + "R"]


def trsm_cases():
    z, man = data()
    for pre in man["trsm"]:
        p, upper, unit, a, bad = (int(x) for x in z[pre + "meta"])
        yield pre, p, upper, unit, a, (None if bad < 0 else bad), z[pre + "A"], z[pre + "B"], z[pre + "R"]


def echelon_cases():
    z, man = data()
    for pre in man["echelon"]:
        p, st, r, d = (int(x) for x in z[pre + "meta"])
        yield pre, p, st, r, d, z[pre + "A"], z[pre + "E"]


def echelon_reduced_cases(unit=False):
    """unit: the standard method's form (Elimination::echelonize_reduced)."""
    z, man = data()
    for pre in man["echelon_reduced_unit" if unit else "echelon_reduced"]:
        p, st, r, d = (int(x) for x in z[pre + "meta"])
        yield pre, p, st, r, d, z[pre + "A"], z[pre + "E"]


def pluq_cases():
    z, man = data()
    for pre in man["pluq"]:
        p, st, r, d = (int(x) for x in z[pre + "meta"])
        P = [tuple(int(v) for v in t) for t in z[pre + "P"]]
        Q = [tuple(int(v) for v in t) for t in z[pre + "Q"]]
        yield pre, p, st, r, d, z[pre + "A"], z[pre + "E"], P, Q


def fl_cases(with_inputs_only=True):
    """Faugere-Lachartre cases whose inputs are stored (the reference test's
    matrix family)."""
    z, man = data()
    for pre in man["fl"]:
        meta = [int(x) for x in z[pre + "meta"]]
        if pre + "rowptr" not in z:
            continue
        p, m, n, red, od, st, rank, det = meta
        yield (pre, p, m, n, red, od, st, rank, det, z[pre + "rowptr"], z[pre + "colidx"],
               z[pre + "vals"], z[pre + "R"])


def gf2_gemm_cases():
    z, man = data()
    for pre in man["gf2_gemm"]:
        m, n, k = (int(x) for x in z[pre + "meta"])
        yield pre, m, n, k, z[pre + "A"], z[pre + "B"], z[pre + "C"], z[pre + "R"]


def gf2_echelon_cases():
    z, man = data()
    for pre in man["gf2_echelon"]:
        m, n, r = (int(x) for x in z[pre + "meta"])
        yield pre, m, n, r, z[pre + "A"], z[pre + "E"]


def transform_cases(gj=False):
    """Elimination::echelonize_reduced with compute_L (gj: GaussJordan::
    echelonize_reduced with its transform), as LELA computed it
    (tests/golden/make_transform_golden.py): (pre, p, status, rank, det, A,
    R, L, P)."""
    fname = "gj_transform_golden.npz" if gj else "transform_golden.npz"
    if fname not in _cache:
        _cache[fname] = dict(np.load(os.path.join(HERE, fname)))
    z = _cache[fname]
    for pre in z["names"]:
        pre = str(pre)
        p, st, r, d = (int(x) for x in z[pre + "meta"])
        P = [tuple(int(v) for v in t) for t in z[pre + "P"]]
        yield pre, p, st, r, d, z[pre + "A"], z[pre + "R"], z[pre + "L"], P


def packed_cases():
    """Elimination::echelonize / GaussJordan::echelonize with L kept below
    the diagonal, as LELA computed them (tests/golden/
    make_transform_golden.py): (pre, gauss_jordan, p, status, rank, det, A,
    E, P)."""
    if "packed" not in _cache:
        _cache["packed"] = dict(np.load(os.path.join(HERE, "packed_golden.npz")))
    z = _cache["packed"]
    for pre in z["names"]:
        pre = str(pre)
        for g in (0, 1):
            p, st, r, d = (int(x) for x in z[pre + "meta%d" % g])
            P = [tuple(int(v) for v in t) for t in z[pre + "P%d" % g]]
            yield pre, bool(g), p, st, r, d, z[pre + "A"], z[pre + "E%d" % g], P
