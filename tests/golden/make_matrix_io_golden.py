"""Generate tests/golden/matrix_io_golden.json from LELA's own matrix I/O.

    python tests/golden/make_matrix_io_golden.py

Needs oracle/_ref/liblela_ref.so (make -C oracle ref).  Records, for the
cases below, what LELA's MatrixReader::detectFormat returns on a first
line, what MatrixWriter::write writes for small matrices from
lela_b200.gen (FORMAT_DUMAS, and every text format), and what
MatrixReader::read makes of hand-written texts in the SMS, Turner, Matlab
and Pretty formats (status: 0 read, 1 InvalidMatrixInput).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from lela_b200 import gen  # noqa: E402

P = 65521

FIRST_LINES = [
    "3 4 M", "12 34 M", "dig it M", "1 2 3", "tt dd gg", "[[1, 2], [3, 4]]", "[ [ 1 , 2 ] ]",
    "[1, 2; 3, 4]", "[ 1, 2; 3, 4]", "matrix(GF(7), [[1, 2]])", "[ 1 2 ]", "[ . 2 ]",
    "[ : ]", "[ : : ]", "[ :d : , t ]", "hello", "", "a very long first line that is longer than the buffer M",
]

READ_CASES = [
    "3 4 M\n1 1 5\n2 3 -7\n3 4 70000\n0 0 0\n",
    "2 2 M\n1 1 5\n1 1 0\n2 2 3\n2 2 9\n0 0 0\n",
    "2 2 M\n1 1 5\n-1 0 0\n2 2 3\n",
    "2 2 M\n1 2 4\n",
    "2 2 M\n3 1 4\n0 0 0\n",
    "2 2 M\n1 3 4\n0 0 0\n",
    "2 2 M\n-5 1 4\n0 0 0\n",
    "2 2 X\n1 1 1\n",
    "1 1 M\n1 1 123456789012345\n0 0 0\n",
    "1 2 M\n1 1 9223372036854775807\n1 2 -9223372036854775807\n0 0 0\n",
    "2 2 M\r\n1 1 5\r\n2 1 65521\r\n0 0 0\r\n",
    "2 3 M\n1\t3\t8\n2 2 65530\n0 0 0\n",
    "0 0 M\n0 0 0\n",
    "2 2 M\n1 1\n",
    "2 2 M\n99999999999999999999 1 5\n",
    "4 3 M\n4 3 1\n1 1 2\n3 2 -1\n0 0 0\n2 2 7\n",
]


# (format, shape, text): the Turner (2), Matlab (6) and Pretty (8) readers
OTHER_READS = [
    (2, (2, 3), "0 0 3\n1 2 -1\n\n5\n1 1\n-1\n0 1 4\n"),
    (2, (2, 2), "1 0 70000\n0 1 65521"),
    (2, (3, 3), "0 0 1 and a first line past 31 chars\n1 1 1\n"),
    (6, (2, 3), "[ 1, 0, 5; 0, 7, 0]\n"),
    (6, (2, 2), "  [1,-2 ;3, 4 ]"),
    (6, (2, 2), "[ 1, 2; 3, 4"),
    (6, (2, 2), "[ 1 2 ]"),
    (6, (1, 1), "[]"),
    (6, (1, 2), "( 1, 2 )"),
    (8, (2, 3), "  [     1     . 65520 ]\n  [     .     7     . ]\n"),
    (8, (3, 2), "[1 .]\n[]\n[ -4 5"),
    (8, (2, 2), "1 2\n"),
]


def main():
    assert oracle.have_ref(), "build oracle/_ref first (make -C oracle ref)"
    out = {"p": P, "detect": [], "write": [], "read": []}
    for line in FIRST_LINES:
        out["detect"].append({"text": line + "\n1 1 1\n", "format": oracle.ref_detect_format(line + "\n1 1 1\n")})
    for i, (m, n) in enumerate([(1, 1), (3, 5), (6, 4), (7, 9)]):
        A = gen.dense_zp(900 + i, m, n, P)
        A[A % 3 == 0] = 0
        out["write"].append({"A": A.tolist(), "text": oracle.ref_write_dumas(P, A)})
    for text in READ_CASES:
        st, A = oracle.ref_read_dumas(P, text)
        out["read"].append({"text": text, "status": st, "A": None if A is None else A.tolist()})
    out["write_all"] = []
    for i, (p, m, n) in enumerate([(7, 2, 3), (65521, 3, 4), (4294967291, 2, 2), (10, 3, 3)]):
        A = gen.dense_zp(950 + i, m, n, p)
        A[A % 3 == 0] = 0
        out["write_all"].append({"p": p, "A": A.tolist(),
                                 "text": {str(fmt): oracle.ref_write_matrix(fmt, p, A) for fmt in range(2, 9)}})
    out["read_other"] = []
    for fmt, shape, text in OTHER_READS:
        st, A = oracle.ref_read_matrix(fmt, P, text, *shape)
        out["read_other"].append({"format": fmt, "shape": list(shape), "text": text, "status": st,
                                  "A": None if A is None else A.tolist()})
    with open(os.path.join(HERE, "matrix_io_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", len(out["detect"]), "detections,", len(out["write"]), "writes,", len(out["read"]), "reads")


if __name__ == "__main__":
    main()
