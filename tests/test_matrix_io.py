"""Matrix files (lela_b200/matrix_io.py) against LELA's MatrixReader /
MatrixWriter (lela/matrix/io.tcc): the committed fixtures of
tests/golden/matrix_io_golden.json (made by make_matrix_io_golden.py from
LELA itself), LELA live where oracle/_ref is built, and the SMS path into
the FL input.  No GPU needed."""
import json
import os

import numpy as np
import pytest

import oracle
from lela_b200 import gen
from lela_b200 import matrix_io as mio

HERE = os.path.dirname(os.path.abspath(__file__))
need_ref = pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref (LELA's CPU code) not built")


def _golden():
    with open(os.path.join(HERE, "golden", "matrix_io_golden.json")) as f:
        return json.load(f)


def _read(text, p):
    try:
        return 0, mio.read_sms(text, p)
    except mio.InvalidMatrixInput:
        return 1, None


def test_golden_detect():
    for case in _golden()["detect"]:
        assert mio.detect_format(case["text"]) == case["format"], case["text"]


def test_golden_write():
    for case in _golden()["write"]:
        A = np.array(case["A"], dtype=np.uint32)
        assert mio.write_sms(A) == case["text"]


def test_golden_read():
    g = _golden()
    for case in g["read"]:
        st, A = _read(case["text"], g["p"])
        assert st == case["status"], case["text"]
        if st == 0:
            want = np.array(case["A"], dtype=np.uint32).reshape(A.shape)
            assert np.array_equal(A, want), case["text"]


def test_read_detect_and_errors():
    """read () with FORMAT_DETECT: a real SMS header is FORMAT_UNKNOWN for
    the reference's patterns, so it raises UnrecognisedFormat; naming the
    format reads it.  Formats the reference does not read raise."""
    text = mio.write_sms(np.array([[1, 0], [0, 2]], dtype=np.uint32))
    with pytest.raises(mio.UnrecognisedFormat):
        mio.read(text, 7)
    assert np.array_equal(mio.read(text, 7, mio.FORMAT_DUMAS), [[1, 0], [0, 2]])
    assert mio.detect_format("tt dd gg\n") == mio.FORMAT_TURNER
    with pytest.raises(ValueError):                      # Turner: the size must be given
        mio.read("tt dd gg\n", 7)
    assert mio.detect_format("[:]\n") == mio.FORMAT_MAPLE
    with pytest.raises(NotImplementedError):             # the reference reads no Maple
        mio.read("[:]\n", 7)
    with pytest.raises(mio.InvalidMatrixInput):
        mio.read_sms("2 2 M\n1 0 5\n0 0 0\n", 7)   # column 0: undefined in the reference


def test_sms_to_fl_input():
    """An F4 matrix written as SMS and read back as CSR rows gives the same
    Faugere-Lachartre result (oracle) as the original rows."""
    p = 65521
    X = gen.f4_matrix_small(5, 60, 80, p)
    D = np.zeros((X.m, X.n), dtype=np.uint32)
    for i in range(X.m):
        a, b = int(X.rowptr[i]), int(X.rowptr[i + 1])
        D[i, X.colidx[a:b]] = X.vals[a:b]
    Y = mio.read_sms_csr(mio.write_sms(D), p)
    assert np.array_equal(Y.rowptr, np.asarray(X.rowptr, dtype=np.uint64))
    assert np.array_equal(Y.colidx, np.asarray(X.colidx, dtype=np.uint32))
    assert np.array_equal(Y.vals, np.asarray(X.vals, dtype=np.uint32))
    want = oracle.fl_echelonize_zp(p, X.m, X.n, X.rowptr, X.colidx, X.vals)
    got = oracle.fl_echelonize_zp(p, Y.m, Y.n, Y.rowptr, Y.colidx, Y.vals)
    assert got["status"] == want["status"] == 0
    assert np.array_equal(got["R"], want["R"]) and got["rank"] == want["rank"]


@need_ref
@pytest.mark.parametrize("p", [2, 251, 65521, 2147483647, 4294967291])
def test_live_round_trip(p):
    rng = np.random.default_rng(p % 977)
    for (m, n) in ((1, 1), (4, 9), (17, 5), (40, 40)):
        A = gen.dense_zp(int(rng.integers(1 << 30)), m, n, p)
        A[rng.random((m, n)) < 0.6] = 0
        text = oracle.ref_write_dumas(p, A)
        assert mio.write_sms(A) == text
        st, B = oracle.ref_read_dumas(p, text)
        assert st == 0 and np.array_equal(mio.read_sms(text, p), B)


@need_ref
def test_live_read_random_texts():
    """Hand-made SMS texts: unsorted and repeated entries, zeros, signed and
    large values, both terminators, missing terminators, entries past the
    size, mixed white space."""
    rng = np.random.default_rng(11)
    p = 65521
    for trial in range(200):
        m, n = int(rng.integers(0, 6)), int(rng.integers(0, 6))
        lines = ["%d %d M" % (m, n)]
        for _ in range(int(rng.integers(0, 12))):
            i = int(rng.integers(1, m + 2)) if rng.random() < 0.95 else -int(rng.integers(2, 5))
            j = int(rng.integers(1, n + 2))
            v = int(rng.choice([0, 1, p, p - 1, -1, -p - 3, 1 << 40, -(1 << 62), int(rng.integers(-10**6, 10**6))]))
            lines.append("%d %d %d" % (i, j, v))
        r = rng.random()
        if r < 0.4:
            lines.append("0 0 0")
        elif r < 0.6:
            lines.append("-1 3 4")
            lines.append("1 1 5")
        sep = ["\n", "\r\n", " \t\n"][trial % 3]
        text = sep.join(lines) + sep
        st, want = oracle.ref_read_dumas(p, text)
        got_st, got = _read(text, p)
        assert got_st == st, text
        if st == 0:
            assert np.array_equal(got, want), text


@need_ref
def test_live_detect():
    rng = np.random.default_rng(3)
    alphabet = list("0123456789 :digtspace[],;.M()GFZQmatrix\t")
    for _ in range(400):
        line = "".join(rng.choice(alphabet, size=int(rng.integers(0, 40))))
        text = line + "\n1 1 1\n"
        assert mio.detect_format(text) == oracle.ref_detect_format(text), repr(line)


def test_golden_write_all_formats():
    for case in _golden()["write_all"]:
        A = np.array(case["A"], dtype=np.uint32)
        for fmt, text in case["text"].items():
            assert mio.write(A, case["p"], int(fmt)) == text, fmt


def test_golden_read_other_formats():
    g = _golden()
    for case in g["read_other"]:
        try:
            st, A = 0, mio.read(case["text"], g["p"], case["format"], tuple(case["shape"]))
        except mio.InvalidMatrixInput:
            st, A = 1, None
        assert st == case["status"], case["text"]
        if st == 0:
            assert np.array_equal(A, np.array(case["A"], dtype=np.uint32)), case["text"]


def _random_value(rng, p):
    return int(rng.choice([0, 1, p - 1, p, -1, -p - 2, 1 << 40, int(rng.integers(-10**6, 10**6))]))


@need_ref
def test_live_read_turner():
    """Short lines only: the reference overflows its 32-byte buffer on lines
    of 32 to 79 characters after the first."""
    rng = np.random.default_rng(21)
    p = 65521
    for _ in range(150):
        m, n = int(rng.integers(1, 5)), int(rng.integers(1, 5))
        lines = []
        for _ in range(int(rng.integers(0, 9))):
            r = rng.random()
            if r < 0.75:
                lines.append("%d %d %d" % (rng.integers(0, m), rng.integers(0, n), _random_value(rng, p) % (10**9)))
            elif r < 0.85:
                lines.append(rng.choice(["", "7", "1 2", "x 1 1", "  "]))
            else:
                lines.append("-1")
        text = "\n".join(lines) + ("\n" if rng.random() < 0.7 else "")
        st, want = oracle.ref_read_matrix(mio.FORMAT_TURNER, p, text, m, n)
        assert st == 0
        assert np.array_equal(mio.read(text, p, mio.FORMAT_TURNER, (m, n)), want), text


@need_ref
def test_live_read_matlab_pretty():
    """Well-formed texts with random spacing and values, and ones cut short
    or with a stray character, within the matrix bounds (the reference
    writes outside them unchecked, and loops without end on a Pretty entry
    that is not a number, '.' or ']')."""
    rng = np.random.default_rng(22)
    p = 65521
    sp = lambda: rng.choice(["", " ", "  ", "\n", "\t"])
    for trial in range(300):
        m, n = int(rng.integers(1, 4)), int(rng.integers(1, 4))
        vals = [[_random_value(rng, p) for _ in range(n)] for _ in range(m)]
        if trial % 2 == 0:
            fmt = mio.FORMAT_MATLAB
            text = sp() + "[" + sp() + (sp() + ";" + sp()).join(
                (sp() + "," + sp()).join(str(v) for v in row) for row in vals) + sp() + "]"
            r = rng.random()
            if r < 0.15:
                text = text[:-1]
            elif r < 0.3:
                k = int(rng.integers(1, len(text)))
                text = text[:k] + rng.choice(["x", ":", "(", "--"]) + text[k:]
        else:
            fmt = mio.FORMAT_PRETTY
            rows = ["[" + " ".join("." if v % p == 0 and rng.random() < 0.5 else str(v) for v in row) + sp() + "]"
                    for row in vals]
            text = sp().join(r + "\n" for r in rows)
            if rng.random() < 0.2:
                text = text.rstrip()[:-1]
        st, want = oracle.ref_read_matrix(fmt, p, text, m, n)
        try:
            got_st, got = 0, mio.read(text, p, fmt, (m, n))
        except mio.InvalidMatrixInput:
            got_st, got = 1, None
        assert got_st == st, (fmt, text)
        if st == 0:
            assert np.array_equal(got, want), (fmt, text)


@need_ref
@pytest.mark.parametrize("p", [2, 7, 10, 251, 65521, 4294967291])
def test_live_write_all_formats(p):
    """Every text format; not m x 0 in the triple formats, where the
    reference's raw iteration of a dense matrix crashes."""
    for (m, n) in ((0, 0), (0, 3), (2, 0), (1, 1), (2, 3), (5, 4)):
        A = gen.dense_zp(m * 10 + n, m, n, p) if m * n else np.zeros((m, n), dtype=np.uint32)
        if m * n:
            A[A % 3 == 0] = 0
        for fmt in range(2, 9):
            if m > 0 and n == 0 and fmt in (mio.FORMAT_TURNER, mio.FORMAT_ONE_BASED, mio.FORMAT_DUMAS):
                continue
            assert mio.write(A, p, fmt) == oracle.ref_write_matrix(fmt, p, A), (m, n, fmt)
