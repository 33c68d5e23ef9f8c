"""Matrix files in LELA's text formats, for callers of the C ABI and of
CudaModule (LELA's own C++ callers keep LELA's MatrixReader / MatrixWriter,
which do not depend on the Modules type).

Covered: the SMS format of Jean-Guillaume Dumas (FORMAT_DUMAS) -- the
exchange format of F4 matrices -- read and written as MatrixReader::
readDumas and MatrixWriter::writeDumas do over Modular<uint32>
(lela/matrix/io.tcc:233-268, 510-534), and MatrixReader::detectFormat
(io.tcc:163-200) with the reference's own patterns (io.tcc:73-160).

Those patterns write POSIX classes outside a bracket, so "[:digit:]" is
the set of the characters : d i g t, not a digit: the reference detects
"dig it M" as an SMS header and a real one such as "3 4 M" as
FORMAT_UNKNOWN, and its read () with FORMAT_DETECT then raises
UnrecognisedFormat.  detect_format reproduces that; name the format
(read_sms) to read an SMS file, as a LELA caller must.

Reading follows the reference's stream extraction: sizes and indices are
read as size_t (a leading '-' wraps, so "-1" is the largest value), values
as integers truncated to a signed 64-bit long (GMP's mpz_get_si: the low 63
bits of |v| with v's sign) and reduced into [0, p)
(Modular<uint32>::read, lela/ring/modular.h:405-414).  A header whose third
item is not 'M', or an index past the declared size, raises
InvalidMatrixInput; a row index of 0 or -1 ends the entries (its column
and value are consumed); the first item that cannot be read ends them
too, without an error.  Zero values are skipped, so a later zero does not
erase an earlier value at the same place; a later nonzero replaces it.
Where the reference's behaviour is undefined -- a column index of 0 with a
row index in range, which it writes before the row -- this module raises
InvalidMatrixInput.
"""
import math
import re

import numpy as np

FORMAT_DETECT, FORMAT_UNKNOWN, FORMAT_TURNER, FORMAT_ONE_BASED, FORMAT_DUMAS, FORMAT_MAPLE, \
    FORMAT_MATLAB, FORMAT_SAGE, FORMAT_PRETTY = range(9)


class UnrecognisedFormat(Exception):
    """MatrixReader::read could not detect the format (lela/matrix/io.h:46)."""


class InvalidMatrixInput(ValueError):
    """The input is not a valid matrix in the named format (lela/matrix/io.h:51)."""


# The reference's detection patterns in its order (io.tcc:73-160, 172-186).
_DETECT = [
    (FORMAT_DUMAS, r"^[:digit:]+ [:digit:]+ M$"),
    (FORMAT_TURNER, r"^[:digit:]+ [:digit:]+ [:digit:]+$"),
    (FORMAT_MAPLE, r"(\[[:space:]+\])|(\[[:space:]+\[[:space:]+([:digit:]+[:space:]+,[:space:]+)*[:digit:]+)"),
    (FORMAT_MATLAB, r"(\[[:space:]+\])|(\[[:space:]+([:digit:]+[:space:]+,[:space:]+)*[:digit:]+)"),
    (FORMAT_SAGE, r"matrix\((GF\([:digit:]+\),|ZZ|QQ)?[ \t\n]+\[[ \t\n]+\[[:space:]+"
                  r"([:digit:]+[:space:]+,[:space:]+)*[:digit:]+"),
    (FORMAT_PRETTY, r"((\[[:space:]+\])|(\[[:space:]+((\.|[:digit:]+)[:space:]+)*(\.|[:digit:]+)))"),
]
_DETECT = [(tag, re.compile(pat)) for tag, pat in _DETECT]

# the reference reads the first line into a 32-byte buffer (BUF_SIZE, io.tcc:27)
_LINE_CHARS = 31
_SIZE_MAX = (1 << 64) - 1


def detect_format(text):
    """MatrixReader::detectFormat on the start of text: the first line, at
    most 31 characters of it, against the reference's patterns."""
    line = text.split("\n", 1)[0][:_LINE_CHARS]
    for tag, pat in _DETECT:
        if pat.search(line):
            return tag
    return FORMAT_UNKNOWN


class _Scanner:
    """The extractions of std::istream the readers use, on a string."""

    def __init__(self, text):
        self.t = text
        self.i = 0

    def _skip(self):
        t, i = self.t, self.i
        while i < len(t) and t[i].isspace():
            i += 1
        self.i = i

    def _digits(self):
        self._skip()
        t, i = self.t, self.i
        neg = False
        if i < len(t) and t[i] in "+-":
            neg = t[i] == "-"
            i += 1
        j = i
        while j < len(t) and "0" <= t[j] <= "9":
            j += 1
        if j == i:
            return None
        self.i = j
        return neg, int(t[i:j])

    def size(self):
        """is >> size_t: optional sign and decimal digits; a '-' negates
        modulo 2^64; None when nothing can be read or the value overflows."""
        r = self._digits()
        if r is None:
            return None
        neg, v = r
        if v > _SIZE_MAX:
            return None
        return (-v) & _SIZE_MAX if neg else v

    def char(self):
        """is >> char: the next character that is not white space."""
        self._skip()
        if self.i >= len(self.t):
            return None
        c = self.t[self.i]
        self.i += 1
        return c

    def integer(self):
        """is >> mpz_class then get_si: a signed decimal integer truncated to
        a 64-bit long."""
        r = self._digits()
        if r is None:
            return None
        neg, v = r
        if v < (1 << 63) or (neg and v == 1 << 63):
            return -v if neg else v
        low = v & ((1 << 63) - 1)
        return -1 - ((v - 1) & ((1 << 63) - 1)) if neg else low


def read_sms_entries(text, p):
    """readDumas over Z/p: returns (m, n, entries), entries a dict
    {(row, col): value} of the nonzero values, zero-based."""
    s = _Scanner(text)
    m, n, c = s.size(), s.size(), None
    if m is not None and n is not None:
        c = s.char()
    if c != "M":
        raise InvalidMatrixInput("SMS header must be 'm n M'")
    entries = {}
    while True:
        i = s.size()
        if i is None:
            break
        if i == 0 or i == _SIZE_MAX:   # terminator: its column and value are read too
            s.size()
            s.integer()
            break
        j = s.size()
        if j is None:
            break
        if i > m or j > n:
            raise InvalidMatrixInput("entry (%d, %d) outside %d x %d" % (i, j, m, n))
        if j == 0:
            raise InvalidMatrixInput("column index 0 in row %d" % i)
        x = s.integer()
        if x is None:
            break
        x %= p
        if x:
            entries[(i - 1, j - 1)] = x
    return m, n, entries


def read_sms(text, p):
    """The SMS matrix as a dense uint32 array (m x n)."""
    m, n, entries = read_sms_entries(text, p)
    A = np.zeros((m, n), dtype=np.uint32)
    for (i, j), x in entries.items():
        A[i, j] = x
    return A


class CSR:
    """Rows of a sparse matrix in the form the FL entry points take: rowptr
    (uint64, m + 1), colidx and vals (uint32), columns increasing in a row."""

    def __init__(self, m, n, rowptr, colidx, vals):
        self.m, self.n = m, n
        self.rowptr, self.colidx, self.vals = rowptr, colidx, vals


def read_sms_csr(text, p):
    """The SMS matrix as CSR rows (the input of CudaModule.fl_echelonize)."""
    m, n, entries = read_sms_entries(text, p)
    keys = sorted(entries)
    rowptr = np.zeros(m + 1, dtype=np.uint64)
    for (i, _) in keys:
        rowptr[i + 1] += 1
    rowptr = np.cumsum(rowptr, dtype=np.uint64)
    colidx = np.array([j for (_, j) in keys], dtype=np.uint32)
    vals = np.array([entries[k] for k in keys], dtype=np.uint32)
    return CSR(m, n, rowptr, colidx, vals)


def write_sms(A):
    """MatrixWriter::writeDumas of a dense matrix over Z/p (entries already
    reduced): 'm n M', then 'i j v' one-based for every nonzero in row
    order, then '0 0 0', one item per line."""
    A = np.asarray(A)
    m, n = A.shape
    out = ["%d %d M\n" % (m, n)]
    rows, cols = np.nonzero(A)
    out.extend("%d %d %d\n" % (i + 1, j + 1, int(A[i, j])) for i, j in zip(rows, cols))
    out.append("0 0 0\n")
    return "".join(out)


def _ones(A):
    """(i, j, value) of the nonzero entries in row order."""
    rows, cols = np.nonzero(A)
    return [(int(i), int(j), int(A[i, j])) for i, j in zip(rows, cols)]


def _rows_listed(A):
    return [", ".join(str(int(v)) for v in row) for row in A]


def write(A, p, format=FORMAT_PRETTY):
    """MatrixWriter::write of a dense matrix over Z/p (entries already
    reduced) in LELA's text formats (lela/matrix/io.tcc:438-680):
    FORMAT_TURNER (zero-based triples, then -1), FORMAT_ONE_BASED,
    FORMAT_DUMAS, FORMAT_MAPLE, FORMAT_MATLAB, FORMAT_SAGE and FORMAT_PRETTY
    (columns as wide as the decimal width of p, zeros as '.')."""
    A = np.asarray(A)
    m, n = A.shape
    if format == FORMAT_TURNER:
        return "".join("%d %d %d\n" % e for e in _ones(A)) + "-1\n"
    if format == FORMAT_ONE_BASED:
        return "".join("%d %d %d\n" % (i + 1, j + 1, v) for i, j, v in _ones(A))
    if format == FORMAT_DUMAS:
        return write_sms(A)
    if format == FORMAT_MAPLE:
        if m == 0:
            return "[]"
        return "[ " + "], ".join("[" + r for r in _rows_listed(A)) + "] ]\n"
    if format == FORMAT_MATLAB:
        if m == 0:
            return "[]"
        return "[ " + "; ".join(_rows_listed(A)) + "]\n"
    if format == FORMAT_SAGE:
        if m == 0:
            return "matrix([])\n"
        return "matrix([ " + " ],\n         ".join("[ " + r for r in _rows_listed(A)) + " ] ])\n"
    if format == FORMAT_PRETTY:
        if m == 0 or n == 0:
            return "(empty %dx%d matrix)\n" % (m, n)
        # ModularTraits<uint32>::element_width (lela/ring/modular.h:225-226)
        w = int(math.ceil(math.log(float(p)) / math.log(10.0)))
        out = []
        for row in A:
            cells = [(" " * (w - 1) + ". ") if int(v) == 0 else (str(int(v)).rjust(w) + " ") for v in row]
            out.append("  [ " + "".join(cells) + "]\n")
        return "".join(out)
    raise ValueError("no writer for matrix format %d" % format)


def _put(A, i, j, x):
    """A.setEntry (i, j, x) of a matrix the reader does not resize: an index
    outside it is undefined in the reference and an error here."""
    if i >= A.shape[0] or j >= A.shape[1]:
        raise InvalidMatrixInput("entry (%d, %d) outside %d x %d" % ((i, j) + A.shape))
    A[i, j] = x


def read_turner(text, p, shape):
    """MatrixReader::readTurner (lela/matrix/io.tcc:202-231) into a zero m x n
    matrix: one zero-based 'i j v' per line up to a row index of -1.  A line
    that cannot be read as such sets nothing.  The reference reads the first
    line into 32 bytes and the others with a limit of 80: a first line of 32
    or more characters is cut to 31 and ends the input, a line of 80 or more
    ends it unread (lines of 32 to 79 characters after the first overflow
    the reference's buffer; they are read whole here)."""
    A = np.zeros(shape, dtype=np.uint32)
    lines = text.split("\n")
    if text.endswith("\n"):
        lines.pop()
    for k, line in enumerate(lines):
        limit = 31 if k == 0 else 79
        last = len(line) > limit
        if last and k > 0:
            break
        s = _Scanner(line[:limit] if last else line)
        i = s.size()
        if i == _SIZE_MAX:
            break
        j = s.size() if i is not None else None
        x = s.integer() if j is not None else None
        if x is not None and x % p:
            _put(A, i, j, x % p)
        if last:
            break
    return A


def read_matlab(text, p, shape):
    """MatrixReader::readMatlab (lela/matrix/io.tcc:276-341) into a zero m x n
    matrix: '[', then values separated by ',' (next column) and ';' (next
    row), then ']'.  Anything else, a value that does not start with a digit
    or '-', or the end of the text before ']' raises InvalidMatrixInput (so
    does '[]', which the reference's writer produces for an empty matrix)."""
    A = np.zeros(shape, dtype=np.uint32)
    s = _Scanner(text)
    if s.char() != "[":
        raise InvalidMatrixInput("Matlab matrix must start with '['")
    i = j = 0
    while True:
        c = s.char()
        if c is None or not (c.isdigit() or c == "-"):
            raise InvalidMatrixInput("value expected")
        s.i -= 1
        x = s.integer()
        if x is None:
            raise InvalidMatrixInput("value expected")
        if x % p:
            _put(A, i, j, x % p)
        c = s.char()
        if c == ";":
            i, j = i + 1, 0
        elif c == "]":
            break
        elif c == ",":
            j += 1
        else:
            raise InvalidMatrixInput("',', ';' or ']' expected")
    return A


def read_pretty(text, p, shape):
    """MatrixReader::readPretty (lela/matrix/io.tcc:351-409) into a zero m x n
    matrix: one row per '[ ... ]', entries separated by white space, '.' for
    a zero.  A row that is not opened by '[' raises InvalidMatrixInput; the
    end of the text closes an open row.  An entry that is neither a number,
    '.' nor ']' raises InvalidMatrixInput here (the reference does not
    terminate on it)."""
    A = np.zeros(shape, dtype=np.uint32)
    t, n = text, len(text)
    k, i = 0, 0
    while True:
        while k < n and t[k].isspace():
            k += 1
        if k >= n:
            break
        if t[k] != "[":
            raise InvalidMatrixInput("row must start with '['")
        k += 1
        j = 0
        while True:
            while k < n and t[k].isspace():
                k += 1
            if k >= n:
                break
            if t[k] == "]":
                k += 1
                break
            if t[k] == ".":
                k += 1
                j += 1
                continue
            s = _Scanner(t)
            s.i = k
            x = s.integer()
            if x is None:
                raise InvalidMatrixInput("entry expected")
            k = s.i
            if x % p:
                _put(A, i, j, x % p)
            j += 1
        i += 1
    return A


def read(text, p, format=FORMAT_DETECT, shape=None):
    """MatrixReader::read: detects the format unless one is named.  SMS sets
    the size; the Turner, Matlab and Pretty readers fill a zero matrix of the
    given shape, as the reference fills the matrix it is handed.  The
    reference reads no other format (one-based, Maple and Sage raise
    NotImplemented there)."""
    if format == FORMAT_DETECT:
        format = detect_format(text)
    if format == FORMAT_UNKNOWN:
        raise UnrecognisedFormat()
    if format == FORMAT_DUMAS:
        return read_sms(text, p)
    readers = {FORMAT_TURNER: read_turner, FORMAT_MATLAB: read_matlab, FORMAT_PRETTY: read_pretty}
    if format in readers:
        if shape is None:
            raise ValueError("this format does not carry the matrix size: give shape")
        return readers[format](text, p, shape)
    raise NotImplementedError("the reference reads no matrix format %d" % format)
