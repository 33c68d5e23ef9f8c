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


def read(text, p, format=FORMAT_DETECT):
    """MatrixReader::read: detects the format unless one is named; the SMS
    format is read here, the other formats raise NotImplementedError."""
    if format == FORMAT_DETECT:
        format = detect_format(text)
    if format == FORMAT_UNKNOWN:
        raise UnrecognisedFormat()
    if format == FORMAT_DUMAS:
        return read_sms(text, p)
    raise NotImplementedError("matrix format %d is not read by this module" % format)
