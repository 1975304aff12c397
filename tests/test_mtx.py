"""Matrix files on the host: the MatrixMarket reader (spmx_mtx_read) against
the oracle's ReadMTX restatement, the restatement against the reference's own
ReadMTX (compiled from its sources into oracle/_ref when the reference tree is
present), and the binary CSR cache against the reference's storeCSR / loadCSR
in both directions.  Host only.

The product returns the COO in file order (the sort runs on the GPU); here it
is sorted stably by (row, col) with numpy before the comparison, which is
what the oracle's stable sort does.  The reference's std::sort is not stable,
so files with duplicate (row, col) entries compare as multisets against it.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle.oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")

# name -> (text, has duplicate (row, col) entries)
CASES = {
    "general_real": ("%%MatrixMarket matrix coordinate real general\n"
                     "% a comment\n"
                     "4 5 7\n"
                     "1 1 1.5\n3 2 -2.25e-3\n2 5 +7\n4 4 .5\n1 3 1e-40\n4 1 -0\n2 2 3.4028235e38\n",
                     False),
    "symmetric_real": ("%%MatrixMarket matrix coordinate real symmetric\n"
                       "5 5 6\n"
                       "1 1 2.0\n2 1 -1.0\n3 2 0.125\n5 5 9\n5 1 1e5\n4 3 -7.75\n", False),
    "pattern_symmetric": ("%%MatrixMarket matrix coordinate pattern symmetric\n"
                          "6 6 5\n2 1\n3 1\n6 2\n4 4\n6 5\n", False),
    "integer_general": ("%%MatrixMarket matrix coordinate integer general\n"
                        "3 3 4\n1 2 -5\n3 3 16777217\n2 1 42\n1 1 0\n", False),
    "complex_general": ("%%MatrixMarket matrix coordinate complex general\n"
                        "2 3 3\n1 3 1.5 -2\n2 1 0 1\n1 1 3 3\n", False),
    "comments_crlf_tabs": ("%%MatrixMarket matrix coordinate real general\r\n"
                           "%\r\n% second comment line\r\n\r\n"
                           "3 4 3\r\n1\t4\t0.75\r\n  3 1  -1\r\n2 2 2\r\n", False),
    "empty": ("%%MatrixMarket matrix coordinate real general\n7 3 0\n", False),
    "skew_symmetric": ("%%MatrixMarket matrix coordinate real skew-symmetric\n"
                       "3 3 2\n2 1 1.0\n3 2 -2.0\n", False),
    "no_trailing_newline": ("%%MatrixMarket matrix coordinate real general\n"
                            "2 2 2\n1 1 1\n2 2 2", False),
    "duplicates": ("%%MatrixMarket matrix coordinate real general\n"
                   "3 3 6\n2 2 1\n1 3 2\n2 2 3\n1 3 4\n3 1 5\n2 2 6\n", True),
}


def _write(tmp_path, name, text):
    p = tmp_path / f"{name}.mtx"
    p.write_bytes(text.encode())
    return str(p)


def _sorted(coo):
    order = np.lexsort((coo.col, coo.row))  # stable: row, then column
    return coo.row[order], coo.col[order], coo.val[order]


def _same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref/libref_host.so not built (no reference tree on this machine)")
    lib = ctypes.CDLL(REF_SO)
    P = ctypes.c_void_p
    lib.ref_read_mtx.argtypes = [ctypes.c_char_p] + [P] * 6
    lib.ref_read_mtx.restype = None
    lib.ref_free.argtypes = [P]
    lib.ref_store_csr.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
    lib.ref_store_csr.restype = None
    lib.ref_load_csr.argtypes = [ctypes.c_char_p, P, P, P, P, P, P, ctypes.c_int, ctypes.c_int]
    lib.ref_load_csr.restype = ctypes.c_int
    return lib


def _ref_read(lib, path):
    m, n, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rp, cp, vp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    lib.ref_read_mtx(os.fsencode(path), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz),
                     ctypes.byref(rp), ctypes.byref(cp), ctypes.byref(vp))
    k = nnz.value
    out = []
    for ptr, ct, dt in ((rp, ctypes.c_int32, np.int32), (cp, ctypes.c_int32, np.int32),
                        (vp, ctypes.c_float, np.float32)):
        out.append(np.frombuffer((ct * k).from_address(ptr.value), dt).copy() if k else
                   np.zeros(0, dt))
        if ptr.value:
            lib.ref_free(ptr)
    return (m.value, n.value, *out)


@pytest.mark.parametrize("name", sorted(CASES))
def test_read_mtx_matches_oracle(tmp_path, name):
    from spmx import io
    path = _write(tmp_path, name, CASES[name][0])
    A = io.read_mtx(path)
    m, n, row, col, val = orc.mtx_read_sorted(path)
    assert (A.m, A.n) == (m, n)
    r, c, v = _sorted(A)
    assert np.array_equal(r, row) and np.array_equal(c, col) and _same(v, val)


def test_read_mtx_file_order_and_mirrors(tmp_path):
    """Symmetric files: each off-diagonal entry is followed by its mirror."""
    from spmx import io
    A = io.read_mtx(_write(tmp_path, "s", CASES["symmetric_real"][0]))
    assert A.symmetry == "symmetric" and A.field == "real"
    assert A.row.tolist() == [0, 1, 0, 2, 1, 4, 4, 0, 3, 2]
    assert A.col.tolist() == [0, 0, 1, 1, 2, 4, 0, 4, 2, 3]
    assert A.val.tolist() == [2.0, -1.0, -1.0, 0.125, 0.125, 9.0, 1e5, 1e5, -7.75, -7.75]
    S = io.read_mtx(_write(tmp_path, "k", CASES["skew_symmetric"][0]))
    assert S.symmetry == "skew-symmetric" and S.nnz == 2  # not expanded, as in the reference
    C = io.read_mtx(_write(tmp_path, "c", CASES["complex_general"][0]))
    assert C.field == "complex" and C.val.tolist() == [1.0, 1.0, 1.0]


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_readmtx(tmp_path, ref, name):
    text, dups = CASES[name]
    path = _write(tmp_path, name, text)
    got = orc.mtx_read_sorted(path)
    want = _ref_read(ref, path)
    assert got[:2] == want[:2]
    if not dups:
        assert np.array_equal(got[2], want[2]) and np.array_equal(got[3], want[3])
        assert _same(got[4], want[4])
    else:
        key = lambda t: sorted(zip(t[2].tolist(), t[3].tolist(), t[4].tolist()))
        assert key(got) == key(want)
        assert np.array_equal(got[2], want[2]) and np.array_equal(got[3], want[3])


def _big_symmetric(tmp_path, n=100000, per_row=6, seed=3):
    """A multi-chunk file (about 15 MB): lower-triangle entries of a random
    symmetric matrix with values of mixed magnitude, columns unsorted."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(n), per_row)
    cols = (rng.random(rows.size) * (rows + 1)).astype(np.int64)
    vals = (rng.standard_normal(rows.size) * 10.0 ** rng.integers(-8, 8, rows.size)).astype(np.float32)
    p = tmp_path / "big.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n%big\n")
        f.write(f"{n} {n} {rows.size}\n")
        f.write("".join(f"{a + 1} {b + 1} {float(v):.9g}\n" for a, b, v in zip(rows, cols, vals)))
    return str(p)


def test_read_mtx_multi_chunk(tmp_path):
    from spmx import io
    path = _big_symmetric(tmp_path)
    assert os.path.getsize(path) > 3 * (4 << 20)  # several parse chunks
    A = io.read_mtx(path)
    m, n, row, col, val = orc.mtx_read_sorted(path)
    r, c, v = _sorted(A)
    assert A.nnz == row.size and np.array_equal(r, row) and np.array_equal(c, col) and _same(v, val)


def test_read_mtx_multi_chunk_reference(tmp_path, ref):
    path = _big_symmetric(tmp_path, n=20000)
    got = orc.mtx_read_sorted(path)
    want = _ref_read(ref, path)
    # lower-triangle draws can repeat a (row, col): compare as multisets
    assert got[:2] == want[:2]
    assert np.array_equal(got[2], want[2]) and np.array_equal(got[3], want[3])
    o1 = np.lexsort((got[4].view(np.uint32), got[3], got[2]))
    o2 = np.lexsort((want[4].view(np.uint32), want[3], want[2]))
    assert _same(got[4][o1], want[4][o2])


BAD = {
    "no banner": ("3 3 1\n1 1 1\n", 1),
    "array format": ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", 1),
    "unknown symmetry": ("%%MatrixMarket matrix coordinate real upper\n1 1 1\n1 1 1\n", 1),
    "no size line": ("%%MatrixMarket matrix coordinate real general\n% only a comment\n", 2),
    "row index 0": ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n0 2 1\n", 4),
    "column past n": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 1\n", 3),
    "too few entries": ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 1\n", 2),
    "too many entries": ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n2 2 1\n", 2),
    "bad value": ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n2 2 x1\n", 4),
    "missing value": ("%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1\n", 3),
}


@pytest.mark.parametrize("what", sorted(BAD))
def test_read_mtx_rejects_malformed(tmp_path, what):
    from spmx import io, SpmxError
    text, line = BAD[what]
    path = _write(tmp_path, "bad", text)
    with pytest.raises(SpmxError) as e:
        io.read_mtx(path)
    assert f"bad.mtx:{line}:" in str(e.value), str(e.value)


def test_read_mtx_missing_file(tmp_path):
    from spmx import io, SpmxError
    with pytest.raises(SpmxError):
        io.read_mtx(str(tmp_path / "absent.mtx"))


# ---- binary CSR cache -------------------------------------------------------
def _csr(seed=4):
    from conftest import rand_csr
    return rand_csr(700, 500, density=0.01, seed=seed)


def test_csr_cache_round_trip(tmp_path):
    from spmx import io
    A = _csr()
    p = str(tmp_path / "a.csr")
    io.store_csr(p, A)
    B = io.load_csr(p)
    assert (B.m, B.n) == (A.m, A.n)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.col, A.col)
    assert _same(B.val, A.val)
    raw = open(p, "rb").read()
    assert raw[:9] == b"Hola\x01CSR\x01" and len(raw) == 24 + 8 * A.nnz + 4 * (A.m + 1)


def test_csr_cache_against_reference(tmp_path, ref):
    """Files written here load in the reference's loadCSR and the other way
    round; the bytes agree except the 3 padding bytes after the magic."""
    from spmx import io
    A = _csr(seed=6)
    ours, theirs = str(tmp_path / "ours.csr"), str(tmp_path / "theirs.csr")
    io.store_csr(ours, A)
    ref.ref_store_csr(os.fsencode(theirs), A.m, A.n, A.nnz, A.rowptr.ctypes.data,
                      A.col.ctypes.data, A.val.ctypes.data)
    a, b = open(ours, "rb").read(), open(theirs, "rb").read()
    assert len(a) == len(b) and a[:9] == b[:9] and a[12:] == b[12:]
    B = io.load_csr(theirs)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.col, A.col) and _same(B.val, A.val)
    m, n, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rp = np.zeros(A.m + 1, np.int32)
    cl = np.zeros(A.nnz, np.int32)
    vl = np.zeros(A.nnz, np.float32)
    assert ref.ref_load_csr(os.fsencode(ours), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz),
                            rp.ctypes.data, cl.ctypes.data, vl.ctypes.data, A.m, A.nnz) == 0
    assert (m.value, n.value, nnz.value) == (A.m, A.n, A.nnz)
    assert np.array_equal(rp, A.rowptr) and np.array_equal(cl, A.col) and _same(vl, A.val)


def test_csr_cache_errors(tmp_path):
    from spmx import io, abi, SpmxError
    A = _csr()
    p = str(tmp_path / "a.csr")
    io.store_csr(p, A)
    raw = open(p, "rb").read()
    # wrong sizes against the header
    rp = np.zeros(A.m + 2, np.int32)
    cl = np.zeros(A.nnz, np.int32)
    assert abi.lib.spmx_csr_load(os.fsencode(p), A.m + 1, A.n, A.nnz, rp.ctypes.data,
                                 cl.ctypes.data, None) == abi.ERR_INVALID_VALUE
    # values may be skipped
    assert abi.lib.spmx_csr_load(os.fsencode(p), A.m, A.n, A.nnz, rp.ctypes.data,
                                 cl.ctypes.data, None) == 0
    assert np.array_equal(rp[:A.m + 1], A.rowptr) and np.array_equal(cl, A.col)
    bad = tmp_path / "bad.csr"
    bad.write_bytes(b"Hola\x02" + raw[5:])
    with pytest.raises(SpmxError):
        io.load_csr(str(bad))
    short = tmp_path / "short.csr"
    short.write_bytes(raw[:-4])
    with pytest.raises(SpmxError):
        io.load_csr(str(short))


def test_write_mtx_round_trip(tmp_path):
    """write_mtx + read_mtx reproduce a CSR exactly (9 significant digits)."""
    from spmx import io
    A = _csr(seed=9)
    p = str(tmp_path / "w.mtx")
    io.write_mtx(p, A)
    B = io.read_mtx(p)
    assert np.array_equal(B.row, np.repeat(np.arange(A.m), np.diff(A.rowptr)))
    assert np.array_equal(B.col, A.col) and _same(B.val, A.val)


def test_write_mtx_pattern_symmetric(tmp_path):
    """A pattern triangle written as "symmetric" reads back expanded, and the
    writer rejects an index outside the matrix."""
    from spmx import io, SpmxError
    from spmx.gen import Csr
    rng = np.random.default_rng(21)
    r = rng.integers(0, 300, 2000).astype(np.int32)
    c = (rng.random(2000) * (r + 1)).astype(np.int32)  # lower triangle, diagonal included
    p = str(tmp_path / "p.mtx")
    io.write_mtx(p, Csr(300, 300, np.zeros(301, np.int32), np.zeros(0, np.int32), None),
                 symmetry="symmetric")
    assert io.read_mtx(p).nnz == 0
    coo = io.Coo(300, 300, r, c, np.ones(2000, np.float32))
    coo.val = None
    io.write_mtx(p, coo, symmetry="symmetric")
    B = io.read_mtx(p)
    assert B.field == "pattern" and B.symmetry == "symmetric"
    m, n, row, col, val = orc.mtx_read_sorted(p)
    rr, cc, vv = _sorted(B)
    assert np.array_equal(rr, row) and np.array_equal(cc, col) and _same(vv, val)
    assert B.nnz == 2 * 2000 - int(np.sum(r == c))
    coo.col = coo.col.copy()
    coo.col[5] = 300
    with pytest.raises(SpmxError):
        io.write_mtx(p, coo)
