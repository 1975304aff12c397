"""The CPU oracle against hand-derived known answers and independent numpy
restatements (no GPU)."""
import json
import os

import numpy as np
import pytest

from conftest import rand_csr, sym_graph
import oracle.oracle as orc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_kat():
    with open(os.path.join(GOLDEN, "kat_small.json")) as f:
        return json.load(f)


def test_kat_spmv_and_spmspv():
    k = load_kat()
    A = k["matrix"]
    rowptr, col, val = np.array(A["rowptr"]), np.array(A["col"]), np.array(A["val"], np.float32)
    x = np.array(k["x_dense"], np.float32)
    y, mag = orc.spmv_f64(rowptr, col, val, x, alpha=k["alpha"])
    assert np.allclose(y, k["y_spmv"], rtol=0, atol=1e-12)
    # faithful FP32 serialspmv reproduces the same small-integer results exactly
    y32 = orc.serialspmv_f32(rowptr, col, val, x, alpha=k["alpha"])
    assert np.array_equal(y32, np.array(k["y_spmv"], np.float32))
    # CSC SpMSpV with the sparse x
    from spmx.gen import Csr
    colptr, row, cval = Csr(A["m"], A["n"], rowptr, col, val).to_csc()
    assert colptr.tolist() == A["csc_colptr"] and row.tolist() == A["csc_row"]
    ys, _, touched = orc.spmspv_csc_f64(A["m"], colptr, row, cval, k["x_key"], k["x_val"],
                                        alpha=k["alpha"])
    assert np.allclose(ys, k["y_spmv"], atol=1e-12)
    assert touched.nonzero()[0].tolist() == k["touched_rows"]
    key, v = orc.dense2sparse(ys.astype(np.float32))
    assert key.tolist() == k["y_nonzero_rows"]


def test_kat_features():
    k = load_kat()
    A = k["matrix"]
    f = orc.mat_features(A["n"], np.array(A["rowptr"]))
    for name, idx in (("max", 3), ("min", 4), ("avg", 5), ("range", 6), ("stdRow", 7),
                      ("edge_equlity", 8), ("gini", 9)):
        assert f[idx] == pytest.approx(k["mat_features"][name], rel=1e-12, abs=1e-12), name
    v = orc.vec_features(np.array(A["csc_colptr"]), np.array(k["x_key"]))
    assert v.tolist() == k["vec_features"]
    assert orc.gm(A["m"], A["nnz"], len(k["x_key"]), v[0]).tolist() == pytest.approx(k["gm"])


def test_kat_bfs():
    k = load_kat()["bfs"]
    g = sym_graph(k["n"], k["edges"])
    colptr, row, _ = g.to_csc()
    lv, depth = orc.bfs_spmspv(k["n"], colptr, row, k["source"])
    assert lv.tolist() == k["levels"] and depth == k["depth"]
    lq, dq = orc.bfs_queue(k["n"], g.rowptr, g.col, k["source"])
    assert lq.tolist() == k["levels"] and dq == k["depth"]


def test_sigma_rule():
    # setSigma auto rule: <=4 -> 4, <=32 -> nnz/row, <=256 -> 32, else 6
    assert orc.csr5_sigma(100, 300) == 4
    assert orc.csr5_sigma(100, 1700) == 17
    assert orc.csr5_sigma(100, 10000) == 32
    assert orc.csr5_sigma(100, 100000) == 6


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_spmv_matches_dense_numpy(seed):
    A = rand_csr(300, 250, density=0.05, seed=seed)
    x = np.random.default_rng(seed).uniform(-1, 1, 250).astype(np.float32)
    D = np.zeros((300, 250))
    for i in range(300):
        D[i, A.col[A.rowptr[i]:A.rowptr[i + 1]]] = A.val[A.rowptr[i]:A.rowptr[i + 1]]
    y, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=0.5)
    assert np.allclose(y, 0.5 * D @ x.astype(np.float64), atol=1e-12)
    assert np.allclose(mag, 0.5 * np.abs(D) @ np.abs(x.astype(np.float64)), atol=1e-12)


@pytest.mark.parametrize("seed", [0, 3])
def test_spmspv_csc_matches_spmv(seed):
    A = rand_csr(400, 500, density=0.02, seed=seed)
    colptr, row, cval = A.to_csc()
    rng = np.random.default_rng(seed)
    key = np.sort(rng.choice(500, 37, replace=False)).astype(np.int32)
    xv = rng.uniform(-1, 1, 37).astype(np.float32)
    xd, bits = orc.sparse2dense_bits(500, key, xv)
    y1, _, touched = orc.spmspv_csc_f64(400, colptr, row, cval, key, xv, alpha=2.0)
    y2, _ = orc.spmv_f64(A.rowptr, A.col, A.val, xd, alpha=2.0)
    assert np.allclose(y1, y2, atol=1e-12)
    # the bitarray gate selects exactly the keys
    y3, _ = orc.spmv_f64(A.rowptr, A.col, A.val, np.ones(500, np.float32) * 0 + xd, bits=bits.view(np.int32), alpha=2.0)
    assert np.allclose(y3, y2, atol=1e-12)
    # structural output = rows that appear in any selected column
    exp = np.zeros(400, bool)
    for c in key:
        exp[row[colptr[c]:colptr[c + 1]]] = True
    assert np.array_equal(touched, exp)


def test_vector_conversions():
    rng = np.random.default_rng(5)
    d = rng.uniform(-1, 1, 1000).astype(np.float32)
    d[rng.random(1000) < 0.7] = 0
    key, val = orc.dense2sparse(d)
    assert np.array_equal(key, np.nonzero(d)[0]) and np.array_equal(val, d[key])
    bits = orc.dense2bitarray(d)
    unpacked = np.unpackbits(bits.view(np.uint8), bitorder="little")[:1000].astype(bool)
    assert np.array_equal(unpacked, d != 0)
    d2, b2 = orc.sparse2dense_bits(1000, key, val)
    assert np.array_equal(d2, d) and np.array_equal(b2, bits)


def test_features_match_numpy():
    A = rand_csr(2000, 1500, lens=np.random.default_rng(1).zipf(2.0, 2000) % 300, seed=1)
    f = orc.mat_features(A.n, A.rowptr)
    d = np.diff(A.rowptr).astype(np.float64)
    m, nnz = A.m, A.nnz
    avg = float(np.float32(nnz) / np.float32(m))
    assert f[3] == d.max() and f[4] == d.min() and f[5] == pytest.approx(avg)
    assert f[7] == pytest.approx(np.sqrt(np.mean((d - avg) ** 2)), rel=1e-12)
    p = d[d > 0] / nnz
    assert f[8] == pytest.approx(-(p * np.log(p)).sum() / np.log(m), rel=1e-12)
    s = np.sort(d)
    s1 = float(np.sum(np.arange(1, m) * s[1:]))
    s2 = float(np.sum(s[:-1]))
    assert f[9] == pytest.approx(abs(2 * s1 / (m * s2) - (m + 1) / m), rel=1e-12)
    # the reference's float accumulators drift from the exact values but stay close
    ff = orc.mat_features_faithful(A.n, A.rowptr)
    assert ff[4] == pytest.approx(f[7], rel=1e-4) and ff[6] == pytest.approx(f[9], rel=1e-3)
    # stdRow of extractMatFeature truncates the mean to int
    ai = int(np.float32(nnz) / np.float32(m))
    assert orc.std_row_intmean(A.rowptr) == pytest.approx(np.sqrt(np.mean((d - ai) ** 2)))


def test_bfs_oracles_agree_on_rmat():
    from spmx import gen
    g = gen.rmat(12, 16, seed=11)
    colptr, row, _ = g.to_csc()
    for src in (0, 5, 1000):
        a, da = orc.bfs_spmspv(g.n, colptr, row, src)
        b, db = orc.bfs_queue(g.n, g.rowptr, g.col, src)
        assert np.array_equal(a, b) and da == db


def test_adjoint_oracles():
    A = rand_csr(50, 40, density=0.2, seed=9)
    rng = np.random.default_rng(9)
    dy = rng.normal(size=50).astype(np.float32)
    x = rng.normal(size=40).astype(np.float32)
    D = np.zeros((50, 40))
    for i in range(50):
        D[i, A.col[A.rowptr[i]:A.rowptr[i + 1]]] = A.val[A.rowptr[i]:A.rowptr[i + 1]]
    dx, _ = orc.spmv_t_f64(40, A.rowptr, A.col, A.val, dy)
    assert np.allclose(dx, D.T @ dy.astype(np.float64), atol=1e-12)
    dv = orc.dvals_f64(A.rowptr, A.col, dy, x)
    exp = np.concatenate([dy[i] * x[A.col[A.rowptr[i]:A.rowptr[i + 1]]].astype(np.float64)
                          for i in range(50)])
    assert np.allclose(dv, exp, atol=1e-12)


def test_within_tol_is_strict():
    y64 = np.array([1.0, 0.0, -2.0])
    mag = np.array([1.0, 0.0, 4.0])
    ok, _ = orc.within_tol(np.array([1.0 + 5e-6, 0.0, -2.0]), y64, mag)
    assert ok
    bad, _ = orc.within_tol(np.array([1.0, 1e-30, -2.0]), y64, mag)
    assert not bad   # an untouched row must be exactly zero
