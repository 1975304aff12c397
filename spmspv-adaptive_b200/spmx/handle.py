"""SpmspvHandle: the reference's engine handle, over the spmx C ABI.

Method names, argument meaning and ownership follow SpmspvHandle<int,
unsigned, float> (hice-spmspv/hice/la/include/spmspv/csc-spmspv/spmspv.h,
H:88-344): CSR and x buffers are caller-owned device tensors (the handle keeps
a reference so they outlive it), CSC / Hola / CSR5 tables and scratch belong
to the handle.  Differences from the reference:

- methods return None and raise SpmxError on failure (the reference returns
  SPMSPV_* codes, prints, or exits);
- y_nnz outputs are returned as Python ints;
- alpha scales the result (y = alpha*A*x), as the reference's CPU
  serialspmv does; its GPU kernels ignore alpha, which coincides for 1.0.

All tensors must be CUDA tensors: int32 indices, float32 values.  Work runs on
torch's current CUDA stream at construction time (set_stream changes it).
"""
import ctypes

import torch

from . import _lib
from ._lib import lib, check, c_int, c_ll, c_double, c_float, c_void_p


def _ptr(t):
    if t is None:
        return None
    if not isinstance(t, torch.Tensor):
        raise TypeError("expected a torch tensor")
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _i32(t):
    if t is not None and t.dtype != torch.int32:
        raise TypeError("index tensors must be int32")
    return _ptr(t)


def _f32(t):
    if t is not None and t.dtype != torch.float32:
        raise TypeError("value tensors must be float32")
    return _ptr(t)


class SpmspvHandle:
    def __init__(self, m, n, nnz, stream=None):
        h = c_void_p()
        check(lib.spmx_create(int(m), int(n), int(nnz), ctypes.byref(h)), "create")
        self._h = h
        self.m, self.n, self.nnz = int(m), int(n), int(nnz)
        self._keep = {}
        s = stream if stream is not None else torch.cuda.current_stream()
        self.set_stream(s)

    # -- lifecycle -----------------------------------------------------------
    def set_stream(self, stream):
        self._stream = stream
        check(lib.spmx_set_stream(self._h, stream.cuda_stream), "set_stream")

    def warmup(self):
        check(lib.spmx_warmup(self._h), "warmup")

    def Destroy(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.spmx_destroy(self._h)
            self._h = c_void_p()
        self._keep = {}

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass

    def check_device_error(self):
        check(lib.spmx_check_device_error(self._h), "device")

    @property
    def raw(self):
        """The C handle (for callers that use the C ABI directly)."""
        return self._h

    # -- matrix --------------------------------------------------------------
    def InputCSR(self, nnz, csr_row, csr_col, csr_val=None):
        check(lib.spmx_input_csr(self._h, int(nnz), _i32(csr_row), _i32(csr_col), _f32(csr_val)),
              "InputCSR")
        self._keep["csr"] = (csr_row, csr_col, csr_val)

    def InputCSC(self, nnz, csc_row, csc_col, csc_val=None):
        check(lib.spmx_input_csc(self._h, int(nnz), _i32(csc_row), _i32(csc_col), _f32(csc_val)),
              "InputCSC")
        self._keep["csc"] = (csc_row, csc_col, csc_val)

    def InputCOO(self, nnz, row, col, val=None):
        """COO device arrays (any order) -> handle-owned CSR sorted by (row, col).
        Synchronous; the inputs are not kept."""
        check(lib.spmx_input_coo(self._h, int(nnz), _i32(row), _i32(col), _f32(val)), "InputCOO")
        self._keep.pop("csr", None)

    def get_csr(self):
        """(rowptr[m+1], col[nnz], val[nnz]) copied into new tensors (val is
        left unwritten for a pattern-only matrix)."""
        rowptr = torch.empty(self.m + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(self.nnz, dtype=torch.int32, device="cuda")
        val = torch.empty(self.nnz, dtype=torch.float32, device="cuda")
        check(lib.spmx_copy_csr(self._h, _ptr(rowptr), _ptr(col) if self.nnz else None,
                                _ptr(val) if self.nnz else None), "copy_csr")
        self._stream.synchronize()
        return rowptr, col, val

    # -- hybrid CSR/CSC split (a candidate ninth kernel) ------------------------
    def hybridPreprocess(self):
        check(lib.spmx_hybrid_preprocess(self._h), "hybridPreprocess")

    def hybridPostprocess(self):
        check(lib.spmx_hybrid_postprocess(self._h), "hybridPostprocess")

    def hybrid_info(self):
        """(nonzeros in the CSR part, nonzeros in the CSC part)"""
        a, b = c_int(), c_int()
        check(lib.spmx_hybrid_info(self._h, ctypes.byref(a), ctypes.byref(b)), "hybrid_info")
        return a.value, b.value

    def hybrid_parts(self):
        """((rowptr, col, val) of the CSR part, (colptr, row, val) of the CSC
        part) copied into new tensors."""
        a, b = self.hybrid_info()
        i32 = dict(dtype=torch.int32, device="cuda")
        rp, cl, vl = (torch.empty(self.m + 1, **i32), torch.empty(max(a, 1), **i32),
                      torch.empty(max(a, 1), device="cuda"))
        cp, rw, cv = (torch.empty(self.n + 1, **i32), torch.empty(max(b, 1), **i32),
                      torch.empty(max(b, 1), device="cuda"))
        check(lib.spmx_hybrid_copy(self._h, _ptr(rp), _ptr(cl), _ptr(vl), _ptr(cp), _ptr(rw),
                                   _ptr(cv)), "hybrid_copy")
        self._stream.synchronize()
        return (rp, cl[:a], vl[:a]), (cp, rw[:b], cv[:b])

    def hybridspmv(self, alpha, y):
        check(lib.spmx_hybridspmv(self._h, float(alpha), _f32(y)), "hybridspmv")

    def ToCSC(self):
        check(lib.spmx_to_csc(self._h), "ToCSC")

    def get_csc(self):
        """(row[nnz], colptr[n+1], val[nnz]) copied into new tensors."""
        row = torch.empty(self.nnz, dtype=torch.int32, device="cuda")
        colptr = torch.empty(self.n + 1, dtype=torch.int32, device="cuda")
        val = torch.empty(self.nnz, dtype=torch.float32, device="cuda")
        check(lib.spmx_copy_csc(self._h, _ptr(row) if self.nnz else None, _ptr(colptr),
                                _ptr(val) if self.nnz else None), "copy_csc")
        self._stream.synchronize()
        return row, colptr, val

    # -- vectors -------------------------------------------------------------
    def set_x(self, x):
        check(lib.spmx_set_x(self._h, _f32(x)), "set_x")
        self._keep["x"] = x

    def set_sparse_x(self, x_key, x_val, xnnz):
        check(lib.spmx_set_sparse_x(self._h, _i32(x_key), _f32(x_val), int(xnnz)), "set_sparse_x")
        self._keep["xs"] = (x_key, x_val)

    def set_bitvector(self, bitvector, num_ints):
        check(lib.spmx_set_bitvector(self._h, _i32(bitvector), int(num_ints)), "set_bitvector")
        self._keep["bits"] = bitvector

    def set_sparse_x_dense_x(self, x_key, x_val, x_dense, xnnz):
        check(lib.spmx_set_sparse_x_dense_x(self._h, _i32(x_key), _f32(x_val), _f32(x_dense),
                                            int(xnnz)), "set_sparse_x_dense_x")
        self._keep["xs"] = (x_key, x_val)
        self._keep["x"] = x_dense

    def set_vector_type(self, code):
        check(lib.spmx_set_vector_type(self._h, int(code)), "set_vector_type")

    def sparse2dense(self):
        check(lib.spmx_sparse2dense(self._h), "sparse2dense")

    def sparse2bitarray(self):
        check(lib.spmx_sparse2bitarray(self._h), "sparse2bitarray")

    def dense2sparse(self):
        n = c_int()
        check(lib.spmx_dense2sparse(self._h, ctypes.byref(n)), "dense2sparse")
        return n.value

    def bitarray2sparse(self):
        n = c_int()
        check(lib.spmx_bitarray2sparse(self._h, ctypes.byref(n)), "bitarray2sparse")
        return n.value

    def dense2bitarray(self):
        check(lib.spmx_dense2bitarray(self._h), "dense2bitarray")

    def dense2sparse_outer(self, m, d_dense, d_key, d_val):
        n = c_int()
        check(lib.spmx_dense2sparse_outer(self._h, int(m), _f32(d_dense), ctypes.byref(n),
                                          _i32(d_key), _f32(d_val)), "dense2sparse_outer")
        return n.value

    def dense2sparse_to_host(self, m, d_dense, h_key, h_val, h_count):
        """Nonzeros of d_dense[:m] into pinned host tensors h_key / h_val and
        their count into h_count[0] (pinned int32), without synchronising:
        read them after the stream has passed this call."""
        for t, dt in ((h_key, torch.int32), (h_val, torch.float32), (h_count, torch.int32)):
            if t.is_cuda or not t.is_pinned():
                raise ValueError("h_key, h_val and h_count must be pinned host tensors")
            if t.dtype != dt:
                raise TypeError("h_key / h_count must be int32 and h_val float32")
        check(lib.spmx_dense2sparse_to_host(self._h, int(m), _f32(d_dense), h_key.data_ptr(),
                                            h_val.data_ptr(), h_count.data_ptr()),
              "dense2sparse_to_host")

    def sparse2dense_outer(self, ynnz, d_key, d_val, m, d_dense):
        check(lib.spmx_sparse2dense_outer(self._h, int(ynnz), _i32(d_key), _f32(d_val), int(m),
                                          _f32(d_dense)), "sparse2dense_outer")

    # -- scratch / preprocess ----------------------------------------------------
    def allocPreBuffer(self):
        check(lib.spmx_alloc_pre_buffer(self._h), "allocPreBuffer")

    def deallocPreBuffer(self):
        check(lib.spmx_dealloc_pre_buffer(self._h), "deallocPreBuffer")

    def holaPreprocess(self):
        check(lib.spmx_hola_preprocess(self._h), "holaPreprocess")

    def holaPostprocess(self):
        check(lib.spmx_hola_postprocess(self._h), "holaPostprocess")

    def setSigma(self, sigma):
        check(lib.spmx_set_sigma(self._h, int(sigma)), "setSigma")

    def CSR5Preprocess(self):
        check(lib.spmx_csr5_preprocess(self._h), "CSR5Preprocess")

    def CSR5Postprocess(self):
        check(lib.spmx_csr5_postprocess(self._h), "CSR5Postprocess")

    def tiledPreprocess(self, rb_rows=0, win=0, chunk=0, warps=0):
        check(lib.spmx_tiled_preprocess(self._h, int(rb_rows), int(win), int(chunk), int(warps)),
              "tiledPreprocess")

    def tiledPostprocess(self):
        check(lib.spmx_tiled_postprocess(self._h), "tiledPostprocess")

    def tiled_info(self):
        """Geometry of the tiled format: row blocks, CTAs per cluster, stages,
        window, chunk, shared y rows, shared bytes, row warps."""
        info = (ctypes.c_int * 8)()
        check(lib.spmx_tiled_info(self._h, info), "tiled_info")
        names = ("row_blocks", "cluster", "stages", "win", "chunk", "rmax", "smem", "warps")
        return dict(zip(names, list(info)))

    def tiledspmv(self, alpha, y):
        check(lib.spmx_tiledspmv(self._h, float(alpha), _f32(y)), "tiledspmv")

    def tiledspmspv(self, alpha, y):
        check(lib.spmx_tiledspmspv(self._h, float(alpha), _f32(y)), "tiledspmspv")

    def roundPreprocess(self, rb_rows=0, parts=1):
        """Round format with `parts` CTAs per row block (1: one CTA per row
        block, no cluster; 2: a 2-CTA cluster over row blocks twice as tall;
        4: two clusters over row blocks four times as tall)."""
        if parts == 1:
            check(lib.spmx_round_preprocess(self._h, int(rb_rows)), "roundPreprocess")
        else:
            check(lib.spmx_round_preprocess_parts(self._h, int(rb_rows), int(parts)), "roundPreprocess")

    def roundPostprocess(self):
        check(lib.spmx_round_postprocess(self._h), "roundPostprocess")

    def round_info(self):
        """Geometry of the round format: row blocks, CTAs per row block, rounds,
        nonzeros per round, accumulator slots per CTA, shared y rows, shared
        bytes, grid."""
        info = (ctypes.c_int * 8)()
        check(lib.spmx_round_info(self._h, info), "round_info")
        names = ("row_blocks", "parts", "rounds", "round", "slots", "rmax", "smem", "grid")
        return dict(zip(names, list(info)))

    def roundspmv(self, alpha, y):
        check(lib.spmx_roundspmv(self._h, float(alpha), _f32(y)), "roundspmv")

    def roundspmspv(self, alpha, y):
        check(lib.spmx_roundspmspv(self._h, float(alpha), _f32(y)), "roundspmspv")

    def set_spmv_type(self, code):
        check(lib.spmx_set_spmv_type(self._h, int(code)), "set_spmv_type")

    # -- SpMV / CSR SpMSpV ---------------------------------------------------------
    def naivespmv(self, alpha, y):
        check(lib.spmx_naivespmv(self._h, float(alpha), _f32(y)), "naivespmv")

    def holaspmv(self, alpha, y):
        check(lib.spmx_holaspmv(self._h, float(alpha), _f32(y)), "holaspmv")

    def csr5spmv(self, alpha, y):
        check(lib.spmx_csr5spmv(self._h, float(alpha), _f32(y)), "csr5spmv")

    def naivespmspv(self, alpha, y):
        check(lib.spmx_naivespmspv(self._h, float(alpha), _f32(y)), "naivespmspv")

    def holaspmspv(self, alpha, y):
        check(lib.spmx_holaspmspv(self._h, float(alpha), _f32(y)), "holaspmspv")

    def csr5spmspv(self, alpha, y):
        check(lib.spmx_csr5spmspv(self._h, float(alpha), _f32(y)), "csr5spmspv")

    def spmv(self, alpha, y):
        check(lib.spmx_spmv(self._h, float(alpha), _f32(y)), "spmv")

    def spmspv(self, alpha, y):
        check(lib.spmx_spmspv(self._h, float(alpha), _f32(y)), "spmspv")

    # -- CSC SpMSpV (reference names) --------------------------------------------------
    def spmspv_csc(self, variant, writeback, alpha, y=None, y_key=None, y_val=None, sync=True):
        n = c_int()
        check(lib.spmx_spmspv_csc(self._h, int(variant), int(writeback), float(alpha), _f32(y),
                                  _i32(y_key), _f32(y_val), ctypes.byref(n) if sync else None),
              "spmspv_csc")
        return n.value if sync else None

    def CscBasedNoSortNaiveSpmspv(self, alpha, y):
        n = c_int()
        check(lib.spmx_csc_naive_atomic(self._h, float(alpha), ctypes.byref(n), _f32(y)),
              "CscBasedNoSortNaiveSpmspv")
        return n.value

    def CscBasedNoSortNaiveSpmspv_keyval(self, alpha, y, y_key, y_val):
        n = c_int()
        check(lib.spmx_csc_naive_atomic_keyval(self._h, float(alpha), ctypes.byref(n), _f32(y),
                                               _i32(y_key), _f32(y_val)),
              "CscBasedNoSortNaiveSpmspv_keyval")
        return n.value

    def CscBasedSortNaiveSpmspv(self, alpha, y_key, y_val):
        n = c_int()
        check(lib.spmx_csc_naive_sort(self._h, float(alpha), ctypes.byref(n), _i32(y_key),
                                      _f32(y_val)), "CscBasedSortNaiveSpmspv")
        return n.value

    def _lb(self, fn, name, alpha, y, y_key, y_val):
        n = c_int()
        check(fn(self._h, 1, float(alpha), ctypes.byref(n), _f32(y), _i32(y_key), _f32(y_val)), name)
        return n.value

    def CscBasedNoSortMergeSpmspv(self, IsBinLenComputed, alpha, y, y_key=None, y_val=None):
        return self._lb(lib.spmx_csc_merge_atomic, "CscBasedNoSortMergeSpmspv", alpha, y, None, None)

    def CscBasedNoSortMergeSpmspv_keyval(self, IsBinLenComputed, alpha, y, y_key, y_val):
        return self._lb(lib.spmx_csc_merge_atomic_keyval, "CscBasedNoSortMergeSpmspv_keyval",
                        alpha, y, y_key, y_val)

    def CscBasedSortMergeSpmspv(self, IsBinLenComputed, alpha, y, y_key, y_val):
        return self._lb(lib.spmx_csc_merge_sort, "CscBasedSortMergeSpmspv", alpha, y, y_key, y_val)

    def CscBasedMyNoSortSpmspv(self, IsBinLenComputed, alpha, y, y_key=None, y_val=None):
        return self._lb(lib.spmx_csc_twolayer_atomic, "CscBasedMyNoSortSpmspv", alpha, y, None, None)

    def CscBasedMyNoSortSpmspv_keyval(self, IsBinLenComputed, alpha, y, y_key, y_val):
        return self._lb(lib.spmx_csc_twolayer_atomic_keyval, "CscBasedMyNoSortSpmspv_keyval",
                        alpha, y, y_key, y_val)

    def CscBasedSortMySpmspv(self, IsBinLenComputed, alpha, y, y_key, y_val):
        return self._lb(lib.spmx_csc_twolayer_sort, "CscBasedSortMySpmspv", alpha, y, y_key, y_val)

    def CscBasedBucketSpmspv(self, alpha, y=None, y_key=None, y_val=None, buckets=0):
        n = c_int()
        check(lib.spmx_csc_bucket(self._h, float(alpha), ctypes.byref(n), _f32(y), _i32(y_key),
                                  _f32(y_val), int(buckets)), "CscBasedBucketSpmspv")
        return n.value

    # -- features / selector -------------------------------------------------------------
    def computeBinlenVer2(self):
        v = c_ll()
        check(lib.spmx_compute_binlen(self._h, ctypes.byref(v)), "computeBinlenVer2")
        return v.value

    def computeGM(self):
        gm = (c_double * 3)()
        check(lib.spmx_compute_gm(self._h, gm), "computeGM")
        return list(gm)

    def computeGM1(self):
        return self.computeGM()[0]

    def computeGM2(self):
        return self.computeGM()[1]

    def computeGM3(self):
        return self.computeGM()[2]

    def computeMatFeture(self):
        """{m, n, nnz, max, min, avg, range, stdRow, edge_equlity, gini}"""
        out = (c_double * 10)()
        check(lib.spmx_mat_features(self._h, out), "computeMatFeture")
        return list(out)

    def extractMatFeatureParallel(self):
        v = c_float()
        check(lib.spmx_std_row(self._h, ctypes.byref(v)), "extractMatFeatureParallel")
        return v.value

    def computeVecFeture(self):
        """(bin_len, max, min) of the column lengths of x's keys"""
        out = (c_ll * 3)()
        check(lib.spmx_vec_features(self._h, out), "computeVecFeture")
        return tuple(out)

    def features(self):
        out = (c_double * _lib.NUM_FEATURES)()
        check(lib.spmx_features(self._h, out), "features")
        return dict(zip(_lib.FEATURE_NAMES, list(out)))

    def selector_inputs(self):
        out = (c_double * _lib.NUM_FEATURES)()
        check(lib.spmx_selector_inputs(self._h, out), "selector_inputs")
        return list(out)

    def select(self):
        k = c_int()
        check(lib.spmx_select(self._h, ctypes.byref(k)), "select")
        return k.value

    def run_adaptive(self, alpha, y):
        k = c_int()
        check(lib.spmx_run_adaptive(self._h, float(alpha), _f32(y), ctypes.byref(k)), "run_adaptive")
        return k.value

    def autotune(self, cache_path=None):
        """Time the tunable choices on this matrix and keep the fastest;
        returns the chosen SpMV back-end (0 Hola, 1 CSR5, 2 tiled, 3 round)."""
        t = c_int()
        check(lib.spmx_autotune(self._h, cache_path.encode() if cache_path else None,
                                ctypes.byref(t)), "autotune")
        return t.value

    def set_naive_lanes(self, row_lanes=0, col_lanes=0):
        """Lanes per row / column of the naive kernels (0: from the mean
        length; else 1, 2, 4, 8, 16 or 32), as the autotuner sets them."""
        check(lib.spmx_set_naive_lanes(self._h, int(row_lanes), int(col_lanes)), "set_naive_lanes")

    def run_kernel(self, kid, alpha, y):
        check(lib.spmx_run_kernel(self._h, int(kid), float(alpha), _f32(y)), "run_kernel")

    # -- adjoint -----------------------------------------------------------------------
    def spmv_backward(self, x, dy, dx=None, dvals=None):
        check(lib.spmx_spmv_backward(self._h, _f32(x), _f32(dy), _f32(dx), _f32(dvals)),
              "spmv_backward")

    def spmv_backward_sparse(self, x, dy_key, dy_val, dy_nnz, dx=None, dvals=None):
        check(lib.spmx_spmv_backward_sparse(self._h, _f32(x), _i32(dy_key), _f32(dy_val),
                                            int(dy_nnz), _f32(dx), _f32(dvals)),
              "spmv_backward_sparse")

    # -- batched SpMSpV (no reference counterpart) ------------------------------
    def set_batch_options(self, flags):
        """SPMX_BATCH_REUSE_INVERSION (1) | SPMX_BATCH_FUSED_DXVAL (2); 0 = none."""
        check(lib.spmx_set_batch_options(self._h, int(flags)), "set_batch_options")

    def spmspv_batched(self, xptr, xkey, xval, alpha, Y, x_total=None):
        """Y = alpha * A @ X for the nvec = len(xptr) - 1 sparse vectors of the
        concatenated (xkey, xval); Y is (m, nvec) float32 on the device.
        x_total (= xptr[-1]) is read back from xptr when not given."""
        nvec = int(xptr.numel()) - 1
        if x_total is None:
            x_total = int(xptr[-1].item())
        check(lib.spmx_spmspv_batched(self._h, nvec, int(x_total), _i32(xptr), _i32(xkey), _f32(xval),
                                      float(alpha), _f32(Y)), "spmspv_batched")

    def spmspv_batched_backward(self, xptr, xkey, xval, alpha, dY, dxval=None, dvals=None, x_total=None):
        """dxval (layout of xval) and dvals (CSR order) for an upstream dY (m, nvec)."""
        nvec = int(xptr.numel()) - 1
        if x_total is None:
            x_total = int(xptr[-1].item())
        check(lib.spmx_spmspv_batched_backward(self._h, nvec, int(x_total), _i32(xptr), _i32(xkey),
                                               _f32(xval), float(alpha), _f32(dY), _f32(dxval),
                                               _f32(dvals)), "spmspv_batched_backward")

    # -- BFS ---------------------------------------------------------------------------
    def bfs(self, source, levels, sync=True):
        """Levels of a BFS from `source` into `levels` (int32 [n]); returns the
        number of levels (reads it back) unless sync=False."""
        d = c_int()
        check(lib.spmx_bfs(self._h, int(source), _i32(levels), ctypes.byref(d) if sync else None),
              "bfs")
        return d.value if sync else None

    def set_bfs_mode(self, mode):
        check(lib.spmx_set_bfs_mode(self._h, int(mode)), "set_bfs_mode")

    def bfs_batched(self, sources, levels, layout=1, sync=True):
        """Up to 64 sources in one launch; levels is [n*len(sources)] int32
        (layout 1: source-major [s][v]; layout 0: vertex-major [v][s])."""
        src = (c_int * len(sources))(*[int(s) for s in sources])
        d = c_int()
        check(lib.spmx_bfs_batched(self._h, src, len(sources), _i32(levels), int(layout),
                                   ctypes.byref(d) if sync else None), "bfs_batched")
        return d.value if sync else None
