"""ctypes binding of libspmx.so (the C ABI declared in include/spmx.h).

The shared library is built in-tree by ``make -C spmspv-adaptive_b200/csrc``
(``__graft_entry__.build()`` does this).  There is no fallback: importing this
module without the library raises ImportError, and every entry point that
needs a GPU returns SPMX_ERR_NO_DEVICE when none is visible.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspmx.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libspmx.so not found at {LIB_PATH}; build it with "
        "`make -C spmspv-adaptive_b200/csrc` (or __graft_entry__.build())")

lib = ctypes.CDLL(LIB_PATH)

c_int, c_float, c_double, c_ll = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_longlong
c_void_p, c_u64 = ctypes.c_void_p, ctypes.c_uint64
P = c_void_p            # device or host pointer passed as an integer
PI = ctypes.POINTER(c_int)
PLL = ctypes.POINTER(c_ll)
PD = ctypes.POINTER(c_double)
PF = ctypes.POINTER(c_float)
PP = ctypes.POINTER(c_void_p)

# status codes (include/spmx.h)
SUCCESS = 0
ERR_INVALID_VALUE = -20
ERR_CUDA = -21
ERR_TIMEOUT = -22
ERR_OOB = -23
ERR_ALLOC = -24
ERR_NOT_READY = -25
ERR_NO_DEVICE = -26

VEC_SPARSE, VEC_DENSE, VEC_BITARRAY = 0, 1, 2
SPMV_HOLA, SPMV_CSR5, SPMV_TILED, SPMV_ROUND = 0, 1, 2, 3
CSC_NAIVE, CSC_LB_MERGE, CSC_LB_TWOLAYER, CSC_BUCKET = 0, 1, 2, 3
WB_ATOMIC, WB_SORT = 0, 1
BATCH_REUSE_INVERSION, BATCH_FUSED_DXVAL = 1, 2
(K_CSC_NAIVE_SORT, K_CSC_NAIVE_ATOMIC, K_CSC_LB_SORT, K_CSC_LB_ATOMIC,
 K_CSR_NAIVE_SPMSPV, K_CSR_LB_SPMSPV, K_NAIVE_SPMV, K_LB_SPMV) = range(8)
NUM_KERNELS = 8
KERNEL_NAMES = ["csc-naive-sort", "csc-naive-atomic", "csc-lb-sort", "csc-lb-atomic",
                "csr-naive-spmspv", "csr-lb-spmspv", "naive-spmv", "lb-spmv"]
NUM_FEATURES = 23
FEATURE_NAMES = ("m,n,nnz,maxRow,minRow,avgRow,range,stdRow,edge_equlity,gini_coefficiency,"
                 "x_nnz,bin_len,max,min,xnnz/n,bin_len/nnz,xnnz_range,GM1,GM2,GM3,GM1/GM2,"
                 "GM2/GM3,GM1/GM3").split(",")

# name -> (restype, argtypes)
_SIGS = {
    "spmx_create": (c_int, [c_int, c_int, c_int, PP]),
    "spmx_destroy": (c_int, [P]),
    "spmx_set_stream": (c_int, [P, P]),
    "spmx_warmup": (c_int, [P]),
    "spmx_last_error_string": (ctypes.c_char_p, []),
    "spmx_launch_count": (ctypes.c_ulonglong, []),
    "spmx_check_device_error": (c_int, [P]),
    "spmx_input_csr": (c_int, [P, c_int, P, P, P]),
    "spmx_input_csc": (c_int, [P, c_int, P, P, P]),
    "spmx_to_csc": (c_int, [P]),
    "spmx_get_csc": (c_int, [P, PP, PP, PP]),
    "spmx_copy_csc": (c_int, [P, P, P, P]),
    "spmx_input_coo": (c_int, [P, c_int, P, P, P]),
    "spmx_hybrid_preprocess": (c_int, [P]),
    "spmx_hybrid_postprocess": (c_int, [P]),
    "spmx_hybrid_info": (c_int, [P, PI, PI]),
    "spmx_hybrid_copy": (c_int, [P, P, P, P, P, P, P]),
    "spmx_hybridspmv": (c_int, [P, c_float, P]),
    "spmx_copy_csr": (c_int, [P, P, P, P]),
    "spmx_set_x": (c_int, [P, P]),
    "spmx_set_sparse_x": (c_int, [P, P, P, c_int]),
    "spmx_set_bitvector": (c_int, [P, P, c_int]),
    "spmx_set_sparse_x_dense_x": (c_int, [P, P, P, P, c_int]),
    "spmx_set_vector_type": (c_int, [P, c_int]),
    "spmx_sparse2dense": (c_int, [P]),
    "spmx_sparse2bitarray": (c_int, [P]),
    "spmx_dense2sparse": (c_int, [P, PI]),
    "spmx_bitarray2sparse": (c_int, [P, PI]),
    "spmx_dense2bitarray": (c_int, [P]),
    "spmx_dense2sparse_outer": (c_int, [P, c_int, P, PI, P, P]),
    "spmx_dense2sparse_to_host": (c_int, [P, c_int, P, P, P, P]),
    "spmx_sparse2dense_outer": (c_int, [P, c_int, P, P, c_int, P]),
    "spmx_alloc_pre_buffer": (c_int, [P]),
    "spmx_dealloc_pre_buffer": (c_int, [P]),
    "spmx_hola_preprocess": (c_int, [P]),
    "spmx_hola_postprocess": (c_int, [P]),
    "spmx_set_sigma": (c_int, [P, c_int]),
    "spmx_csr5_preprocess": (c_int, [P]),
    "spmx_csr5_postprocess": (c_int, [P]),
    "spmx_csr5_sigma": (c_int, [P, PI]),
    "spmx_set_spmv_type": (c_int, [P, c_int]),
    "spmx_tiled_preprocess": (c_int, [P, c_int, c_int, c_int, c_int]),
    "spmx_tiled_postprocess": (c_int, [P]),
    "spmx_tiled_info": (c_int, [P, P]),
    "spmx_spmspv_batched": (c_int, [P, c_int, c_int, P, P, P, c_float, P]),
    "spmx_set_batch_options": (c_int, [P, c_int]),
    "spmx_spmspv_batched_backward": (c_int, [P, c_int, c_int, P, P, P, c_float, P, P, P]),
    "spmx_tiledspmv": (c_int, [P, c_float, P]),
    "spmx_tiledspmspv": (c_int, [P, c_float, P]),
    "spmx_round_preprocess": (c_int, [P, c_int]),
    "spmx_round_preprocess_parts": (c_int, [P, c_int, c_int]),
    "spmx_round_postprocess": (c_int, [P]),
    "spmx_round_info": (c_int, [P, P]),
    "spmx_roundspmv": (c_int, [P, c_float, P]),
    "spmx_roundspmspv": (c_int, [P, c_float, P]),
    "spmx_naivespmv": (c_int, [P, c_float, P]),
    "spmx_holaspmv": (c_int, [P, c_float, P]),
    "spmx_csr5spmv": (c_int, [P, c_float, P]),
    "spmx_naivespmspv": (c_int, [P, c_float, P]),
    "spmx_holaspmspv": (c_int, [P, c_float, P]),
    "spmx_csr5spmspv": (c_int, [P, c_float, P]),
    "spmx_spmv": (c_int, [P, c_float, P]),
    "spmx_spmspv": (c_int, [P, c_float, P]),
    "spmx_spmspv_csc": (c_int, [P, c_int, c_int, c_float, P, P, P, PI]),
    "spmx_csc_naive_atomic": (c_int, [P, c_float, PI, P]),
    "spmx_csc_naive_atomic_keyval": (c_int, [P, c_float, PI, P, P, P]),
    "spmx_csc_naive_sort": (c_int, [P, c_float, PI, P, P]),
    "spmx_csc_merge_atomic": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_merge_atomic_keyval": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_merge_sort": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_twolayer_atomic": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_twolayer_atomic_keyval": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_twolayer_sort": (c_int, [P, c_int, c_float, PI, P, P, P]),
    "spmx_csc_bucket": (c_int, [P, c_float, PI, P, P, P, c_int]),
    "spmx_spmspv_csc_noalloc": (c_int, [c_int, c_int, c_int, P, P, P, c_int, P, P, c_float, P, P]),
    "spmx_spmspv_csc_noalloc_check": (c_int, [P]),
    "spmx_compute_binlen": (c_int, [P, PLL]),
    "spmx_compute_gm": (c_int, [P, PD]),
    "spmx_mat_features": (c_int, [P, PD]),
    "spmx_std_row": (c_int, [P, PF]),
    "spmx_vec_features": (c_int, [P, PLL]),
    "spmx_features": (c_int, [P, PD]),
    "spmx_select": (c_int, [P, PI]),
    "spmx_select_features": (c_int, [PD, PI]),
    "spmx_selector_inputs": (c_int, [P, PD]),
    "spmx_run_adaptive": (c_int, [P, c_float, P, PI]),
    "spmx_set_naive_lanes": (c_int, [P, c_int, c_int]),
    "spmx_run_kernel": (c_int, [P, c_int, c_float, P]),
    "spmx_autotune": (c_int, [P, ctypes.c_char_p, PI]),
    "spmx_bfs": (c_int, [P, c_int, P, PI]),
    "spmx_set_bfs_mode": (c_int, [P, c_int]),
    "spmx_bfs_batched": (c_int, [P, PI, c_int, P, c_int, PI]),
    "spmx_get_device_counts": (c_int, [P, PP]),
    "spmx_spmv_backward": (c_int, [P, P, P, P, P]),
    "spmx_spmv_backward_sparse": (c_int, [P, P, P, P, c_int, P, P]),
    "spmx_host_free": (None, [P]),
    "spmx_gen_rmat": (c_int, [c_int, c_int, c_double, c_double, c_double, c_u64, PI, PLL, PP, PP]),
    "spmx_gen_zipf_rows": (c_int, [c_int, c_double, c_int, c_int, c_u64, PLL, PP, PP, PP]),
    "spmx_gen_chung_lu": (c_int, [c_int, c_double, c_double, c_u64, PLL, PP, PP, PP]),
    "spmx_gen_laplacian": (c_int, [c_int, c_double, c_u64, PLL, PP, PP, PP]),
    "spmx_gen_sparse_vector": (c_int, [c_int, c_int, c_int, c_u64, P, P]),
    "spmx_host_csr2csc": (c_int, [c_int, c_int, P, P, P, P, P, P]),
    "spmx_mtx_read": (c_int, [ctypes.c_char_p, PI, PI, PLL, PP, PP, PP, PI]),
    "spmx_mtx_write": (c_int, [ctypes.c_char_p, c_int, c_int, c_ll, P, P, P, c_int]),
    "spmx_csr_store": (c_int, [ctypes.c_char_p, c_int, c_int, c_int, P, P, P]),
    "spmx_csr_load_header": (c_int, [ctypes.c_char_p, PI, PI, PI]),
    "spmx_csr_load": (c_int, [ctypes.c_char_p, c_int, c_int, c_int, P, P, P]),
}

# optional entry points (present once their components are built)
_OPTIONAL = set()

for _name, (_res, _args) in _SIGS.items():
    try:
        _fn = getattr(lib, _name)
    except AttributeError:
        if _name in _OPTIONAL:
            continue
        raise ImportError(f"libspmx.so does not export {_name}")
    _fn.restype = _res
    _fn.argtypes = _args


def declared_symbols():
    """Names of every entry point this binding declares."""
    return sorted(_SIGS)


class SpmxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"spmx error {code}: {msg}")
        self.code = code


def last_error():
    s = lib.spmx_last_error_string()
    return s.decode() if s else ""


def check(rc, what=""):
    if rc != SUCCESS:
        raise SpmxError(rc, (what + ": " if what else "") + last_error())
    return rc
