"""ctypes binding of libprovekit_b200.so (the C ABI in include/provekit_b200.h).

The library is built in-tree by provekit_b200.build; importing this module
without it raises immediately -- there is no CPU fallback for the product path.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprovekit_b200.so")

PKG_OK = 0
PKG_ERR_INVALID_ARGUMENT = -1
PKG_ERR_CUDA = -2
PKG_ERR_OUT_OF_MEMORY = -3
PKG_ERR_UNSUPPORTED = -4
PKG_ERR_TIMEOUT = -5

PKG_LEAF_CANONICAL = 0
PKG_LEAF_MONTGOMERY = 1

_c_sz = ctypes.c_size_t
_c_u64p = ctypes.POINTER(ctypes.c_uint64)
_c_u8p = ctypes.POINTER(ctypes.c_uint8)
_c_vp = ctypes.c_void_p
_c_int = ctypes.c_int
_c_uint = ctypes.c_uint

# name -> argtypes; every entry point returns int
SIGNATURES = {
    "pkg_sample_fr": [ctypes.c_uint64, _c_sz, _c_vp, _c_int],
    "pkg_ntt_nr": [_c_vp, _c_sz, _c_sz, _c_sz, _c_vp],
    "pkg_intt_rn": [_c_vp, _c_sz, _c_vp],
    "pkg_intt_rn_noalloc": [_c_vp, _c_sz, _c_vp],
    "pkg_ntt_engine_reserve": [_c_sz],
    "pkg_host_ntt_nr": [_c_vp, _c_sz, _c_sz, _c_sz],
    "pkg_host_intt_rn": [_c_vp, _c_sz],
    "pkg_rs_next_order": [_c_sz, ctypes.POINTER(_c_sz)],
    "pkg_rs_generator": [_c_sz, _c_vp],
    "pkg_rs_evaluation_points": [_c_sz, _c_vp, _c_sz, _c_vp],
    "pkg_rs_interleaved_encode": [_c_vp, _c_sz, _c_sz, _c_vp, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_host_rs_interleaved_encode": [_c_vp, _c_sz, _c_sz, _c_vp, _c_sz, _c_sz, _c_vp],
    "pkg_skyscraper_compress_many": [_c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_skyscraper_hash_many": [_c_sz, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_host_skyscraper_hash_many": [_c_sz, _c_vp, _c_sz, _c_vp],
    "pkg_skyscraper_pow_solve": [_c_vp, _c_vp, _c_u64p],
    "pkg_poseidon2_permutation_many": [_c_vp, _c_sz, _c_vp],
    "pkg_poseidon2_hash_many": [_c_vp, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_merkle_tree": [_c_vp, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_merkle_tree_fr": [_c_vp, _c_sz, _c_sz, _c_int, _c_vp, _c_vp],
    "pkg_merkle_leaves_fr": [_c_vp, _c_sz, _c_sz, _c_int, _c_vp, _c_vp],
    "pkg_merkle_levels": [_c_vp, _c_sz, _c_vp],
    "pkg_whir_commit": [_c_vp, _c_sz, _c_uint, _c_uint, _c_vp, _c_sz, _c_int, _c_vp, _c_vp, _c_vp],
    "pkg_transcript_init": [_c_vp, _c_vp],
    "pkg_transcript_absorb": [_c_vp, _c_vp],
    "pkg_transcript_squeeze": [_c_vp, _c_vp],
    "pkg_eq_hypercube": [_c_vp, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_spartan_round": [_c_vp, _c_vp, _c_vp, _c_vp, _c_sz, _c_vp, _c_vp, _c_vp],
    "pkg_spartan_sumcheck": [_c_vp, _c_vp, _c_vp, _c_sz, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp,
                             _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_spmv_csr": [_c_vp, _c_vp, _c_vp, _c_sz, _c_sz, _c_vp, _c_vp, _c_vp],
    "pkg_csr_transpose": [_c_vp, _c_vp, _c_vp, _c_sz, _c_sz, _c_sz, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_hadamard_pad": [_c_vp, _c_vp, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_dot": [_c_vp, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_spartan_prove": [_c_vp, _c_vp, ctypes.c_uint64, ctypes.c_uint64, _c_uint, _c_uint, _c_vp,
                          _c_vp],
    "pkg_synthetic_r1cs": [ctypes.c_uint64, _c_sz, _c_sz, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_batch_create": [_c_vp, _c_sz, ctypes.c_uint64, _c_vp],
    "pkg_batch_job_info": [_c_vp, _c_sz, _c_vp],
    "pkg_batch_set_params": [_c_vp, _c_int, _c_int],
    "pkg_batch_tune": [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_batch_set_butterflies_per_thread": [_c_vp, _c_int],
    "pkg_batch_get_params": [_c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_batch_run": [_c_vp, _c_int, _c_vp],
    "pkg_batch_sumcheck_result": [_c_vp, _c_sz, _c_vp],
    "pkg_copy_to_host": [_c_vp, _c_vp, _c_sz],
    "pkg_server_create": [_c_sz, _c_int, _c_vp],
    "pkg_server_submit": [_c_vp, _c_vp, _c_vp],
    "pkg_server_wait": [_c_vp, ctypes.c_uint64, _c_vp, _c_vp],
    "pkg_server_get_stats": [_c_vp, _c_vp],
    "pkg_measure_imad_rate": [ctypes.POINTER(ctypes.c_double)],
    "pkg_measure_dfma_rate": [ctypes.POINTER(ctypes.c_double)],
    "pkg_last_prove_stages": [ctypes.c_void_p],
    "pkg_trim_memory": [ctypes.c_size_t],
    "pkg_reserve_memory": [ctypes.c_size_t],
    "pkg_sample_fr_indexed": [ctypes.c_uint64, ctypes.c_uint64, _c_sz, _c_vp, _c_vp],
    "pkg_whir_fold_coeffs": [_c_vp, _c_sz, _c_uint, _c_vp, _c_vp, _c_vp],
    "pkg_whir_fold_rows": [_c_vp, _c_sz, _c_uint, _c_vp, _c_vp, _c_vp],
    "pkg_poly_eval_many": [_c_vp, _c_sz, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_merkle_open": [_c_vp, _c_sz, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_gather_rows": [_c_vp, _c_sz, _c_sz, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_stir_indices": [_c_vp, _c_sz, _c_sz, _c_vp],
    "pkg_whir_sumcheck_round": [_c_vp, _c_vp, _c_sz, _c_vp, _c_vp, _c_vp],
    "pkg_eq_accumulate": [_c_vp, _c_sz, _c_vp, _c_vp, _c_sz, _c_vp],
    "pkg_fr_mul_batch": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                         ctypes.c_int, ctypes.c_void_p],
    "pkg_r1cs_sizing": [_c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_prove_r1cs": [_c_vp, _c_vp, ctypes.c_uint64, ctypes.c_uint64, _c_vp, _c_vp, _c_vp, _c_vp,
                       _c_vp],
    "pkg_last_whir_stages": [_c_vp],
    "pkg_whir_params_init": [_c_vp, _c_uint, _c_uint, _c_uint, _c_uint, _c_uint],
    "pkg_transcript_squeeze_bytes": [_c_vp, _c_vp, _c_sz],
    "pkg_subset_transform": [_c_vp, _c_uint, _c_int, _c_vp],
    "pkg_whir_commit_ood": [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_whir_prove": [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_sz, _c_vp, _c_vp],
    "pkg_version": [],
    "pkg_release_thread_resources": [],
    "pkg_r1cs_build_transposes": [_c_vp, _c_vp, _c_vp],
    "pkg_get_last_error": [_c_vp],
    "pkg_init": [],
    "pkg_prover_config_default": [_c_vp],
    "pkg_prover_create": [_c_sz, _c_sz, _c_sz, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_prover_get_info": [_c_vp, _c_vp],
    "pkg_prover_prove": [_c_vp, _c_vp, ctypes.c_uint64, _c_vp],
    "pkg_prover_serialize": [_c_vp, _c_vp],
    "pkg_prover_load_bytes": [_c_vp, _c_sz, _c_vp],
    "pkg_thread_resource_bytes": [_c_vp, _c_vp],
    "pkg_r1cs_sizing_split": [_c_sz, _c_sz, _c_sz, _c_vp, _c_vp],
    "pkg_dual_prove_begin": [_c_vp, _c_sz, _c_vp, _c_sz, _c_vp, ctypes.c_uint64, ctypes.c_uint64,
                             _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_dual_prove_finish": [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_vp],
    "pkg_synthetic_r1cs_dual": [ctypes.c_uint64, _c_sz, _c_sz, _c_sz, _c_sz, _c_vp, _c_vp, _c_vp,
                                _c_vp, _c_vp, _c_vp],
    "pkg_synthetic_dual_solve": [_c_sz, _c_sz, _c_vp, _c_vp, _c_vp, _c_sz, _c_vp, _c_sz, _c_vp,
                                 _c_vp],
}


class PkgBuf(ctypes.Structure):
    """pkg_buf: library-owned bytes, released by pkg_free_buf."""
    _fields_ = [("ptr", ctypes.POINTER(ctypes.c_uint8)), ("len", ctypes.c_size_t),
                ("cap", ctypes.c_size_t)]


class PkgError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"provekit_b200 error {code}: {message}")
        self.code = code


_lib = None


def lib():
    """Load the CUDA library (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m provekit_b200.build` "
                "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.pkg_last_error.restype = ctypes.c_char_p
        L.pkg_last_error.argtypes = []
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.pkg_batch_destroy.argtypes = [_c_vp]
        L.pkg_batch_destroy.restype = None
        L.pkg_server_destroy.argtypes = [_c_vp]
        L.pkg_server_destroy.restype = None
        L.pkg_free_buf.argtypes = [PkgBuf]
        L.pkg_free_buf.restype = None
        L.pkg_prover_free.argtypes = [_c_vp]
        L.pkg_prover_free.restype = None
        L.pkg_dual_prove_free.argtypes = [_c_vp]
        L.pkg_dual_prove_free.restype = None
        L.pkg_r1cs_transposes_bytes.argtypes = [_c_vp]
        L.pkg_r1cs_transposes_bytes.restype = ctypes.c_size_t
        for name in ("pkg_whir_commit_words", "pkg_whir_proof_words"):
            fn = getattr(L, name)
            fn.argtypes = [_c_vp] if name == "pkg_whir_commit_words" else [_c_vp, _c_sz]
            fn.restype = ctypes.c_size_t
        L.pkg_kernel_launches.argtypes = []
        L.pkg_kernel_launches.restype = ctypes.c_uint64
        _lib = L
    return _lib


def last_error() -> str:
    return lib().pkg_last_error().decode()


def check(rc: int):
    if rc != PKG_OK:
        raise PkgError(rc, last_error())
    return rc


def exported_symbols():
    return sorted(SIGNATURES) + ["pkg_last_error", "pkg_kernel_launches", "pkg_batch_destroy",
                                  "pkg_server_destroy", "pkg_whir_commit_words",
                                  "pkg_whir_proof_words", "pkg_r1cs_transposes_bytes",
                                  "pkg_free_buf", "pkg_prover_free", "pkg_dual_prove_free"]
