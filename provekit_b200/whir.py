"""Device operations of WHIR's prove rounds (the whir crate's prover is not
vendored with the reference; its arithmetic here follows the reference's Go
WHIR verifier, recursive-verifier/app/).  Tensors are (n, 4) int64 CUDA
tensors of Montgomery-form Fr limbs; small per-round values are (k, 4)
uint64 host arrays."""
import ctypes

import numpy as np
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import PKG_LEAF_CANONICAL, check, lib

SUBSET_ZETA = 0
SUBSET_MOBIUS_T = 1
MAX_ROUNDS = 16


def _host(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64).reshape(-1, 4))


def fold_coeffs(coeffs, k: int, alpha, out=None, stream=None):
    """Fold the 2^k contiguous messages of coeffs with MultivarPoly weights."""
    fr_tensor(coeffs, "coeffs")
    n = coeffs.shape[0]
    if out is None:
        out = torch.empty((n >> k, 4), dtype=torch.int64, device=coeffs.device)
    a = _host(alpha) if k else np.zeros((1, 4), np.uint64)
    check(lib().pkg_whir_fold_coeffs(ptr(coeffs), n, k, a.ctypes.data, ptr(out),
                                     stream_handle(stream)))
    return out


def fold_rows(rows, k: int, alpha, out=None, stream=None):
    """computeFold: MultivarPoly(row, alpha) for every row of 2^k Fr."""
    fr_tensor(rows, "rows")
    nrows = rows.shape[0] >> k
    if out is None:
        out = torch.empty((nrows, 4), dtype=torch.int64, device=rows.device)
    a = _host(alpha) if k else np.zeros((1, 4), np.uint64)
    check(lib().pkg_whir_fold_rows(ptr(rows), nrows, k, a.ctypes.data, ptr(out),
                                   stream_handle(stream)))
    return out


def poly_eval_many(coeffs, points, stream=None) -> np.ndarray:
    """sum_i coeffs[i] z^i for every z in points (host (npts, 4))."""
    fr_tensor(coeffs, "coeffs")
    pts = _host(points)
    out = np.zeros_like(pts)
    check(lib().pkg_poly_eval_many(ptr(coeffs), coeffs.shape[0], pts.ctypes.data, pts.shape[0],
                                   out.ctypes.data, stream_handle(stream)))
    return out


def merkle_open(layers, num_leaves: int, indices, stream=None) -> np.ndarray:
    """(nq, depth, 32) uint8: sibling then auth path of every queried leaf."""
    idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
    depth = num_leaves.bit_length() - 1
    out = np.zeros((max(len(idx), 1), max(depth, 1), 32), np.uint8)
    check(lib().pkg_merkle_open(ptr(layers), num_leaves, idx.ctypes.data, len(idx),
                                out.ctypes.data, stream_handle(stream)))
    return out[: len(idx), :depth]


def gather_rows(codeword, fr_per_row: int, indices, stream=None) -> np.ndarray:
    fr_tensor(codeword, "codeword")
    idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
    out = np.zeros((max(len(idx) * fr_per_row, 1), 4), np.uint64)
    check(lib().pkg_gather_rows(ptr(codeword), fr_per_row, codeword.shape[0] // fr_per_row,
                                idx.ctypes.data, len(idx), out.ctypes.data, stream_handle(stream)))
    return out[: len(idx) * fr_per_row].reshape(len(idx), fr_per_row, 4)


def stir_indices(challenge_bytes: bytes, folded_domain_size: int, nq: int) -> np.ndarray:
    b = np.frombuffer(challenge_bytes, dtype=np.uint8).copy() if challenge_bytes else \
        np.zeros(1, np.uint8)
    out = np.zeros(max(nq, 1), np.uint64)
    check(lib().pkg_stir_indices(b.ctypes.data, folded_domain_size, nq, out.ctypes.data))
    return out[:nq]


def sumcheck_round(f, w, size: int, fold=None, stream=None) -> np.ndarray:
    """(h(0), h(1), h(2)) as a (3, 4) host array; folds the top variable first
    when fold (one Fr) is given."""
    out = np.zeros((3, 4), np.uint64)
    fd = None if fold is None else _host(fold)
    check(lib().pkg_whir_sumcheck_round(ptr(f), ptr(w), size, None if fd is None else fd.ctypes.data,
                                        out.ctypes.data, stream_handle(stream)))
    return out


def eq_accumulate(w, nv: int, points, coeffs, stream=None):
    """w[b] += sum_j coeffs[j] eq(points[j], b); points: host (npts * nv, 4)."""
    pts = _host(points)
    cf = _host(coeffs)
    check(lib().pkg_eq_accumulate(ptr(w), nv, pts.ctypes.data, cf.ctypes.data, cf.shape[0],
                                  stream_handle(stream)))
    return w



# ---- the WHIR prover's round loop (pkg_whir_prove) ------------------------
class WhirParams(ctypes.Structure):
    """pkg_whir_params: the protocol shape (see the C header)."""
    _fields_ = [("num_variables", ctypes.c_uint32), ("folding_factor", ctypes.c_uint32),
                ("log_inv_rate", ctypes.c_uint32), ("num_rounds", ctypes.c_uint32),
                ("final_vars", ctypes.c_uint32), ("ood_samples", ctypes.c_uint32),
                ("pow_bits", ctypes.c_uint32), ("final_pow_bits", ctypes.c_uint32),
                ("batch_size", ctypes.c_uint32),
                ("queries", ctypes.c_uint32 * (MAX_ROUNDS + 1))]

    @classmethod
    def new(cls, num_variables: int, folding_factor: int = 3, log_inv_rate: int = 2,
            security_bits: int = 128, pow_bits: int = 10, **overrides):
        """The schedule of pkg_whir_params_init; keyword overrides set fields
        afterwards (queries as a list)."""
        p = cls()
        check(lib().pkg_whir_params_init(ctypes.byref(p), num_variables, folding_factor,
                                         log_inv_rate, security_bits, pow_bits))
        for key, v in overrides.items():
            if key == "queries":
                for i, q in enumerate(v):
                    p.queries[i] = q
            else:
                setattr(p, key, v)
        return p

    def commit_words(self) -> int:
        return lib().pkg_whir_commit_words(ctypes.byref(self))

    def proof_words(self, num_covectors: int) -> int:
        n = lib().pkg_whir_proof_words(ctypes.byref(self), num_covectors)
        if n == 0:
            raise ValueError("invalid WHIR parameters")
        return n


def subset_transform(v, n: int, mode: int, stream=None):
    """In place: SUBSET_ZETA (coefficients -> hypercube evaluations) or
    SUBSET_MOBIUS_T (covector -> hypercube weight) over 2^n entries."""
    fr_tensor(v, "v")
    if v.shape[0] != 1 << n:
        raise ValueError("table length must be 2^n")
    check(lib().pkg_subset_transform(ptr(v), n, mode, stream_handle(stream)))
    return v


def squeeze_bytes(transcript, n: int) -> bytes:
    out = np.zeros(max(n, 1), np.uint8)
    check(lib().pkg_transcript_squeeze_bytes(ctypes.byref(transcript), out.ctypes.data, n))
    return out[:n].tobytes()


def commit(coeffs, params: WhirParams, stream=None):
    """pkg_whir_commit of the batch's batch_size x 2^n coefficients
    (concatenated) with canonical leaves: (codeword, layers)."""
    fr_tensor(coeffs, "coeffs")
    n, k, lr, nb = params.num_variables, params.folding_factor, params.log_inv_rate, \
        params.batch_size
    if coeffs.shape[0] != nb << n:
        raise ValueError("coeffs must hold batch_size x 2^num_variables entries")
    kb = k + {1: 0, 2: 1, 4: 2}[nb]
    L = (1 << (n - k)) << lr
    cw = torch.empty(((nb << n) << lr, 4), dtype=torch.int64, device=coeffs.device)
    layers = torch.empty(((2 * L - 1) * 32,), dtype=torch.uint8, device=coeffs.device)
    check(lib().pkg_whir_commit(ptr(coeffs), nb << n, kb, lr, None, 0, PKG_LEAF_CANONICAL,
                                ptr(cw), ptr(layers), stream_handle(stream)))
    return cw, layers


def commit_ood(params: WhirParams, transcript, coeffs, layers, stream=None):
    """Root and OOD answers into the transcript: (commit_words, ood_points)."""
    words = np.zeros(params.commit_words(), np.uint64)
    ood = np.zeros((params.ood_samples + 1, 4), np.uint64)
    check(lib().pkg_whir_commit_ood(ctypes.byref(params), ctypes.byref(transcript), ptr(coeffs),
                                    ptr(layers), words.ctypes.data, ood.ctypes.data,
                                    stream_handle(stream)))
    return words, ood


def prove(params: WhirParams, transcript, coeffs, codeword, layers, ood_points, covectors=None,
          stream=None) -> np.ndarray:
    """The proof words of the statements <covector_j, coeffs> (covectors:
    (ncov * 2^n, 4) device tensor or None)."""
    N = 1 << params.num_variables
    ncov = 0 if covectors is None else covectors.shape[0] // N
    if covectors is not None:
        fr_tensor(covectors, "covectors")
        if covectors.shape[0] != ncov * N:
            raise ValueError("covectors must be a multiple of 2^n entries")
    proof = np.zeros(params.proof_words(ncov), np.uint64)
    ood = np.ascontiguousarray(ood_points, dtype=np.uint64)
    check(lib().pkg_whir_prove(ctypes.byref(params), ctypes.byref(transcript), ptr(coeffs),
                               ptr(codeword), ptr(layers), ood.ctypes.data, ptr(covectors), ncov,
                               proof.ctypes.data, stream_handle(stream)))
    return proof
