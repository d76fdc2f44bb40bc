"""Device operations of WHIR's prove rounds (the whir crate's prover is not
vendored with the reference; its arithmetic here follows the reference's Go
WHIR verifier, recursive-verifier/app/).  Tensors are (n, 4) int64 CUDA
tensors of Montgomery-form Fr limbs; small per-round values are (k, 4)
uint64 host arrays."""
import numpy as np
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib


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

