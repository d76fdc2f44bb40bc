"""The Spartan side of provekit's prover (provekit/common/src/utils/sumcheck.rs,
provekit/prover/src/whir_r1cs.rs) over the CUDA implementation."""
import ctypes

import numpy as np
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib


class Transcript(ctypes.Structure):
    """Fiat-Shamir transcript state (see pkg_transcript in the C header)."""
    _fields_ = [("l", ctypes.c_uint64 * 4), ("r", ctypes.c_uint64 * 4)]

    @classmethod
    def new(cls, domain: int):
        t = cls()
        d = np.array([domain & (2**64 - 1), (domain >> 64) & (2**64 - 1),
                      (domain >> 128) & (2**64 - 1), (domain >> 192) & (2**64 - 1)], np.uint64)
        check(lib().pkg_transcript_init(ctypes.byref(t), d.ctypes.data))
        return t

    def absorb(self, x_mont):
        x = np.ascontiguousarray(np.asarray(x_mont, dtype=np.uint64).reshape(4))
        check(lib().pkg_transcript_absorb(ctypes.byref(self), x.ctypes.data))

    def squeeze(self) -> np.ndarray:
        out = np.zeros(4, np.uint64)
        check(lib().pkg_transcript_squeeze(ctypes.byref(self), out.ctypes.data))
        return out


def eq_hypercube(r: np.ndarray, num_entries: int, out=None, stream=None):
    """calculate_evaluations_over_boolean_hypercube_for_eq (sumcheck.rs:108-120).
    r: host (nr, 4) uint64; returns a CUDA (num_entries, 4) tensor."""
    r = np.ascontiguousarray(r, dtype=np.uint64).reshape(-1, 4)
    if out is None:
        out = torch.empty((num_entries, 4), dtype=torch.int64, device="cuda")
    check(lib().pkg_eq_hypercube(r.ctypes.data if r.size else None, r.shape[0], num_entries,
                                 ptr(out) if num_entries else None, stream_handle(stream)))
    return out


def spartan_round(a, b, c, eq, size: int, fold=None, stream=None) -> np.ndarray:
    """One round of the Spartan map-reduce; returns (3, 4) host array
    (f(0), f(-1), f(inf))."""
    out = np.zeros((3, 4), np.uint64)
    f = None if fold is None else np.ascontiguousarray(np.asarray(fold, np.uint64).reshape(4))
    check(lib().pkg_spartan_round(ptr(a), ptr(b), ptr(c), ptr(eq), size,
                                  None if f is None else f.ctypes.data, out.ctypes.data,
                                  stream_handle(stream)))
    return out


def spartan_sumcheck(a, b, c, m0: int, g: np.ndarray, w1_blinding: np.ndarray,
                     transcript: Transcript, stream=None):
    """run_zk_sumcheck_prover (whir_r1cs.rs:519-621).  a, b, c: CUDA tables of
    2^m0 Fr (modified in place).  Returns a dict of host arrays."""
    g = np.ascontiguousarray(g, dtype=np.uint64).reshape(-1, 4)
    wb = np.ascontiguousarray(w1_blinding, dtype=np.uint64).reshape(-1, 4)
    out = {"r": np.zeros((m0, 4), np.uint64), "rho": np.zeros(4, np.uint64),
           "sum_g": np.zeros(4, np.uint64), "coeffs": np.zeros((4 * m0, 4), np.uint64),
           "alpha": np.zeros((m0, 4), np.uint64), "blinding_eval": np.zeros(4, np.uint64)}
    check(lib().pkg_spartan_sumcheck(
        ptr(a), ptr(b), ptr(c), m0, g.ctypes.data, wb.ctypes.data, ctypes.byref(transcript),
        out["r"].ctypes.data, out["rho"].ctypes.data, out["sum_g"].ctypes.data,
        out["coeffs"].ctypes.data, out["alpha"].ctypes.data, out["blinding_eval"].ctypes.data,
        stream_handle(stream)))
    return out


class CsrMatrix:
    """Device CSR matrix with one Fr per nonzero (a hydrated SparseMatrix)."""

    def __init__(self, num_rows, num_cols, row_ptr, cols, vals):
        self.num_rows, self.num_cols = num_rows, num_cols
        self.row_ptr, self.cols, self.vals = row_ptr, cols, vals

    @classmethod
    def from_host(cls, num_rows, num_cols, row_ptr: np.ndarray, cols: np.ndarray, vals: np.ndarray):
        rp = torch.from_numpy(np.ascontiguousarray(row_ptr, np.uint64).view(np.int64)).cuda()
        cl = torch.from_numpy(np.ascontiguousarray(cols, np.uint32).view(np.int32)).cuda()
        vl = torch.from_numpy(np.ascontiguousarray(vals, np.uint64).reshape(-1, 4).view(np.int64)).cuda()
        return cls(num_rows, num_cols, rp, cl, vl)

    @property
    def nnz(self):
        return self.cols.numel()

    def mul(self, x, y=None, stream=None):
        """HydratedSparseMatrix * &[Fr] (sparse_matrix.rs:606-627)."""
        fr_tensor(x, "x")
        if y is None:
            y = torch.empty((self.num_rows, 4), dtype=torch.int64, device=x.device)
        if x.shape[0] != self.num_cols:
            raise ValueError("Vector length does not match number of columns.")
        check(lib().pkg_spmv_csr(ptr(self.row_ptr), ptr(self.cols), ptr(self.vals), self.num_rows,
                                 self.num_cols, ptr(x), ptr(y), stream_handle(stream)))
        return y

    def transpose(self, stream=None):
        """SparseMatrix::transpose (sparse_matrix.rs:409)."""
        rp = torch.empty(self.num_cols + 1, dtype=torch.int64, device="cuda")
        cl = torch.empty(max(self.nnz, 1), dtype=torch.int32, device="cuda")
        vl = torch.empty((max(self.nnz, 1), 4), dtype=torch.int64, device="cuda")
        check(lib().pkg_csr_transpose(ptr(self.row_ptr), ptr(self.cols), ptr(self.vals),
                                      self.num_rows, self.num_cols, self.nnz, ptr(rp), ptr(cl),
                                      ptr(vl), stream_handle(stream)))
        return CsrMatrix(self.num_cols, self.num_rows, rp, cl[: self.nnz], vl[: self.nnz])


def hadamard_pad(a, b, n: int, padded: int, out=None, stream=None):
    if out is None:
        out = torch.empty((padded, 4), dtype=torch.int64, device="cuda")
    check(lib().pkg_hadamard_pad(ptr(a), ptr(b), n, padded, ptr(out), stream_handle(stream)))
    return out


def dot(a, b, n=None, stream=None) -> np.ndarray:
    n = a.shape[0] if n is None else n
    out = np.zeros(4, np.uint64)
    check(lib().pkg_dot(ptr(a), ptr(b), n, out.ctypes.data, stream_handle(stream)))
    return out
