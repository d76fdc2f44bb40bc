"""Batched form: many uneven jobs (NTT + WHIR commit + zk-sumcheck each) as one
CUDA graph of grouped kernels (see pkg_batch_* in the C header)."""
import ctypes

import numpy as np
import torch

from ._lib import check, lib
from .spartan import Transcript


class BatchJobC(ctypes.Structure):
    _fields_ = [("log_n", ctypes.c_uint32), ("n", ctypes.c_size_t), ("coeffs", ctypes.c_void_p),
                ("ntt", ctypes.c_void_p), ("codeword", ctypes.c_void_p), ("layers", ctypes.c_void_p),
                ("num_leaves", ctypes.c_size_t), ("transcript_domain", ctypes.c_uint64),
                ("g", ctypes.c_uint64 * 480), ("w1_blinding", ctypes.c_uint64 * 480)]


class SumcheckResultC(ctypes.Structure):
    _fields_ = [("m0", ctypes.c_size_t), ("r", ctypes.c_uint64 * 120),
                ("coeffs", ctypes.c_uint64 * 480), ("alpha", ctypes.c_uint64 * 120),
                ("rho", ctypes.c_uint64 * 4), ("sum_g", ctypes.c_uint64 * 4),
                ("blinding_eval", ctypes.c_uint64 * 4), ("transcript", Transcript)]

    def as_dict(self):
        m0 = self.m0
        arr = lambda x, n: np.array(x[: 4 * n], dtype=np.uint64).reshape(n, 4)  # noqa: E731
        return {"r": arr(self.r, m0), "coeffs": arr(self.coeffs, 4 * m0), "alpha": arr(self.alpha, m0),
                "rho": np.array(self.rho, np.uint64), "sum_g": np.array(self.sum_g, np.uint64),
                "blinding_eval": np.array(self.blinding_eval, np.uint64),
                "transcript": (list(self.transcript.l), list(self.transcript.r))}


class Batch:
    def __init__(self, log_sizes, seed: int):
        self._b = ctypes.c_void_p()
        ls = (ctypes.c_uint32 * len(log_sizes))(*log_sizes)
        check(lib().pkg_batch_create(ls, len(log_sizes), seed, ctypes.byref(self._b)))
        self.log_sizes = list(log_sizes)

    def close(self):
        if self._b:
            lib().pkg_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def job(self, j: int) -> BatchJobC:
        out = BatchJobC()
        check(lib().pkg_batch_job_info(self._b, j, ctypes.byref(out)))
        return out

    def set_params(self, kmax: int, log_elems: int, log_bpt: int = None):
        """NTT plan: passes of at most kmax stages, 2^log_elems elements per
        CTA and (if given) 2^log_bpt butterflies per thread per stage."""
        if log_bpt is not None:
            check(lib().pkg_batch_set_butterflies_per_thread(self._b, log_bpt))
        check(lib().pkg_batch_set_params(self._b, kmax, log_elems))

    def params(self):
        """(kmax, log2 elements per CTA, log2 butterflies per thread)."""
        k, e, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().pkg_batch_get_params(self._b, ctypes.byref(k), ctypes.byref(e),
                                         ctypes.byref(t)))
        return k.value, e.value, t.value

    def tune(self, stream=None):
        """Autotune (kmax, elements per CTA, butterflies per thread); returns
        (kmax, log2 elements per CTA, best ms); params() gives all three."""
        k, e, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        s = (stream or torch.cuda.current_stream()).cuda_stream
        check(lib().pkg_batch_tune(self._b, s, ctypes.byref(k), ctypes.byref(e), ctypes.byref(ms)))
        return k.value, e.value, ms.value

    def run(self, use_graph=True, stream=None):
        s = (stream or torch.cuda.current_stream()).cuda_stream
        check(lib().pkg_batch_run(self._b, int(use_graph), s))

    def sumcheck_result(self, j: int) -> dict:
        out = SumcheckResultC()
        check(lib().pkg_batch_sumcheck_result(self._b, j, ctypes.byref(out)))
        return out.as_dict()

    @staticmethod
    def read(ptr, nbytes: int) -> bytes:
        """Copy nbytes of batch-owned device memory to the host."""
        out = np.zeros(max(nbytes, 1), np.uint8)
        check(lib().pkg_copy_to_host(out.ctypes.data, ptr, nbytes))
        return out[:nbytes].tobytes()

    @staticmethod
    def read_fr(ptr, n_fr) -> np.ndarray:
        return np.frombuffer(Batch.read(ptr, 32 * n_fr), dtype=np.uint64).reshape(n_fr, 4).copy()
