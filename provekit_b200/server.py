"""Served form: a proving service with HBM-footprint admission and overlapped
device execution (pkg_server_* in the C header)."""
import ctypes

import numpy as np

from ._lib import check, lib
from .prover import SpartanProofC, statement_count, whir_params_for


class ProveRequestC(ctypes.Structure):
    _fields_ = [("num_constraints", ctypes.c_size_t), ("num_witnesses", ctypes.c_size_t),
                ("row_ptr", ctypes.c_void_p * 3), ("cols", ctypes.c_void_p * 3),
                ("vals", ctypes.c_void_p * 3), ("nnz", ctypes.c_size_t * 3),
                ("witness", ctypes.c_void_p), ("blinding_seed", ctypes.c_uint64),
                ("transcript_domain", ctypes.c_uint64), ("folding_factor", ctypes.c_uint),
                ("log_inv_rate", ctypes.c_uint), ("whir", ctypes.c_void_p),
                ("whir_commit_words", ctypes.c_void_p), ("whir_proof", ctypes.c_void_p),
                ("num_public_inputs", ctypes.c_size_t)]


class RequestTimesC(ctypes.Structure):
    _fields_ = [("submit_ns", ctypes.c_uint64), ("admit_ns", ctypes.c_uint64),
                ("done_ns", ctypes.c_uint64), ("footprint_bytes", ctypes.c_size_t)]


class ServerStatsC(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_size_t), ("queued", ctypes.c_size_t),
                ("inflight", ctypes.c_size_t), ("reserved_bytes", ctypes.c_size_t),
                ("peak_reserved_bytes", ctypes.c_size_t), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("p999_ms", ctypes.c_double),
                ("proofs_per_s", ctypes.c_double)]


def make_request(h, blinding_seed=1, transcript_domain=3, folding_factor=3, log_inv_rate=2,
                 whole=None):
    """pkg_prove_request over a HostR1CS (the arrays must outlive submit).
    whole: None for the Spartan part, or (WhirParams, commit_words buffer,
    proof buffer) for a whole proof."""
    req = ProveRequestC()
    req.num_constraints, req.num_witnesses = h.num_constraints, h.num_witnesses
    for k in range(3):
        for arr in (h.row_ptr[k], h.cols[k], h.vals[k]):
            if not arr.flags["C_CONTIGUOUS"]:
                raise ValueError("request arrays must be contiguous (the server reads them in place)")
        req.row_ptr[k] = h.row_ptr[k].ctypes.data
        req.cols[k] = h.cols[k].ctypes.data
        req.vals[k] = h.vals[k].ctypes.data
        req.nnz[k] = h.nnz[k]
    req.witness = h.witness.ctypes.data
    req.num_public_inputs = getattr(h, "num_public_inputs", 0)
    req.blinding_seed, req.transcript_domain = blinding_seed, transcript_domain
    req.folding_factor, req.log_inv_rate = folding_factor, log_inv_rate
    if whole is not None:
        p, cw, pr = whole
        req.whir = ctypes.addressof(p)
        req.whir_commit_words = cw.ctypes.data
        req.whir_proof = pr.ctypes.data
    return req


class ProofServer:
    def __init__(self, hbm_budget_bytes: int, max_inflight: int = 4):
        self._live = {}
        self._s = ctypes.c_void_p()
        check(lib().pkg_server_create(hbm_budget_bytes, max_inflight, ctypes.byref(self._s)))

    def submit(self, h, whole_proof=False, whir=None, **kw) -> int:
        """Queue a HostR1CS; the server reads its arrays until wait() returns.
        whole_proof: prove with WHIR's rounds too (whir: WhirParams, by
        default the reference's configuration for the R1CS's m)."""
        whole = None
        if whole_proof or whir is not None:
            p = whir if whir is not None else whir_params_for(h)
            whole = (p, np.zeros(p.commit_words(), np.uint64),
                     np.zeros(p.proof_words(statement_count(h)), np.uint64))
        req = make_request(h, whole=whole, **kw)
        rid = ctypes.c_uint64()
        check(lib().pkg_server_submit(self._s, ctypes.byref(req), ctypes.byref(rid)))
        self._live[rid.value] = (h, whole)  # keep the request's buffers alive until wait()
        return rid.value

    def wait(self, rid: int):
        """(Spartan fields, times) -- plus (commit words, WHIR proof) appended
        to the fields as "whir_commit_words" / "whir_proof" for whole proofs."""
        proof, times = SpartanProofC(), RequestTimesC()
        try:
            check(lib().pkg_server_wait(self._s, rid, ctypes.byref(proof), ctypes.byref(times)))
            _, whole = self._live.get(rid, (None, None))
        finally:
            self._live.pop(rid, None)
        out = proof.as_dict()
        if whole is not None:
            out["whir_commit_words"], out["whir_proof"] = whole[1], whole[2]
        return out, {"submit_ns": times.submit_ns, "admit_ns": times.admit_ns,
                     "done_ns": times.done_ns, "footprint": times.footprint_bytes}

    def stats(self) -> dict:
        st = ServerStatsC()
        check(lib().pkg_server_get_stats(self._s, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStatsC._fields_}

    def close(self):
        if self._s:
            lib().pkg_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
