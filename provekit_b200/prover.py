"""Prover-level entry points: the synthetic R1CS workload, the Spartan
prove core (provekit/prover/src/whir_r1cs.rs up to WHIR's prove call), the
whole proof with WHIR's rounds (pkg_prove_r1cs) and the two-commitment
proof of an R1CS with verifier challenges (pkg_dual_prove_*)."""
import ctypes

import numpy as np
import torch

from ._lib import check, lib
from .spartan import Transcript


class R1csC(ctypes.Structure):
    _fields_ = [("num_constraints", ctypes.c_size_t), ("num_witnesses", ctypes.c_size_t),
                ("row_ptr", ctypes.c_void_p * 3), ("cols", ctypes.c_void_p * 3),
                ("vals", ctypes.c_void_p * 3), ("nnz", ctypes.c_size_t * 3),
                ("num_public_inputs", ctypes.c_size_t), ("row_ptr_t", ctypes.c_void_p * 3),
                ("cols_t", ctypes.c_void_p * 3), ("vals_t", ctypes.c_void_p * 3)]


class SpartanProofC(ctypes.Structure):
    _fields_ = [("m", ctypes.c_size_t), ("m0", ctypes.c_size_t), ("root", ctypes.c_uint8 * 32),
                ("r", ctypes.c_uint64 * 120), ("coeffs", ctypes.c_uint64 * 480),
                ("alpha", ctypes.c_uint64 * 120), ("rho", ctypes.c_uint64 * 4),
                ("sum_g", ctypes.c_uint64 * 4), ("blinding_eval", ctypes.c_uint64 * 4),
                ("public_x", ctypes.c_uint64 * 4), ("evals", ctypes.c_uint64 * 12),
                ("transcript", Transcript), ("public_hash", ctypes.c_uint64 * 4),
                ("public_eval", ctypes.c_uint64 * 4)]

    def as_dict(self):
        m0 = self.m0
        arr = lambda x, n: np.array(x[: 4 * n], dtype=np.uint64).reshape(n, 4)  # noqa: E731
        return {"m": self.m, "m0": m0, "root": bytes(self.root), "r": arr(self.r, m0),
                "coeffs": arr(self.coeffs, 4 * m0), "alpha": arr(self.alpha, m0),
                "rho": np.array(self.rho, np.uint64), "sum_g": np.array(self.sum_g, np.uint64),
                "blinding_eval": np.array(self.blinding_eval, np.uint64),
                "public_x": np.array(self.public_x, np.uint64), "evals": arr(self.evals, 3),
                "transcript": (list(self.transcript.l), list(self.transcript.r)),
                "public_hash": np.array(self.public_hash, np.uint64),
                "public_eval": np.array(self.public_eval, np.uint64)}


class HostR1CS:
    """Synthetic satisfiable R1CS in host memory (pkg_synthetic_r1cs)."""

    def __init__(self, seed: int, num_constraints: int, num_inputs: int, num_public_inputs: int = 0):
        """num_public_inputs: the first inputs (witness[1 ..= this]) are public."""
        nc, ni = num_constraints, num_inputs
        if num_public_inputs > ni:
            raise ValueError("more public inputs than inputs")
        self.num_constraints, self.num_inputs = nc, ni
        self.num_public_inputs = num_public_inputs
        self.num_witnesses = 1 + ni + nc
        self.row_ptr = [np.zeros(nc + 1, np.uint64) for _ in range(3)]
        caps = [3 * nc, 3 * nc, nc]
        self.cols = [np.zeros(max(c, 1), np.uint32) for c in caps]
        self.vals = [np.zeros((max(c, 1), 4), np.uint64) for c in caps]
        self.witness = np.zeros((self.num_witnesses, 4), np.uint64)
        nnz = (ctypes.c_size_t * 3)()
        rp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.cols])
        vl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.vals])
        check(lib().pkg_synthetic_r1cs(seed, nc, ni, rp, cl, vl, nnz, self.witness.ctypes.data))
        self.nnz = list(nnz)
        self.cols = [np.ascontiguousarray(c[:n]) for c, n in zip(self.cols, self.nnz)]
        self.vals = [np.ascontiguousarray(v[:n]) for v, n in zip(self.vals, self.nnz)]

    def to_device(self, device="cuda", transposes=True):
        return DeviceR1CS(self, device, transposes)


class HostDualR1CS:
    """Synthetic R1CS with verifier challenges in host memory
    (pkg_synthetic_r1cs_dual): w1 = a HostR1CS-like instance of nc1 rows,
    w2 = num_challenges challenges and rows2 products challenge x w1 terms;
    the witness's w2 part is zero until solve() fills it."""

    def __init__(self, seed: int, nc1: int, num_inputs: int, num_challenges: int, rows2: int,
                 num_public_inputs: int = 0):
        if num_public_inputs > num_inputs:
            raise ValueError("more public inputs than inputs")
        nc = nc1 + rows2
        self.num_constraints, self.num_public_inputs, self.first_row = nc, num_public_inputs, nc1
        self.w1_size = 1 + num_inputs + nc1
        self.num_witnesses = self.w1_size + num_challenges + rows2
        self.row_ptr = [np.zeros(nc + 1, np.uint64) for _ in range(3)]
        caps = [3 * nc, 3 * nc, nc]
        cols = [np.zeros(max(c, 1), np.uint32) for c in caps]
        vals = [np.zeros((max(c, 1), 4), np.uint64) for c in caps]
        self.witness = np.zeros((self.num_witnesses, 4), np.uint64)
        offs = np.zeros(max(num_challenges, 1), np.uint64)
        nnz = (ctypes.c_size_t * 3)()
        rp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in cols])
        vl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in vals])
        check(lib().pkg_synthetic_r1cs_dual(seed, nc1, num_inputs, num_challenges, rows2, rp, cl,
                                            vl, nnz, self.witness.ctypes.data, offs.ctypes.data))
        self.challenge_offsets = offs[:num_challenges]
        self.nnz = list(nnz)
        self.cols = [np.ascontiguousarray(c[:n]) for c, n in zip(cols, self.nnz)]
        self.vals = [np.ascontiguousarray(v[:n]) for v, n in zip(vals, self.nnz)]

    def solve(self, challenges) -> np.ndarray:
        """w2 for these challenges ((k, 4) Montgomery words), on the host."""
        w = np.ascontiguousarray(self.witness.copy())
        ch = np.ascontiguousarray(np.asarray(challenges, dtype=np.uint64).reshape(-1, 4))
        k = len(self.challenge_offsets)
        offs = np.ascontiguousarray(self.challenge_offsets, dtype=np.uint64)
        rp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.cols])
        vl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.vals])
        check(lib().pkg_synthetic_dual_solve(self.num_constraints, self.first_row, rp, cl, vl,
                                             self.w1_size, offs.ctypes.data if k else None, k,
                                             ch.ctypes.data if k else None, w.ctypes.data))
        return w[self.w1_size:]

    def to_device(self, device="cuda", transposes=True):
        return DeviceR1CS(self, device, transposes)


class DeviceR1CS:
    """An R1CS resident on the device.  transposes: build A^T, B^T, C^T once
    (pkg_r1cs_build_transposes) so that proofs of this circuit skip the
    per-proof transposes; False leaves them to every proof."""

    def __init__(self, h: HostR1CS, device="cuda", transposes=True):
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(  # noqa: E731
            np.int32 if a.dtype == np.uint32 else np.int64)).to(device)
        self.num_constraints, self.num_witnesses = h.num_constraints, h.num_witnesses
        self.num_public_inputs = getattr(h, "num_public_inputs", 0)
        self.row_ptr = [t(a) for a in h.row_ptr]
        self.cols = [t(a) for a in h.cols]
        self.vals = [t(a) for a in h.vals]
        self.nnz = list(h.nnz)
        self.witness = t(h.witness)
        self.c = R1csC(h.num_constraints, h.num_witnesses,
                       (ctypes.c_void_p * 3)(*[x.data_ptr() for x in self.row_ptr]),
                       (ctypes.c_void_p * 3)(*[x.data_ptr() for x in self.cols]),
                       (ctypes.c_void_p * 3)(*[x.data_ptr() for x in self.vals]),
                       (ctypes.c_size_t * 3)(*self.nnz), self.num_public_inputs)
        self.transposes = None
        if transposes:
            nbytes = lib().pkg_r1cs_transposes_bytes(ctypes.byref(self.c))
            self.transposes = torch.empty(nbytes, dtype=torch.uint8, device=device)
            s = torch.cuda.current_stream(self.transposes.device).cuda_stream
            check(lib().pkg_r1cs_build_transposes(ctypes.byref(self.c),
                                                  self.transposes.data_ptr(), s))


def spartan_prove(r1cs: DeviceR1CS, witness=None, blinding_seed=1, transcript_domain=3,
                  folding_factor=3, log_inv_rate=2, stream=None):
    """pkg_spartan_prove: returns the proof fields as a dict of host values."""
    w = r1cs.witness if witness is None else witness
    out = SpartanProofC()
    s = (stream if stream is not None else torch.cuda.current_stream()).cuda_stream
    check(lib().pkg_spartan_prove(ctypes.byref(r1cs.c), w.data_ptr(), blinding_seed,
                                  transcript_domain, folding_factor, log_inv_rate,
                                  ctypes.byref(out), s))
    return out.as_dict()


def r1cs_sizing(num_constraints: int, num_witnesses: int):
    """(m, m0) of WhirR1CSScheme::new_for_r1cs."""
    m, m0 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    check(lib().pkg_r1cs_sizing(num_constraints, num_witnesses, ctypes.byref(m), ctypes.byref(m0)))
    return m.value, m0.value


def whir_params_for(r1cs, folding_factor=3, log_inv_rate=2, security_bits=128, pow_bits=10,
                    zk=True, **overrides):
    """The WHIR parameters of the R1CS's witness commitment (by default the
    reference's: provekit/r1cs-compiler/src/whir_r1cs.rs:103-118, whir-ZK,
    i.e. the witness committed in a batch of 2 with a blinding polynomial)."""
    from .whir import WhirParams
    m, _ = r1cs_sizing(r1cs.num_constraints, r1cs.num_witnesses)
    if zk:
        overrides.setdefault("batch_size", 2)
    return WhirParams.new(m, folding_factor, log_inv_rate, security_bits, pow_bits, **overrides)


def prove_r1cs(r1cs: DeviceR1CS, whir=None, witness=None, blinding_seed=1, transcript_domain=3,
               stream=None):
    """pkg_prove_r1cs: a whole proof.  Returns (spartan fields dict,
    WHIR commitment words, WHIR proof words)."""
    p = whir_params_for(r1cs) if whir is None else whir
    w = r1cs.witness if witness is None else witness
    out = SpartanProofC()
    cwords = np.zeros(p.commit_words(), np.uint64)
    proof = np.zeros(p.proof_words(statement_count(r1cs)), np.uint64)
    s = (stream if stream is not None else torch.cuda.current_stream()).cuda_stream
    check(lib().pkg_prove_r1cs(ctypes.byref(r1cs.c), w.data_ptr(), blinding_seed,
                               transcript_domain, ctypes.byref(p), ctypes.byref(out),
                               cwords.ctypes.data, proof.ctypes.data, s))
    return out.as_dict(), cwords, proof


def statement_count(r1cs) -> int:
    """The whole proof's WHIR statements (prove_from_alphas,
    provekit/prover/src/whir_r1cs.rs:258-301): the public weight when there
    are public inputs, A^T eq, B^T eq, C^T eq, and the blinding covector."""
    return 4 + (1 if getattr(r1cs, "num_public_inputs", 0) else 0)


class DualProofC(ctypes.Structure):
    _fields_ = [("spartan", SpartanProofC), ("root2", ctypes.c_uint8 * 32),
                ("evals2", ctypes.c_uint64 * 12), ("challenge_eval", ctypes.c_uint64 * 4)]

    def as_dict(self):
        d = self.spartan.as_dict()
        d["root2"] = bytes(self.root2)
        d["evals2"] = np.array(self.evals2, np.uint64).reshape(3, 4)
        d["challenge_eval"] = np.array(self.challenge_eval, np.uint64)
        return d


def r1cs_sizing_split(num_constraints: int, num_witnesses: int, w1_size: int):
    """(m, m0) of WhirR1CSScheme::new_for_r1cs with the witness split at w1_size."""
    m, m0 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    check(lib().pkg_r1cs_sizing_split(num_constraints, num_witnesses, w1_size, ctypes.byref(m),
                                      ctypes.byref(m0)))
    return m.value, m0.value


def dual_statement_counts(num_public_inputs: int, num_challenges: int):
    """WHIR statements of the two proofs (prove_from_alphas's dual branch,
    provekit/prover/src/whir_r1cs.rs:302-425): [public?, A|w1, B|w1, C|w1,
    blinding] and [A|w2, B|w2, C|w2, challenge weight?]."""
    return 4 + (1 if num_public_inputs else 0), 3 + (1 if num_challenges else 0)


def prove_r1cs_dual(r1cs: DeviceR1CS, w1_size: int, challenge_offsets, solve_w2, whir=None,
                    blinding_seed=1, transcript_domain=3, stream=None):
    """A proof of an R1CS with verifier challenges (two commitments):
    pkg_dual_prove_begin commits w1 = the resident witness's first w1_size
    entries and draws the challenges; solve_w2(challenges) -- challenges a
    (k, 4) uint64 array of Montgomery words -- returns w2 (the witness's
    remaining entries: a device tensor or a host array of (n, 4) words, the
    challenge values at challenge_offsets); pkg_dual_prove_finish commits it
    and proves.  Returns (fields dict, challenges, commitment words of w1
    and w2, WHIR proofs 1 and 2)."""
    from .whir import WhirParams
    offs = np.ascontiguousarray(np.asarray(challenge_offsets, dtype=np.uint64).reshape(-1))
    k = offs.shape[0]
    m, _ = r1cs_sizing_split(r1cs.num_constraints, r1cs.num_witnesses, w1_size)
    p = WhirParams.new(m, 3, 2, 128, 10, batch_size=2) if whir is None else whir
    n1, n2 = dual_statement_counts(r1cs.num_public_inputs, k)
    ch = np.zeros((max(k, 1), 4), np.uint64)
    cw1 = np.zeros(p.commit_words(), np.uint64)
    cw2 = np.zeros_like(cw1)
    pr1 = np.zeros(p.proof_words(n1), np.uint64)
    pr2 = np.zeros(p.proof_words(n2), np.uint64)
    st = ctypes.c_void_p()
    strm = stream if stream is not None else torch.cuda.current_stream()
    w = r1cs.witness
    check(lib().pkg_dual_prove_begin(ctypes.byref(r1cs.c), w1_size,
                                     offs.ctypes.data if k else None, k, w.data_ptr(),
                                     blinding_seed, transcript_domain, ctypes.byref(p),
                                     cw1.ctypes.data, ch.ctypes.data, ctypes.byref(st),
                                     strm.cuda_stream))
    try:
        w2 = solve_w2(ch[:k].copy())
        n2w = r1cs.num_witnesses - w1_size
        if not torch.is_tensor(w2):
            w2 = torch.from_numpy(np.ascontiguousarray(w2, dtype=np.uint64).view(np.int64))
        w2 = w2.reshape(-1, 4).to(w.device).contiguous()
        if w2.shape[0] != n2w:
            raise ValueError(f"w2 has {w2.shape[0]} entries, the R1CS needs {n2w}")
        out = DualProofC()
        strm.wait_stream(torch.cuda.current_stream())
        check(lib().pkg_dual_prove_finish(st, w2.data_ptr() if n2w else None, ctypes.byref(out),
                                          cw2.ctypes.data, pr1.ctypes.data, pr2.ctypes.data))
    finally:
        lib().pkg_dual_prove_free(st)
    return out.as_dict(), ch[:k], cw1, cw2, pr1, pr2
