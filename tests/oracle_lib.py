"""ctypes binding of the C oracle (oracle/libpk_oracle.so).  Test
infrastructure: used only to check the CUDA path and as the timed CPU
baseline."""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle.build import build as _build_oracle  # noqa: E402

_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_sz = ctypes.c_size_t

class Transcript(ctypes.Structure):
    _fields_ = [("l", ctypes.c_uint64 * 4), ("r", ctypes.c_uint64 * 4)]


class R1CS(ctypes.Structure):
    _fields_ = [("num_constraints", ctypes.c_size_t), ("num_witnesses", ctypes.c_size_t),
                ("row_ptr", ctypes.c_void_p * 3), ("cols", ctypes.c_void_p * 3),
                ("vals", ctypes.c_void_p * 3), ("num_public_inputs", ctypes.c_size_t)]


class SpartanProof(ctypes.Structure):
    _fields_ = [("m", ctypes.c_size_t), ("m0", ctypes.c_size_t), ("root", ctypes.c_uint8 * 32),
                ("r", ctypes.c_uint64 * 120), ("coeffs", ctypes.c_uint64 * 480),
                ("alpha", ctypes.c_uint64 * 120), ("rho", ctypes.c_uint64 * 4),
                ("sum_g", ctypes.c_uint64 * 4), ("blinding_eval", ctypes.c_uint64 * 4),
                ("public_x", ctypes.c_uint64 * 4), ("evals", ctypes.c_uint64 * 12),
                ("transcript", Transcript), ("public_hash", ctypes.c_uint64 * 4),
                ("public_eval", ctypes.c_uint64 * 4)]


def _r1cs_c(h):
    return R1CS(h.num_constraints, h.num_witnesses,
                (ctypes.c_void_p * 3)(*[a.ctypes.data for a in h.row_ptr]),
                (ctypes.c_void_p * 3)(*[a.ctypes.data for a in h.cols]),
                (ctypes.c_void_p * 3)(*[a.ctypes.data for a in h.vals]),
                getattr(h, "num_public_inputs", 0))


def statement_count(h) -> int:
    """The whole proof's WHIR statements: [public?, A, B, C, blinding]."""
    return 4 + (1 if getattr(h, "num_public_inputs", 0) else 0)


def spartan_prove(h, blinding_seed, domain, ff, lr):
    """Run pko_spartan_prove on a HostR1CS-like object; returns the proof dict."""
    r = _r1cs_c(h)
    out = SpartanProof()
    rc = lib().pko_spartan_prove(ctypes.byref(r), p64(np.ascontiguousarray(h.witness)), blinding_seed,
                                 domain, ff, lr, ctypes.byref(out))
    assert rc == 0, rc
    return _spartan_dict(out)


class SyntheticR1CS:
    """The synthetic satisfiable R1CS of the prove workload, generated by the
    oracle (pko_synthetic_r1cs) without loading the CUDA library; the same
    attributes as provekit_b200.prover.HostR1CS."""

    def __init__(self, seed: int, num_constraints: int, num_inputs: int,
                 num_public_inputs: int = 0):
        nc, ni = num_constraints, num_inputs
        if num_public_inputs > ni:
            raise ValueError("more public inputs than inputs")
        self.num_constraints, self.num_inputs = nc, ni
        self.num_public_inputs = num_public_inputs
        self.num_witnesses = 1 + ni + nc
        self.row_ptr = [np.zeros(nc + 1, np.uint64) for _ in range(3)]
        caps = [3 * nc, 3 * nc, nc]
        cols = [np.zeros(max(c, 1), np.uint32) for c in caps]
        vals = [np.zeros((max(c, 1), 4), np.uint64) for c in caps]
        self.witness = np.zeros((self.num_witnesses, 4), np.uint64)
        nnz = (ctypes.c_size_t * 3)()
        rp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in cols])
        vl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in vals])
        rc = lib().pko_synthetic_r1cs(seed, nc, ni, rp, cl, vl, nnz, p64(self.witness))
        assert rc == 0, rc
        self.nnz = list(nnz)
        self.cols = [np.ascontiguousarray(c[:n]) for c, n in zip(cols, self.nnz)]
        self.vals = [np.ascontiguousarray(v[:n]) for v, n in zip(vals, self.nnz)]


def r1cs_sizing(nc, nw):
    m, m0 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    lib().pko_r1cs_sizing(nc, nw, ctypes.byref(m), ctypes.byref(m0))
    return m.value, m0.value


def prove_r1cs(h, blinding_seed, domain, wp):
    """pko_prove_r1cs: (spartan dict, WHIR commitment words, WHIR proof)."""
    r = _r1cs_c(h)
    out = SpartanProof()
    cwords = np.zeros(lib().pko_whir_commit_words(ctypes.byref(wp)), np.uint64)
    proof = np.zeros(lib().pko_whir_proof_words(ctypes.byref(wp), statement_count(h)), np.uint64)
    rc = lib().pko_prove_r1cs(ctypes.byref(r), p64(np.ascontiguousarray(h.witness)), blinding_seed,
                              domain, ctypes.byref(wp), ctypes.byref(out), p64(cwords), p64(proof))
    assert rc == 0, rc
    return _spartan_dict(out), cwords, proof


class DualProof(ctypes.Structure):
    _fields_ = [("spartan", SpartanProof), ("root2", ctypes.c_uint8 * 32),
                ("evals2", ctypes.c_uint64 * 12), ("challenge_eval", ctypes.c_uint64 * 4)]


def dual_dict(out):
    d = _spartan_dict(out.spartan)
    d["root2"] = bytes(out.root2)
    d["evals2"] = np.array(out.evals2, np.uint64).reshape(3, 4)
    d["challenge_eval"] = np.array(out.challenge_eval, np.uint64)
    return d


class SyntheticDualR1CS:
    """pko_synthetic_r1cs_dual: w1 = the synthetic R1CS of nc1 rows over ni
    inputs, w2 = num_challenges challenges spread over it plus rows2 products
    challenge x w1 terms; the witness's w2 part is zero until solve()."""

    def __init__(self, seed: int, nc1: int, ni: int, num_challenges: int, rows2: int,
                 num_public_inputs: int = 0):
        nc = nc1 + rows2
        self.num_constraints, self.num_public_inputs = nc, num_public_inputs
        self.w1_size = 1 + ni + nc1
        self.num_witnesses = self.w1_size + num_challenges + rows2
        self.first_row = nc1
        self.row_ptr = [np.zeros(nc + 1, np.uint64) for _ in range(3)]
        caps = [3 * nc, 3 * nc, nc]
        cols = [np.zeros(max(c, 1), np.uint32) for c in caps]
        vals = [np.zeros((max(c, 1), 4), np.uint64) for c in caps]
        self.witness = np.zeros((self.num_witnesses, 4), np.uint64)
        self.challenge_offsets = np.zeros(max(num_challenges, 1), np.uint64)
        nnz = (ctypes.c_size_t * 3)()
        rp = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in self.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in cols])
        vl = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in vals])
        rc = lib().pko_synthetic_r1cs_dual(seed, nc1, ni, num_challenges, rows2, rp, cl, vl, nnz,
                                           p64(self.witness), p64(self.challenge_offsets))
        assert rc == 0, rc
        self.challenge_offsets = self.challenge_offsets[:num_challenges]
        self.nnz = list(nnz)
        self.cols = [np.ascontiguousarray(c[:n]) for c, n in zip(cols, self.nnz)]
        self.vals = [np.ascontiguousarray(v[:n]) for v, n in zip(vals, self.nnz)]

    def solver_ctx(self):
        """(pko_synthetic_dual, the objects it points into) for pko_prove_r1cs_dual."""
        r = _r1cs_c(self)
        offs = np.ascontiguousarray(self.challenge_offsets, dtype=np.uint64)
        ctx = SyntheticDual(ctypes.pointer(r), self.w1_size, self.first_row,
                            offs.ctypes.data if offs.size else None)
        return ctx, (r, offs)

    def solve(self, challenges: np.ndarray) -> np.ndarray:
        """w2 for these challenges (num_challenges x 4 Montgomery words)."""
        w = np.ascontiguousarray(self.witness.copy())
        ctx, keep = self.solver_ctx()
        ch = np.ascontiguousarray(challenges, dtype=np.uint64).reshape(-1, 4)
        lib().pko_synthetic_dual_solve(ctypes.byref(ctx), p64(ch) if ch.size else None,
                                       len(self.challenge_offsets), p64(w))
        del keep
        return w[self.w1_size:]


class SyntheticDual(ctypes.Structure):
    _fields_ = [("r1cs", ctypes.POINTER(R1CS)), ("w1_size", ctypes.c_size_t),
                ("first_row", ctypes.c_size_t), ("challenge_offsets", ctypes.c_void_p)]


def r1cs_sizing_split(nc, nw, w1_size):
    m, m0 = ctypes.c_size_t(0), ctypes.c_size_t(0)
    lib().pko_r1cs_sizing_split(nc, nw, w1_size, ctypes.byref(m), ctypes.byref(m0))
    return m.value, m0.value


def dual_statement_counts(h):
    npub = getattr(h, "num_public_inputs", 0)
    return 4 + (1 if npub else 0), 3 + (1 if len(h.challenge_offsets) else 0)


def prove_r1cs_dual(h, blinding_seed, domain, wp):
    """pko_prove_r1cs_dual with the instance's own solver: (dual dict,
    challenges, commit words 1 and 2, proofs 1 and 2, the solved witness)."""
    n1, n2 = dual_statement_counts(h)
    r = _r1cs_c(h)
    ctx, keep = h.solver_ctx()
    out = DualProof()
    k = len(h.challenge_offsets)
    ch = np.zeros((max(k, 1), 4), np.uint64)
    cw1 = np.zeros(lib().pko_whir_commit_words(ctypes.byref(wp)), np.uint64)
    cw2 = np.zeros_like(cw1)
    pr1 = np.zeros(lib().pko_whir_proof_words(ctypes.byref(wp), n1), np.uint64)
    pr2 = np.zeros(lib().pko_whir_proof_words(ctypes.byref(wp), n2), np.uint64)
    w = np.ascontiguousarray(h.witness.copy())
    offs = np.zeros(max(k, 1), np.uint64)
    offs[:k] = h.challenge_offsets
    solve = ctypes.cast(lib().pko_synthetic_dual_solve, ctypes.c_void_p)
    rc = lib().pko_prove_r1cs_dual(ctypes.byref(r), h.w1_size, p64(offs), k, p64(w), solve,
                                   ctypes.byref(ctx), blinding_seed, domain, ctypes.byref(wp),
                                   ctypes.byref(out), p64(ch), p64(cw1), p64(cw2), p64(pr1),
                                   p64(pr2))
    del keep
    assert rc == 0, rc
    return dual_dict(out), ch[:k], cw1, cw2, pr1, pr2, w


MONT_ONE = np.array([0xac96341c4ffffffb, 0x36fc76959f60cd29, 0x666ea36f7879462e,
                     0x0e0a77c19a07df2f], np.uint64)  # 2^256 mod p


def _powers(x, n):
    out = np.zeros((n, 4), np.uint64)
    if n:
        out[0] = MONT_ONE
    for i in range(1, n):
        lib().pko_fr_mul(p64(out[i]), p64(out[i - 1]), p64(np.ascontiguousarray(x, np.uint64)))
    return out


def dual_statement_covectors(h, d):
    """(w1's statements, w2's statements) of a dual proof, as the verifier
    builds them from the transcript's alpha and x: [public?, A|w1, B|w1,
    C|w1, blinding] and [A|w2, B|w2, C|w2, challenge weight?]."""
    n, m0, w1 = 1 << d["m"], d["m0"], h.w1_size
    nw = h.num_witnesses
    full = r1cs_covectors(h, d["alpha"], m0, nw).reshape(3, nw, 4)
    npub = getattr(h, "num_public_inputs", 0)
    n1, n2 = dual_statement_counts(h)
    s1 = np.zeros((n1, n, 4), np.uint64)
    b = 1 if npub else 0
    if npub:
        s1[0, : npub + 1] = _powers(d["public_x"], npub + 1)
    s1[b: b + 3, :w1] = full[:, :w1]
    for i in range(m0):
        s1[b + 3, w1 + 4 * i: w1 + 4 * i + 4] = _powers(d["alpha"][i], 4)
    s2 = np.zeros((n2, n, 4), np.uint64)
    s2[:3, : nw - w1] = full[:, w1:]
    if n2 == 4:
        pw = _powers(d["public_x"], len(h.challenge_offsets))
        for j, o in enumerate(h.challenge_offsets):
            e = np.ascontiguousarray(s2[3, int(o)])
            lib().pko_fr_add(p64(e), p64(e.copy()), p64(pw[j]))
            s2[3, int(o)] = e
    return s1.reshape(-1, 4), s2.reshape(-1, 4)


def verify_r1cs_dual(h, wp, domain, d, challenges, cw1, cw2, pr1, pr2):
    """0 when a dual proof is accepted: both commitments with the challenges
    between them on a fresh transcript, both WHIR proofs from the state the
    first WHIR prover started from, each proof's claimed statement values
    equal to the Spartan messages, and the challenge binding
    <[1, x, ..], challenges> = the challenge evaluation.  Else a negative
    WHIR code, or 1 (wrong challenges), 2 (values differ), 3 (binding)."""
    t0 = transcript(domain)
    z1, z2 = np.zeros((5, 4), np.uint64), np.zeros((5, 4), np.uint64)
    rc = lib().pko_whir_verify_commit(ctypes.byref(wp), ctypes.byref(t0), p64(cw1), p64(z1))
    if rc:
        return rc
    k = len(h.challenge_offsets)
    got = np.zeros((max(k, 1), 4), np.uint64)
    for j in range(k):
        lib().pko_transcript_squeeze(ctypes.byref(t0), p64(got[j]))
    if not np.array_equal(got[:k], np.asarray(challenges).reshape(-1, 4)[:k]):
        return 1
    rc = lib().pko_whir_verify_commit(ctypes.byref(wp), ctypes.byref(t0), p64(cw2), p64(z2))
    if rc:
        return rc
    t = Transcript()
    t.l[:], t.r[:] = d["transcript"]
    s1, s2 = dual_statement_covectors(h, d)
    n = 1 << d["m"]
    n1, n2 = s1.shape[0] // n, s2.shape[0] // n
    for s, nc, cw, z, pr in ((s1, n1, cw1, z1, pr1), (s2, n2, cw2, z2, pr2)):
        rc = lib().pko_whir_verify_proof(ctypes.byref(wp), ctypes.byref(t), p64(s), nc, p64(cw),
                                         p64(z), p64(np.ascontiguousarray(pr)), pr.shape[0])
        if rc:
            return rc
    npub = getattr(h, "num_public_inputs", 0)
    want1 = ([d["public_eval"]] if npub else []) + list(d["evals"]) + [d["blinding_eval"]]
    want2 = list(d["evals2"]) + ([d["challenge_eval"]] if k else [])
    if not (np.array_equal(pr1[: 4 * n1].reshape(-1, 4), np.array(want1, np.uint64))
            and np.array_equal(pr2[: 4 * n2].reshape(-1, 4), np.array(want2, np.uint64))):
        return 2
    if k:
        pw = _powers(d["public_x"], k)
        acc = np.zeros(4, np.uint64)
        for j in range(k):
            x = np.zeros(4, np.uint64)
            lib().pko_fr_mul(p64(x), p64(pw[j]), p64(np.ascontiguousarray(got[j])))
            lib().pko_fr_add(p64(acc), p64(acc.copy()), p64(x))
        if not np.array_equal(acc, d["challenge_eval"]):
            return 3
    return 0


def r1cs_covectors(h, alpha, m0, length):
    out = np.zeros((3 * length, 4), np.uint64)
    rc = lib().pko_r1cs_covectors(ctypes.byref(_r1cs_c(h)), p64(np.ascontiguousarray(alpha)), m0,
                                  length, p64(out))
    assert rc == 0
    return out


def verify_r1cs_whir(h, wp, domain, spartan, cwords, proof):
    """The WHIR part of a whole proof: the commitment half on a fresh
    transcript, the proof half from the state the WHIR prover started from."""
    t0 = transcript(domain)
    z = np.zeros((5, 4), np.uint64)
    rc = lib().pko_whir_verify_commit(ctypes.byref(wp), ctypes.byref(t0), p64(cwords), p64(z))
    if rc:
        return rc
    t = Transcript()
    l, r = spartan["transcript"]
    t.l[:] = l
    t.r[:] = r
    cov = statement_covectors(h, spartan)
    return lib().pko_whir_verify_proof(ctypes.byref(wp), ctypes.byref(t), p64(cov),
                                       cov.shape[0] >> spartan["m"], p64(cwords), p64(z),
                                       p64(np.ascontiguousarray(proof)), proof.shape[0])


def statement_covectors(h, spartan):
    """[public?, A^T eq, B^T eq, C^T eq, blinding] as (ncov * 2^m, 4)."""
    n = 1 << spartan["m"]
    out = np.zeros((5 * n, 4), np.uint64)
    px = np.ascontiguousarray(spartan["public_x"], dtype=np.uint64)
    ncov = lib().pko_r1cs_statement_covectors(ctypes.byref(_r1cs_c(h)), p64(px),
                                              p64(np.ascontiguousarray(spartan["alpha"])),
                                              spartan["m0"], h.num_witnesses, n, p64(out))
    assert ncov > 0
    return out[: ncov * n]


def _spartan_dict(out):
    m0 = out.m0
    arr = lambda x, n: np.array(x[: 4 * n], dtype=np.uint64).reshape(n, 4)  # noqa: E731
    return {"m": out.m, "m0": m0, "root": bytes(out.root), "r": arr(out.r, m0),
            "coeffs": arr(out.coeffs, 4 * m0), "alpha": arr(out.alpha, m0),
            "rho": np.array(out.rho, np.uint64), "sum_g": np.array(out.sum_g, np.uint64),
            "blinding_eval": np.array(out.blinding_eval, np.uint64),
            "public_x": np.array(out.public_x, np.uint64), "evals": arr(out.evals, 3),
            "transcript": (list(out.transcript.l), list(out.transcript.r)),
            "public_hash": np.array(out.public_hash, np.uint64),
            "public_eval": np.array(out.public_eval, np.uint64)}


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(_build_oracle())
        L = _lib
        L.pko_fr_mul.argtypes = [_u64p, _u64p, _u64p]
        L.pko_sample_fr.argtypes = [ctypes.c_uint64, _sz, _u64p, ctypes.c_int]
        L.pko_sample_fr_indexed.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _sz, _u64p]
        L.pko_ntt_nr.argtypes = [_u64p, _sz, _sz, _sz]
        L.pko_intt_rn.argtypes = [_u64p, _sz]
        L.pko_roots_reverse_ordered.argtypes = [_u64p, _sz]
        L.pko_rs_interleaved_encode.argtypes = [_u64p, _sz, _sz, _u64p, _sz, _sz, _u64p]
        L.pko_rs_evaluation_points.argtypes = [_sz, ctypes.POINTER(_sz), _sz, _u64p]
        L.pko_sky_compress.argtypes = [_u64p, _u64p, _u64p]
        L.pko_sky_compress_many.argtypes = [_u8p, _sz, _u8p]
        L.pko_sky_permute.argtypes = [_u64p, _u64p]
        L.pko_sky_ss.argtypes = [ctypes.c_int, _u64p, _u64p]
        L.pko_sky_bb.argtypes = [ctypes.c_int, _u64p, _u64p]
        L.pko_sky_sbox.argtypes = [ctypes.c_uint8]
        L.pko_sky_sbox.restype = ctypes.c_uint8
        L.pko_hash_many.argtypes = [_sz, _u8p, _sz, _u8p]
        L.pko_merkle_tree.argtypes = [_u8p, _sz, _sz, _u8p]
        L.pko_sky_pow_solve.argtypes = [_u64p, _u64p]
        L.pko_sky_pow_solve.restype = ctypes.c_uint64
        L.pko_calculate_eq.argtypes = [_u64p, _u64p, _u64p, _sz]
        L.pko_eq_hypercube.argtypes = [_u64p, _sz, _sz, _u64p]
        L.pko_spartan_round.argtypes = [_u64p, _u64p, _u64p, _u64p, _sz, _u64p, _u64p]
        L.pko_spmv.argtypes = [_u64p, _u32p, _u64p, _sz, _u64p, _u64p]
        L.pko_eval_cubic.argtypes = [_u64p, _u64p, _u64p]
        L.pko_blinding_coeffs.argtypes = [_u64p, _sz, _sz, _u64p, _u64p]
        L.pko_dot.argtypes = [_u64p, _u64p, _u64p, _sz]
        L.pko_num_threads.restype = ctypes.c_int
        tp = ctypes.POINTER(Transcript)
        L.pko_transcript_init.argtypes = [tp, _u64p]
        L.pko_transcript_absorb.argtypes = [tp, _u64p]
        L.pko_transcript_squeeze.argtypes = [tp, _u64p]
        L.pko_spartan_sumcheck.argtypes = [tp, _u64p, _u64p, _u64p, _sz, _u64p, _u64p, _sz,
                                           _u64p, _u64p, _u64p, _u64p, _u64p, _u64p]
        L.pko_from_mont_many.argtypes = [_u64p, _sz]
        L.pko_to_mont_many.argtypes = [_u64p, _sz]
        L.pko_poseidon2_permutation.argtypes = [_u64p]
        L.pko_poseidon2_hash.argtypes = [_u64p, _u64p, _sz]
        L.pko_spartan_prove.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.c_uint, ctypes.c_uint, ctypes.c_void_p]
        L.pko_multilinear_weights.argtypes = [_u64p, _u64p, ctypes.c_uint]
        L.pko_whir_fold_coeffs.argtypes = [_u64p, _sz, ctypes.c_uint, _u64p, _u64p]
        L.pko_whir_fold_rows.argtypes = [_u64p, _sz, ctypes.c_uint, _u64p, _u64p]
        L.pko_poly_eval.argtypes = [_u64p, _u64p, _sz, _u64p]
        L.pko_expand_from_univariate.argtypes = [_u64p, _u64p, _sz]
        L.pko_merkle_open.argtypes = [_u8p, _sz, ctypes.c_uint64, _u8p]
        L.pko_merkle_verify.argtypes = [_u64p, _sz, ctypes.c_uint64, _u8p, _sz, _u8p]
        L.pko_stir_indices.argtypes = [_u8p, _sz, _sz, _u64p]
        L.pko_whir_sumcheck_round.argtypes = [_u64p, _u64p, _sz, _u64p, _u64p]
        L.pko_eq_accumulate.argtypes = [_u64p, _sz, _u64p, _u64p, _sz]
        wp = ctypes.POINTER(WhirParams)
        L.pko_whir_params_init.argtypes = [wp] + [ctypes.c_uint] * 5
        L.pko_whir_commit_words.argtypes = [wp]
        L.pko_whir_commit_words.restype = _sz
        L.pko_whir_proof_words.argtypes = [wp, _sz]
        L.pko_whir_proof_words.restype = _sz
        L.pko_transcript_squeeze_bytes.argtypes = [tp, _u8p, _sz]
        L.pko_subset_zeta.argtypes = [_u64p, ctypes.c_uint]
        L.pko_subset_mobius_t.argtypes = [_u64p, ctypes.c_uint]
        L.pko_whir_commit.argtypes = [_u64p, _sz, ctypes.c_uint, ctypes.c_uint, _u64p, _u8p]
        L.pko_whir_commit_ood.argtypes = [wp, tp, _u64p, _u8p, _u64p, _u64p]
        L.pko_whir_prove.argtypes = [wp, tp, _u64p, _u64p, _u8p, _u64p, _u64p, _u64p, _sz, _u64p]
        L.pko_whir_verify.argtypes = [wp, tp, _u64p, _sz, _u64p, _u64p, _sz]
        L.pko_whir_verify_commit.argtypes = [wp, tp, _u64p, _u64p]
        L.pko_whir_verify_proof.argtypes = [wp, tp, _u64p, _sz, _u64p, _u64p, _u64p, _sz]
        L.pko_r1cs_sizing.argtypes = [_sz, _sz, ctypes.POINTER(_sz), ctypes.POINTER(_sz)]
        L.pko_synthetic_r1cs.argtypes = [ctypes.c_uint64, _sz, _sz, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _u64p]
        L.pko_r1cs_covectors.argtypes = [ctypes.c_void_p, _u64p, _sz, _sz, _u64p]
        L.pko_r1cs_statement_covectors.argtypes = [ctypes.c_void_p, _u64p, _u64p, _sz, _sz, _sz,
                                                   _u64p]
        L.pko_public_inputs_hash.argtypes = [_u64p, _u64p, _sz]
        L.pko_prove_r1cs.argtypes = [ctypes.c_void_p, _u64p, ctypes.c_uint64, ctypes.c_uint64, wp,
                                     ctypes.c_void_p, _u64p, _u64p]
        L.pko_fr_add.argtypes = [_u64p, _u64p, _u64p]
        L.pko_r1cs_sizing_split.argtypes = [_sz, _sz, _sz, ctypes.POINTER(_sz),
                                            ctypes.POINTER(_sz)]
        L.pko_synthetic_r1cs_dual.argtypes = [ctypes.c_uint64, _sz, _sz, _sz, _sz,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_void_p, _u64p, _u64p]
        L.pko_synthetic_dual_solve.argtypes = [ctypes.c_void_p, _u64p, _sz, _u64p]
        L.pko_prove_r1cs_dual.argtypes = [ctypes.c_void_p, _sz, _u64p, _sz, _u64p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.c_uint64, wp, ctypes.c_void_p, _u64p, _u64p,
                                          _u64p, _u64p, _u64p]
    return _lib


# ---- WHIR round orchestration ---------------------------------------------
WHIR_MAX_ROUNDS = 16
WHIR_REJECT = {-1: "bad params", -2: "format", -3: "sumcheck", -4: "pow", -5: "merkle",
               -6: "final poly", -7: "final claim"}


class WhirParams(ctypes.Structure):
    _fields_ = [("num_variables", ctypes.c_uint32), ("folding_factor", ctypes.c_uint32),
                ("log_inv_rate", ctypes.c_uint32), ("num_rounds", ctypes.c_uint32),
                ("final_vars", ctypes.c_uint32), ("ood_samples", ctypes.c_uint32),
                ("pow_bits", ctypes.c_uint32), ("final_pow_bits", ctypes.c_uint32),
                ("batch_size", ctypes.c_uint32),
                ("queries", ctypes.c_uint32 * (WHIR_MAX_ROUNDS + 1))]


def whir_params(n: int, k: int, log_inv_rate: int, security: int, pow_bits: int, **over) -> WhirParams:
    p = WhirParams()
    assert lib().pko_whir_params_init(ctypes.byref(p), n, k, log_inv_rate, security, pow_bits) == 0
    for key, v in over.items():
        if key == "queries":
            for i, q in enumerate(v):
                p.queries[i] = q
        else:
            setattr(p, key, v)
    return p


def transcript(domain: int) -> Transcript:
    t = Transcript()
    d = np.array([domain, 0, 0, 0], np.uint64)
    lib().pko_transcript_init(ctypes.byref(t), p64(d))
    return t


def whir_commit(coeffs: np.ndarray, k: int, log_inv_rate: int):
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(-1, 4)
    L = (c.shape[0] >> k) << log_inv_rate
    cw = np.zeros(((c.shape[0] << log_inv_rate), 4), np.uint64)
    layers = np.zeros((2 * L - 1) * 32, np.uint8)
    assert lib().pko_whir_commit(p64(c), c.shape[0], k, log_inv_rate, p64(cw), p8(layers)) == 0
    return cw, layers


def batch_log(p) -> int:
    return {1: 0, 2: 1, 4: 2}[p.batch_size]


def whir_prove(p: WhirParams, domain: int, coeffs: np.ndarray, covectors: np.ndarray):
    """Commit + prove with a fresh transcript; returns (commit_words, proof).
    coeffs: batch_size x 2^n (the batch's polynomials concatenated)."""
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(-1, 4)
    cov = np.ascontiguousarray(covectors, dtype=np.uint64).reshape(-1, 4)
    ncov = cov.shape[0] >> p.num_variables
    cw, layers = whir_commit(c, p.folding_factor + batch_log(p), p.log_inv_rate)
    root = np.ascontiguousarray(layers[-32:])
    t = transcript(domain)
    cwords = np.zeros(lib().pko_whir_commit_words(ctypes.byref(p)), np.uint64)
    ood = np.zeros((p.ood_samples + 1, 4), np.uint64)
    assert lib().pko_whir_commit_ood(ctypes.byref(p), ctypes.byref(t), p64(c), p8(root),
                                     p64(cwords), p64(ood)) == 0
    proof = np.zeros(lib().pko_whir_proof_words(ctypes.byref(p), ncov), np.uint64)
    cov_arg = p64(cov) if ncov else None
    rc = lib().pko_whir_prove(ctypes.byref(p), ctypes.byref(t), p64(c), p64(cw), p8(layers),
                              p64(cwords), p64(ood), cov_arg, ncov, p64(proof))
    assert rc == 0, rc
    return cwords, proof


def whir_verify(p: WhirParams, domain: int, covectors: np.ndarray, ncov: int,
                commit_words: np.ndarray, proof: np.ndarray) -> int:
    cov = np.ascontiguousarray(covectors, dtype=np.uint64).reshape(-1, 4)
    t = transcript(domain)
    cw = np.ascontiguousarray(commit_words, dtype=np.uint64)
    pr = np.ascontiguousarray(proof, dtype=np.uint64)
    return lib().pko_whir_verify(ctypes.byref(p), ctypes.byref(t), p64(cov) if ncov else None, ncov,
                                 p64(cw), p64(pr), pr.shape[0])


# ---- WHIR prove-round building blocks ------------------------------------
def whir_fold_coeffs(coeffs: np.ndarray, k: int, alpha: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(-1, 4)
    out = np.zeros((max(c.shape[0] >> k, 1), 4), np.uint64)
    assert lib().pko_whir_fold_coeffs(p64(c), c.shape[0], k, p64(np.ascontiguousarray(alpha)),
                                      p64(out)) == 0
    return out


def whir_fold_rows(rows: np.ndarray, k: int, alpha: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(rows, dtype=np.uint64).reshape(-1, 4)
    n = r.shape[0] >> k
    out = np.zeros((max(n, 1), 4), np.uint64)
    assert lib().pko_whir_fold_rows(p64(r), n, k, p64(np.ascontiguousarray(alpha)), p64(out)) == 0
    return out[:n]


def poly_eval(coeffs: np.ndarray, z: np.ndarray) -> np.ndarray:
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(-1, 4)
    out = np.zeros(4, np.uint64)
    lib().pko_poly_eval(p64(out), p64(c), c.shape[0], p64(np.ascontiguousarray(z, dtype=np.uint64)))
    return out


def merkle_open(layers: bytes, num_leaves: int, idx: int) -> bytes:
    lay = np.frombuffer(layers, dtype=np.uint8).copy()
    depth = num_leaves.bit_length() - 1
    out = np.zeros(max(32 * depth, 1), np.uint8)
    assert lib().pko_merkle_open(p8(lay), num_leaves, idx, p8(out)) == 0
    return out[: 32 * depth].tobytes()


def whir_sumcheck_round(f: np.ndarray, w: np.ndarray, size: int, fold=None) -> np.ndarray:
    out = np.zeros(12, np.uint64)
    fd = None if fold is None else p64(np.ascontiguousarray(fold, dtype=np.uint64))
    assert lib().pko_whir_sumcheck_round(p64(f), p64(w), size, fd, p64(out)) == 0
    return out.reshape(3, 4)


def p64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def p8(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


def p32(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def sample_fr(seed: int, n: int, mont: bool = True) -> np.ndarray:
    out = np.zeros((max(n, 1), 4), dtype=np.uint64)
    lib().pko_sample_fr(seed, n, p64(out), int(mont))
    return out[:n]


def ntt_nr(values: np.ndarray, codeword_size: int, num_groups: int) -> int:
    v = values.reshape(-1, 4)
    return lib().pko_ntt_nr(p64(v), v.shape[0], codeword_size, num_groups)


def intt_rn(values: np.ndarray) -> int:
    v = values.reshape(-1, 4)
    return lib().pko_intt_rn(p64(v), v.shape[0])


def roots(order: int) -> np.ndarray:
    out = np.zeros((max(order // 2, 1), 4), dtype=np.uint64)
    lib().pko_roots_reverse_ordered(p64(out), order)
    return out[: order // 2]


def rs_interleaved_encode(messages: np.ndarray, masks: np.ndarray, codeword_length: int):
    """messages: (M, L, 4) uint64; masks: (k, 4).  Returns (rc, out)."""
    M, L = messages.shape[0], messages.shape[1]
    out = np.zeros((max(M * codeword_length, 1), 4), dtype=np.uint64)
    msg = np.ascontiguousarray(messages.reshape(-1, 4)) if messages.size else np.zeros((1, 4), np.uint64)
    mk = np.ascontiguousarray(masks.reshape(-1, 4)) if masks.size else np.zeros((1, 4), np.uint64)
    rc = lib().pko_rs_interleaved_encode(p64(msg), M, L, p64(mk), masks.reshape(-1, 4).shape[0],
                                         codeword_length, p64(out))
    return rc, out[: M * codeword_length]


def hash_many(size: int, data: bytes, count: int) -> bytes:
    inp = np.frombuffer(data, dtype=np.uint8).copy() if len(data) else np.zeros(1, np.uint8)
    out = np.zeros(max(32 * count, 1), dtype=np.uint8)
    rc = lib().pko_hash_many(size, p8(inp), count, p8(out))
    assert rc == 0, rc
    return out[: 32 * count].tobytes()


def merkle_tree(leaves: bytes, leaf_size: int, count: int) -> bytes:
    inp = np.frombuffer(leaves, dtype=np.uint8).copy()
    out = np.zeros(32 * (2 * count - 1), dtype=np.uint8)
    rc = lib().pko_merkle_tree(p8(inp), leaf_size, count, p8(out))
    assert rc == 0, rc
    return out.tobytes()


def compress(l, r):
    a = np.array(l, dtype=np.uint64)
    b = np.array(r, dtype=np.uint64)
    o = np.zeros(4, dtype=np.uint64)
    lib().pko_sky_compress(p64(o), p64(a), p64(b))
    return [int(x) for x in o]
