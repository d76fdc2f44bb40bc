"""CPU tests of the oracle's whole WHIR proof (pk_oracle_whir.c).

The prover and the verifier are both restatements: the round order is the
reference's Go verifier runWhir (recursive-verifier/app/circuit/whir.go:587-724),
its checks CheckSumOverBool, the Merkle path walk, CheckPoW, the final
UnivarPoly == computeFold comparison and lastEval == W(r) f(r).  These tests
pin the pair against each other: honest proofs are accepted for many shapes,
and a mistake planted in any section of a proof, in the statement or in the
transcript is rejected by the check that guards it.
"""
import numpy as np
import pytest

import oracle_lib as O


def layout(p, ncov):
    """Word offsets of every section of a proof (the order pko_whir_prove writes)."""
    k, K, o = p.folding_factor, 1 << p.folding_factor, p.ood_samples
    n, lr, B = p.num_variables, p.log_inv_rate, p.batch_size
    pos = 0
    out = {"values": pos}
    pos += 4 * ncov * B
    out["sc0"] = pos
    pos += 12 * k
    rounds = []
    for r in range(p.num_rounds):
        d = {"root": pos}
        pos += 4
        d["ood"] = pos
        pos += 4 * o
        if p.pow_bits:
            d["pow"] = pos
            pos += 1
        depth = n + lr - k - r
        d["open"] = pos
        d["row_words"], d["path_words"] = 4 * K * (B if r == 0 else 1), 4 * depth
        pos += p.queries[r] * (d["row_words"] + 4 * depth)
        d["sc"] = pos
        pos += 12 * k
        rounds.append(d)
    out["rounds"] = rounds
    R = p.num_rounds
    fin = {"coeffs": pos}
    pos += 4 << p.final_vars
    if p.final_pow_bits:
        fin["pow"] = pos
        pos += 1
    depth = n + lr - k - R
    fin["open"] = pos
    fin["row_words"], fin["path_words"] = 4 * K * (B if R == 0 else 1), 4 * depth
    pos += p.queries[R] * (fin["row_words"] + 4 * depth)
    fin["sc"] = pos
    pos += 12 * p.final_vars
    out["final"] = fin
    out["total"] = pos
    return out


CASES = [
    # n, k, log_inv_rate, security, pow, overrides
    (6, 2, 1, 24, 0, {}),
    (4, 4, 1, 20, 1, {}),                                            # R = 0, no final variables
    (12, 3, 2, 30, 2, {"num_rounds": 3, "final_vars": 0,
                       "queries": [20, 12, 9, 7]}),                  # hand-set schedule, 1 final coeff
    (9, 3, 3, 30, 0, {"num_rounds": 1, "final_vars": 3, "final_pow_bits": 5,
                      "queries": [4, 1]}),
    (10, 3, 2, 40, 3, {"batch_size": 2}),                            # the ZK batch
    (12, 2, 1, 30, 2, {"batch_size": 4, "ood_samples": 2}),
    (8, 4, 1, 20, 1, {"batch_size": 2}),                             # R = 0: final opens the batch
    (8, 2, 1, 32, 2, {}),
    (10, 3, 2, 40, 3, {}),
    (12, 3, 2, 60, 4, {"ood_samples": 2}),
    (13, 4, 1, 40, 0, {}),
    (14, 2, 2, 30, 2, {}),
    (15, 5, 1, 30, 1, {}),
    (16, 6, 2, 24, 0, {"ood_samples": 3}),
    (12, 1, 3, 20, 1, {}),
]


def _problem(n, ncov, seed, batch=1):
    N = 1 << n
    return O.sample_fr(seed, batch * N), O.sample_fr(seed + 1, max(ncov, 1) * N)[: ncov * N]


@pytest.mark.parametrize("n,k,lr,sec,pw,over", CASES)
def test_honest_proofs_are_accepted(n, k, lr, sec, pw, over):
    p = O.whir_params(n, k, lr, sec, pw, **over)
    assert (p.num_rounds + 1) * k + p.final_vars == n
    for ncov in (0, 1, 3):
        c, cov = _problem(n, ncov, 1000 * n + 10 * k + ncov, p.batch_size)
        cw, proof = O.whir_prove(p, 0x5eed + n, c, cov)
        lay = layout(p, ncov)
        assert proof.shape[0] == lay["total"] == O.lib().pko_whir_proof_words(
            O.ctypes.byref(p), ncov)
        assert O.whir_verify(p, 0x5eed + n, cov, ncov, cw, proof) == 0
        # the statement values are the covectors' dot products with each
        # polynomial of the batch
        for i in range(p.batch_size):
            for a in range(ncov):
                exp = np.zeros(4, np.uint64)
                O.lib().pko_dot(O.p64(exp), O.p64(np.ascontiguousarray(cov[a << n:(a + 1) << n])),
                                O.p64(np.ascontiguousarray(c[i << n:(i + 1) << n])), 1 << n)
                at = 4 * (i * ncov + a)
                assert np.array_equal(proof[at:at + 4], exp)


def test_params_schedule_of_the_r1cs_config():
    """n = 21 with the reference's whir config (ff 3, rate 1/4, 128 bits,
    10 PoW bits): five folds of three variables, six sent in the clear."""
    p = O.whir_params(21, 3, 2, 128, 10)
    assert (p.num_rounds, p.final_vars, p.ood_samples) == (4, 6, 1)
    assert list(p.queries[:5]) == [118, 59, 40, 30, 24]


@pytest.fixture(scope="module")
def honest():
    p = O.whir_params(12, 3, 2, 40, 4, ood_samples=2)
    ncov = 2
    c, cov = _problem(12, ncov, 4242)
    cw, proof = O.whir_prove(p, 99, c, cov)
    assert O.whir_verify(p, 99, cov, ncov, cw, proof) == 0
    return p, ncov, c, cov, cw, proof, layout(p, ncov)


def _bump(words, at):
    """Add one to the field element at word offset `at` (stays canonical)."""
    w = words.copy()
    x = O.sample_fr(1, 1)[0] * 0  # zero
    one = np.array([1, 0, 0, 0], np.uint64)
    m = np.zeros(4, np.uint64)
    O.lib().pko_fr_to_mont(O.p64(m), O.p64(one))
    O.lib().pko_fr_add(O.p64(x), O.p64(np.ascontiguousarray(w[at:at + 4])), O.p64(m))
    w[at:at + 4] = x
    return w


def _verify(h, proof=None, cw=None, cov=None, domain=99):
    p, ncov, _, cov0, cw0, proof0, _ = h
    return O.whir_verify(p, domain, cov0 if cov is None else cov, ncov,
                         cw0 if cw is None else cw, proof0 if proof is None else proof)


def test_tampered_statement_value_is_rejected(honest):
    lay = honest[6]
    assert _verify(honest, proof=_bump(honest[5], lay["values"] + 4)) == -3


def test_tampered_commitment_answer_is_rejected(honest):
    assert _verify(honest, cw=_bump(honest[4], 4)) == -3


def test_other_statement_is_rejected(honest):
    cov = honest[3].copy()
    cov[5] = O.sample_fr(77, 1)[0]
    assert _verify(honest, cov=cov) == -7


def test_other_transcript_domain_is_rejected(honest):
    assert _verify(honest, domain=100) != 0


def test_tampered_sumcheck_message_is_rejected(honest):
    lay = honest[6]
    for at in (lay["sc0"], lay["rounds"][0]["sc"] + 12, lay["final"]["sc"] + 4):
        assert _verify(honest, proof=_bump(honest[5], at)) == -3


def test_tampered_round_ood_answer_is_rejected(honest):
    """The answer is absorbed before the round's PoW challenge is drawn, so
    the grinding check sees it first; without PoW the sum check does."""
    lay = honest[6]
    assert _verify(honest, proof=_bump(honest[5], lay["rounds"][0]["ood"] + 4)) in (-3, -4)


def test_tampered_opening_is_rejected(honest):
    lay = honest[6]
    for sec in (lay["rounds"][0], lay["final"]):
        row_at = sec["open"] + 3 * (sec["row_words"] + sec["path_words"]) + 4
        assert _verify(honest, proof=_bump(honest[5], row_at)) == -5
        path_at = sec["open"] + sec["row_words"]
        assert _verify(honest, proof=_bump(honest[5], path_at)) == -5


def test_tampered_root_is_rejected(honest):
    lay = honest[6]
    assert _verify(honest, proof=_bump(honest[5], lay["rounds"][0]["root"])) != 0


def test_tampered_pow_nonce_is_rejected(honest):
    lay = honest[6]
    for at in (lay["rounds"][0]["pow"], lay["final"]["pow"]):
        bad = None
        for d in range(1, 64):  # the first nonce above the honest one that fails
            w = honest[5].copy()
            w[at] = w[at] + np.uint64(d)
            rc = _verify(honest, proof=w)
            if rc == -4:
                bad = d
                break
        assert bad is not None


def test_tampered_final_coefficient_is_rejected(honest):
    """The coefficients are absorbed before the final PoW challenge and the
    final query indices are drawn, so a changed coefficient fails the PoW,
    or opens other leaves than the proof carries (Merkle), or -- should the
    indices survive -- UnivarPoly != computeFold."""
    lay = honest[6]
    assert _verify(honest, proof=_bump(honest[5], lay["final"]["coeffs"])) in (-4, -6)
    p = O.whir_params(11, 3, 2, 40, 0)
    c, cov = _problem(11, 1, 515)
    cw, proof = O.whir_prove(p, 8, c, cov)
    at = layout(p, 1)["final"]["coeffs"] + 4
    assert O.whir_verify(p, 8, cov, 1, cw, proof) == 0
    assert O.whir_verify(p, 8, cov, 1, cw, _bump(proof, at)) in (-5, -6)


def test_non_canonical_and_truncated_proofs_are_rejected(honest):
    p, ncov, _, cov, cw, proof, lay = honest
    w = proof.copy()
    w[lay["sc0"]:lay["sc0"] + 4] = np.array([~np.uint64(0)] * 4, np.uint64)
    assert _verify(honest, proof=w) == -2
    assert O.whir_verify(p, 99, cov, ncov, cw, proof[:-1]) == -2


def test_wrong_witness_cannot_be_proven_for_the_claimed_values():
    """A proof for another vector carries other statement values."""
    p = O.whir_params(10, 2, 2, 30, 0)
    c, cov = _problem(10, 1, 31)
    cw1, pr1 = O.whir_prove(p, 5, c, cov)
    c2 = c.copy()
    c2[3] = O.sample_fr(32, 1)[0]
    cw2, pr2 = O.whir_prove(p, 5, c2, cov)
    assert not np.array_equal(pr1[:4], pr2[:4])
    assert not np.array_equal(cw1, cw2)
    # each proof verifies only against its own commitment
    assert O.whir_verify(p, 5, cov, 1, cw1, pr1) == 0
    assert O.whir_verify(p, 5, cov, 1, cw2, pr1) != 0


def test_subset_transforms_are_inverse_pairs():
    """mobius^T is the adjoint inverse of zeta: <mobius^T(a), zeta(c)> = <a, c>."""
    n = 9
    a, c = O.sample_fr(61, 1 << n), O.sample_fr(62, 1 << n)
    za, mc = c.copy(), a.copy()
    O.lib().pko_subset_zeta(O.p64(za), n)
    O.lib().pko_subset_mobius_t(O.p64(mc), n)
    d1, d2 = np.zeros(4, np.uint64), np.zeros(4, np.uint64)
    O.lib().pko_dot(O.p64(d1), O.p64(a), O.p64(c), 1 << n)
    O.lib().pko_dot(O.p64(d2), O.p64(mc), O.p64(za), 1 << n)
    assert np.array_equal(d1, d2)
    # zeta of a one-hot vector at index i is the indicator of supersets of i
    e = np.zeros((1 << n, 4), np.uint64)
    one = np.zeros(4, np.uint64)
    O.lib().pko_fr_to_mont(O.p64(one), O.p64(np.array([1, 0, 0, 0], np.uint64)))
    e[5] = one
    O.lib().pko_subset_zeta(O.p64(e), n)
    for b in range(1 << n):
        assert np.array_equal(e[b], one if (b & 5) == 5 else np.zeros(4, np.uint64))


def test_squeeze_bytes_takes_31_bytes_per_element():
    t1, t2 = O.transcript(3), O.transcript(3)
    out = np.zeros(70, np.uint8)
    O.lib().pko_transcript_squeeze_bytes(O.ctypes.byref(t1), O.p8(out), 70)
    exp = b""
    for _ in range(3):
        m, c = np.zeros(4, np.uint64), np.zeros(4, np.uint64)
        O.lib().pko_transcript_squeeze(O.ctypes.byref(t2), O.p64(m))
        O.lib().pko_fr_from_mont(O.p64(c), O.p64(m))
        exp += c.tobytes()[:31]
    assert out.tobytes() == exp[:70]


@pytest.mark.parametrize("nc,ni,batch", [(1 << 10, 1 << 8, 1), (3000, 500, 1), (1 << 12, 1 << 12, 1),
                                         (1 << 10, 1 << 8, 2), (3000, 500, 2)])
def test_whole_r1cs_proof_verifies(nc, ni, batch):
    """pko_prove_r1cs: the Spartan part, then the WHIR proof of the
    covectors M^T eq(alpha) and the blinding covector against the
    evaluations; the WHIR part verifies from the transcript state the prover
    started it from, and the evaluations are the covectors' dot products
    with the padded witness."""
    from provekit_b200.prover import HostR1CS
    h = HostR1CS(nc + ni, nc, ni)
    m, m0 = O.r1cs_sizing(h.num_constraints, h.num_witnesses)
    wp = O.whir_params(m, 3, 2, 40, 3, batch_size=batch)
    sp, cw, proof = O.prove_r1cs(h, 5, 11, wp)
    assert (sp["m"], sp["m0"]) == (m, m0)
    assert O.verify_r1cs_whir(h, wp, 11, sp, cw, proof) == 0
    cov = O.r1cs_covectors(h, sp["alpha"], m0, 1 << m)
    ncov = O.statement_count(h)  # A, B, C and the blinding covector
    stm = O.statement_covectors(h, sp)
    assert stm.shape[0] == ncov << m
    if batch == 2:
        # whir-ZK: the blinding polynomial is the indexed sampler's
        g = np.zeros((1 << m, 4), np.uint64)
        O.lib().pko_sample_fr_indexed(5 ^ 0x243f6a8885a308d3, 0, 1 << m, O.p64(g))
        for k in range(ncov):
            d = np.zeros(4, np.uint64)
            O.lib().pko_dot(O.p64(d), O.p64(np.ascontiguousarray(stm[k << m:(k + 1) << m])),
                            O.p64(g), 1 << m)
            assert np.array_equal(proof[4 * (ncov + k):4 * (ncov + k) + 4], d)
    for k in range(3):
        assert np.array_equal(proof[4 * k:4 * k + 4], sp["evals"][k])
        d = np.zeros(4, np.uint64)
        O.lib().pko_dot(O.p64(d), O.p64(np.ascontiguousarray(cov[k << m:(k << m) + h.num_witnesses])),
                        O.p64(np.ascontiguousarray(h.witness)), h.num_witnesses)
        assert np.array_equal(d, sp["evals"][k])
    # the fourth statement is the zk-sumcheck's blinding evaluation
    assert np.array_equal(proof[12:16], sp["blinding_eval"])
    # the WHIR part is bound to the Spartan transcript
    bad = dict(sp)
    bad["transcript"] = (list(sp["transcript"][1]), list(sp["transcript"][0]))
    assert O.verify_r1cs_whir(h, wp, 11, bad, cw, proof) != 0


def test_batch_tampering_is_rejected():
    """The ZK batch: the second polynomial's statement value, its half of an
    opened first-round row, and its OOD answer are all bound."""
    p = O.whir_params(11, 3, 2, 40, 0, batch_size=2)
    c, cov = _problem(11, 2, 9191, 2)
    cw, proof = O.whir_prove(p, 17, c, cov)
    assert O.whir_verify(p, 17, cov, 2, cw, proof) == 0
    lay = layout(p, 2)
    assert O.whir_verify(p, 17, cov, 2, cw, _bump(proof, lay["values"] + 4 * 3)) == -3
    sec = lay["rounds"][0]
    row_at = sec["open"] + sec["row_words"] // 2 + 4  # an entry of f_1's half
    assert O.whir_verify(p, 17, cov, 2, cw, _bump(proof, row_at)) == -5
    assert O.whir_verify(p, 17, cov, 2, _bump(cw, 4 + 4), proof) != 0  # f_1's OOD answer
    # a batch proof is not a proof about either polynomial alone
    p1 = O.whir_params(11, 3, 2, 40, 0)
    assert O.whir_verify(p1, 17, cov, 2, cw[:8], proof) != 0



@pytest.mark.parametrize("npub,batch", [(1, 1), (3, 2), (200, 1)])
def test_whole_proof_with_public_inputs_verifies(npub, batch):
    """Public inputs (witness[1 ..= n]): their hash enters the transcript
    (PublicInputs::hash, provekit/common/src/witness/mod.rs:86-97), the
    public weight [1, x, .., x^n] is the first statement and its value
    <weight, w> is sent after the three evaluations."""
    from provekit_b200.prover import HostR1CS
    h = HostR1CS(61 + npub, 1 << 10, 1 << 9, num_public_inputs=npub)
    m, m0 = O.r1cs_sizing(h.num_constraints, h.num_witnesses)
    wp = O.whir_params(m, 3, 2, 40, 3, batch_size=batch)
    sp, cw, proof = O.prove_r1cs(h, 2, 21, wp)
    assert O.statement_count(h) == 5
    assert O.verify_r1cs_whir(h, wp, 21, sp, cw, proof) == 0
    # the hash over the canonical public values
    pub = np.ascontiguousarray(h.witness[1:1 + npub]).copy()
    O.lib().pko_from_mont_many(O.p64(pub), npub)
    exp = np.zeros(4, np.uint64)
    O.lib().pko_public_inputs_hash(O.p64(exp), O.p64(pub), npub)
    assert np.array_equal(sp["public_hash"], exp)
    assert np.array_equal(proof[0:4], sp["public_eval"])
    # another public value changes the hash, hence x and the whole proof
    h.witness[1] = O.sample_fr(999, 1)[0]
    sp2, cw2, proof2 = O.prove_r1cs(h, 2, 21, wp)
    assert not np.array_equal(sp2["public_hash"], sp["public_hash"])
    assert not np.array_equal(sp2["public_x"], sp["public_x"])


def test_public_inputs_hash_cases():
    """0 for none, compress(v, 0) for one, the left fold for more."""
    v = O.sample_fr(5, 3, mont=False)
    out = np.zeros(4, np.uint64)
    O.lib().pko_public_inputs_hash(O.p64(out), O.p64(v), 0)
    assert not out.any()
    O.lib().pko_public_inputs_hash(O.p64(out), O.p64(v), 1)
    assert np.array_equal(out, O.compress(v[0], np.zeros(4, np.uint64)))
    O.lib().pko_public_inputs_hash(O.p64(out), O.p64(v), 3)
    assert np.array_equal(out, O.compress(O.compress(v[0], v[1]), v[2]))
