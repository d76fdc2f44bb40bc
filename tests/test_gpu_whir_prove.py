"""GPU parity of the WHIR prover's round loop (pkg_whir_prove).

The device prover must write the oracle's proof word for word: the
commitment (codeword, tree), the commitment's transcript words, and every
statement value, sumcheck message, root, OOD answer, PoW nonce and STIR
opening of every round.  The oracle's verifier -- a restatement of the
reference's Go verifier runWhir (recursive-verifier/app/circuit/whir.go:587-724)
-- must accept the device proofs, including at the reference's R1CS WHIR
configuration (ff 3, rate 1/4, 128 bits, 10 PoW bits) at 2^20 coefficients.
"""
import numpy as np
import pytest
import torch

import oracle_lib as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).copy()).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64).reshape(-1, 4)


def _params_pair(n, k, lr, sec, pw, over):
    from provekit_b200.whir import WhirParams
    return WhirParams.new(n, k, lr, sec, pw, **over), O.whir_params(n, k, lr, sec, pw, **over)


def _device_proof(p, domain, c, cov):
    from provekit_b200.spartan import Transcript
    from provekit_b200 import whir as W
    N = 1 << p.num_variables
    dc = dev(c)
    dcov = dev(cov) if cov.shape[0] else None
    cw, layers = W.commit(dc, p)
    t = Transcript.new(domain)
    words, ood = W.commit_ood(p, t, dc, layers)
    proof = W.prove(p, t, dc, cw, layers, ood, dcov)
    torch.cuda.synchronize()
    assert (dcov is None and cov.shape[0] == 0) or dcov.shape[0] == cov.shape[0]
    assert p.batch_size * N == dc.shape[0]
    return cw, layers, words, proof, (list(t.l), list(t.r))


CASES = [
    (6, 2, 1, 24, 0, {}),
    (4, 4, 1, 20, 1, {}),
    (12, 3, 2, 30, 2, {"num_rounds": 3, "final_vars": 0, "queries": [20, 12, 9, 7]}),
    (9, 3, 3, 30, 0, {"num_rounds": 1, "final_vars": 3, "final_pow_bits": 5, "queries": [4, 1]}),
    (8, 2, 1, 32, 2, {}),
    (10, 3, 2, 40, 3, {}),
    (12, 3, 2, 60, 4, {"ood_samples": 2}),
    (13, 4, 1, 40, 0, {}),
    (14, 2, 2, 30, 2, {}),
    (15, 5, 1, 30, 1, {}),
    (16, 6, 2, 24, 0, {"ood_samples": 3}),
    (12, 1, 3, 20, 1, {}),
    (11, 3, 2, 40, 2, {"ood_samples": 0}),
    (10, 3, 2, 40, 3, {"batch_size": 2}),
    (12, 2, 1, 30, 2, {"batch_size": 4, "ood_samples": 2}),
    (8, 4, 1, 20, 1, {"batch_size": 2}),
]


@pytest.mark.parametrize("n,k,lr,sec,pw,over", CASES)
def test_device_proof_equals_the_oracle_proof(n, k, lr, sec, pw, over):
    p, po = _params_pair(n, k, lr, sec, pw, over)
    for ncov in (0, 2):
        c = O.sample_fr(3000 + n + ncov, p.batch_size << n)
        cov = O.sample_fr(4000 + n + ncov, ncov << n) if ncov else np.zeros((0, 4), np.uint64)
        cw, layers, words, proof, _ = _device_proof(p, 0xabc + n, c, cov)
        ocw, olayers = O.whir_commit(c, k + O.batch_log(po), lr)
        assert np.array_equal(host(cw), ocw)
        assert np.array_equal(layers.cpu().numpy(), olayers)
        owords, oproof = O.whir_prove(po, 0xabc + n, c, cov)
        assert np.array_equal(words, owords)
        assert proof.shape == oproof.shape
        if not np.array_equal(proof, oproof):
            first = int(np.nonzero(proof != oproof)[0][0])
            pytest.fail(f"proofs differ first at word {first} of {proof.shape[0]}")
        assert O.whir_verify(po, 0xabc + n, cov, ncov, words, proof) == 0


def test_reference_config_at_2p20_verifies():
    """ff 3, rate 1/4, 128 bits, 10 PoW bits (the whir config of
    provekit/r1cs-compiler/src/whir_r1cs.rs:103-118) over 2^20
    coefficients and three covectors: the oracle verifier accepts."""
    n = 20
    p, po = _params_pair(n, 3, 2, 128, 10, {})
    assert (p.num_rounds, p.final_vars) == (4, 5)
    c = O.sample_fr(20, 1 << n)
    cov = O.sample_fr(21, 3 << n)
    _, _, words, proof, _ = _device_proof(p, 77, c, cov)
    assert O.whir_verify(po, 77, cov, 3, words, proof) == 0
    bad = proof.copy()
    bad[16] ^= np.uint64(1)  # h(1) of the first sumcheck round (after 3 values)
    assert O.whir_verify(po, 77, cov, 3, words, bad) != 0


@pytest.mark.parametrize("n,batch", [(20, 1), (21, 1), (21, 2)])
def test_reference_config_word_for_word(n, batch):
    """The reference's R1CS WHIR configuration (ff 3, rate 1/4, 128 bits,
    10 PoW bits) at the whole proof's sizes -- 2^20 and 2^21 coefficients,
    plain and as the whir-ZK batch of 2 -- with three covectors: the device
    proof equals the oracle's word for word (a verifier accepting a proof
    does not make it the same proof: another nonce, query or opening order
    would verify too)."""
    p, po = _params_pair(n, 3, 2, 128, 10, {"batch_size": batch})
    c = O.sample_fr(6000 + n + batch, batch << n)
    cov = O.sample_fr(7000 + n + batch, 3 << n)
    _, _, words, proof, _ = _device_proof(p, 0x5eed + n, c, cov)
    torch.cuda.empty_cache()
    owords, oproof = O.whir_prove(po, 0x5eed + n, c, cov)
    assert np.array_equal(words, owords)
    assert proof.shape == oproof.shape
    if not np.array_equal(proof, oproof):
        first = int(np.nonzero(proof != oproof)[0][0])
        pytest.fail(f"proofs differ first at word {first} of {proof.shape[0]}")
    assert O.whir_verify(po, 0x5eed + n, cov, 3, words, proof) == 0


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5, 8, 10, 11, 13, 17, 18, 20, 21, 22])
def test_subset_transforms_match_the_oracle(n):
    """Every pass split of the tiled transform: one pass (n <= 10), the
    first pass plus a partial one, and full 7-bit passes after it."""
    from provekit_b200.whir import SUBSET_MOBIUS_T, SUBSET_ZETA, subset_transform
    v = O.sample_fr(500 + n, 1 << n)
    for mode, fn in ((SUBSET_ZETA, "pko_subset_zeta"), (SUBSET_MOBIUS_T, "pko_subset_mobius_t")):
        d = dev(v)
        subset_transform(d, n, mode)
        exp = v.copy()
        getattr(O.lib(), fn)(O.p64(exp), n)
        assert np.array_equal(host(d), exp)


def test_pow_solutions_are_the_smallest_nonces():
    """The growing-batch device search returns generic::solve's answer."""
    import ctypes
    from provekit_b200._lib import lib
    for bits, seed in ((1, 1), (8, 2), (12, 3), (15, 4)):
        ch = O.sample_fr(seed, 1, mont=False)[0].copy()
        p = [0x43e1f593f0000001, 0x2833e84879b97091, 0xb85045b68181585d, 0x30644e72e131a029]
        v = sum(x << (64 * i) for i, x in enumerate(p)) >> bits
        thr = np.array([(v >> (64 * i)) & (2**64 - 1) for i in range(4)], np.uint64)
        got = ctypes.c_uint64(0)
        assert lib().pkg_skyscraper_pow_solve(ch.ctypes.data, thr.ctypes.data,
                                              ctypes.byref(got)) == 0
        assert got.value == O.lib().pko_sky_pow_solve(O.p64(ch), O.p64(thr))


def test_largest_commitment_proof_verifies():
    """2^24 coefficients (a 2 GiB codeword at rate 1/4, ff 4): the device
    proof of two statements is accepted by the oracle verifier."""
    n = 24
    p, po = _params_pair(n, 4, 2, 64, 6, {})
    c = O.sample_fr(24, 1 << n)
    cov = O.sample_fr(25, 2 << n)
    _, _, words, proof, _ = _device_proof(p, 31, c, cov)
    torch.cuda.empty_cache()
    assert O.whir_verify(po, 31, cov, 2, words, proof) == 0
