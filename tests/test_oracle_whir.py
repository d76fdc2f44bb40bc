"""CPU pins of the oracle's WHIR prove-round building blocks against
Python big-int restatements of the reference's Go WHIR verifier
(recursive-verifier/app/utilities/utilities.go: MultivarPoly :16-23,
UnivarPoly :25-39, EvaluateQuadraticPolynomialFromEvaluationList :149-155,
CheckSumOverBool :168-171, ExpandFromUnivariate :183-191;
recursive-verifier/app/circuit/whir_utilities.go: verifyMerkleTreeProofs
:14-47, getStirChallenges :49-79, computeFold :182-188), plus the
protocol identities a WHIR prover relies on: folding the interleaved
codeword's rows equals encoding the folded coefficients, and each sumcheck
round polynomial sums to the previous claim evaluated at the challenge."""
import random

import numpy as np
import pytest

import oracle_lib as O
from fieldutil import P, pack, to_limbs, unpack

INV2 = pow(2, P - 2, P)


# ---- the Go verifier's arithmetic, restated ---------------------------------
def multivar_poly(coefs, vs):
    if not vs:
        return coefs[0] % P
    h = len(coefs) // 2
    return (multivar_poly(coefs[:h], vs[:-1]) + vs[-1] * multivar_poly(coefs[h:], vs[:-1])) % P


def univar_poly(coeffs, z):
    ans = 0
    for i in range(len(coeffs)):
        ans = (ans * z + coeffs[len(coeffs) - 1 - i]) % P
    return ans


def expand_from_univariate(z, n):
    res, acc = [0] * n, z % P
    for i in range(n):
        res[n - 1 - i] = acc
        acc = acc * acc % P
    return res


def eval_quadratic(e, x):
    b0 = e[0]
    b1 = (-e[2] + 4 * e[1] - 3 * e[0]) * INV2
    b2 = (e[2] - 2 * e[1] + e[0]) * INV2
    return (b2 * x * x + b1 * x + b0) % P


def go_bits_len(x):  # math/bits.Len
    return x.bit_length()


def stir_indices_go(data: bytes, folded: int, nq: int):
    nbytes = (go_bits_len(folded * 2 - 1) - 1 + 7) // 8
    bit_length = go_bits_len(folded) - 1
    out = []
    for i in range(nq):
        v = 0
        for j in range(nbytes):
            v = data[j + i * nbytes] + v * 256
        out.append(v & ((1 << bit_length) - 1))
    return out


def rand_fr(rng, n):
    return [rng.randrange(P) for _ in range(n)]


# ---- tests --------------------------------------------------------------------
@pytest.mark.parametrize("k", [0, 1, 2, 3, 4, 5])
def test_fold_rows_is_multivar_poly(k):
    rng = random.Random(k)
    m = 1 << k
    rows = [rand_fr(rng, m) for _ in range(40)]
    alpha = rand_fr(rng, k)
    got = unpack(O.whir_fold_rows(pack([v for r in rows for v in r]), k, pack(alpha) if k else
                                  np.zeros((1, 4), np.uint64)))
    assert got == [multivar_poly(r, alpha) for r in rows]


@pytest.mark.parametrize("k,logn,lr", [(1, 6, 1), (3, 10, 2), (4, 12, 2), (2, 9, 3)])
def test_fold_commutes_with_rs_encode(k, logn, lr):
    """fold_rows(interleaved_encode(c)) == encode(fold_coeffs(c)) on the same
    domain: the folded polynomial's codeword is the fold of the committed one."""
    rng = random.Random(logn)
    n, M = 1 << logn, 1 << k
    L = n >> k
    c = pack(rand_fr(rng, n))
    alpha = pack(rand_fr(rng, k))
    cw = L << lr
    rc, rows = O.rs_interleaved_encode(c.reshape(M, L, 4), np.zeros((0, 4), np.uint64), cw)
    assert rc == 0
    folded = O.whir_fold_coeffs(c, k, alpha)
    rc, enc = O.rs_interleaved_encode(folded.reshape(1, L, 4), np.zeros((0, 4), np.uint64), cw)
    assert rc == 0
    assert np.array_equal(O.whir_fold_rows(rows, k, alpha), enc)


def test_poly_eval_is_univar_poly_and_bitreversed_multivar():
    rng = random.Random(7)
    for n in (1, 2, 5, 64, 257):
        c = rand_fr(rng, n)
        z = rng.randrange(P)
        got = unpack(O.poly_eval(pack(c), pack([z])[0]).reshape(1, 4))[0]
        assert got == univar_poly(c, z)
    # MultivarPoly over ExpandFromUnivariate(z) reads the coefficients in
    # bit-reversed order: sum_j c_j z^bitrev(j).
    nv = 5
    c = rand_fr(rng, 1 << nv)
    z = rng.randrange(P)
    rev = [c[int(format(j, f"0{nv}b")[::-1], 2)] for j in range(1 << nv)]
    assert multivar_poly(c, expand_from_univariate(z, nv)) == univar_poly(rev, z)
    e = np.zeros((nv, 4), np.uint64)
    O.lib().pko_expand_from_univariate(O.p64(e), O.p64(pack([z])[0].copy()), nv)
    assert unpack(e) == expand_from_univariate(z, nv)


@pytest.mark.parametrize("folded", [1 << 5, 1 << 8, 1 << 13, 1 << 20, 1 << 17])
def test_stir_indices_match_go(folded):
    rng = np.random.default_rng(folded)
    nq = 37
    nbytes = ((folded.bit_length() - 1) + 7) // 8
    data = rng.integers(0, 256, size=nq * nbytes, dtype=np.uint8)
    out = np.zeros(nq, np.uint64)
    O.lib().pko_stir_indices(O.p8(data), folded, nq, O.p64(out))
    assert [int(v) for v in out] == stir_indices_go(data.tobytes(), folded, nq)


@pytest.mark.parametrize("m,log_leaves", [(8, 6), (16, 4), (2, 7), (1, 3)])
def test_merkle_openings_verify_like_go(m, log_leaves):
    """Trees over canonical Fr leaves (the commit's leaf encoding) open at any
    index into paths that the Go verifier's verifyMerkleTreeProofs accepts."""
    rng = random.Random(m * 100 + log_leaves)
    nl = 1 << log_leaves
    vals = [rand_fr(rng, m) for _ in range(nl)]
    leaf_bytes = pack([v for r in vals for v in r], mont=False).tobytes()
    layers = O.merkle_tree(leaf_bytes, 32 * m, nl)
    root = layers[-32:]
    for idx in list(range(min(nl, 8))) + [nl - 1, rng.randrange(nl)]:
        path = O.merkle_open(layers, nl, idx)
        # restated verifyMerkleTreeProofs: leaf fold, then sibling and auth path
        h = to_limbs(vals[idx][0])
        for x in vals[idx][1:]:
            h = O.compress(h, to_limbs(x))
        for lev in range(log_leaves):
            s = list(np.frombuffer(path[32 * lev:32 * lev + 32], dtype=np.uint64))
            h = O.compress(s, h) if (idx >> lev) & 1 else O.compress(h, s)
        assert np.array(h, dtype=np.uint64).tobytes() == root
        leaf = pack(vals[idx], mont=False)
        pth = np.frombuffer(path, dtype=np.uint8).copy() if log_leaves else np.zeros(1, np.uint8)
        rt = np.frombuffer(root, dtype=np.uint8).copy()
        assert O.lib().pko_merkle_verify(O.p64(leaf), m, idx, O.p8(pth), log_leaves, O.p8(rt)) == 1
        if log_leaves:
            pth[5] ^= 1
            assert O.lib().pko_merkle_verify(O.p64(leaf), m, idx, O.p8(pth), log_leaves,
                                             O.p8(rt)) == 0


def test_whir_sumcheck_rounds_satisfy_the_go_checks():
    """Every round's (h(0), h(1), h(2)) passes CheckSumOverBool against the
    previous claim evaluated at the challenge, and the last claim is f*w at
    the folding point."""
    rng = random.Random(11)
    nv = 7
    f_int, w_int = rand_fr(rng, 1 << nv), rand_fr(rng, 1 << nv)
    f, w = pack(f_int), pack(w_int)
    claim = sum(a * b for a, b in zip(f_int, w_int)) % P
    size, fold = 1 << nv, None
    for _ in range(nv):
        h = unpack(O.whir_sumcheck_round(f, w, size, fold))
        assert (h[0] + h[1]) % P == claim
        a = rng.randrange(P)
        claim = eval_quadratic(h, a)
        if fold is not None:
            size //= 2
        fold = pack([a])[0].copy()
    # fold the last variable and compare with the claim
    last_f, last_w = unpack(f[:2]), unpack(w[:2])
    a = unpack(fold.reshape(1, 4))[0]
    ff = (last_f[0] + a * (last_f[1] - last_f[0])) % P
    ww = (last_w[0] + a * (last_w[1] - last_w[0])) % P
    assert ff * ww % P == claim


def test_eq_accumulate_matches_definition():
    rng = random.Random(13)
    nv, npts = 6, 5
    w0 = rand_fr(rng, 1 << nv)
    pts = [rand_fr(rng, nv) for _ in range(npts)]
    cf = rand_fr(rng, npts)
    w = pack(w0)
    assert O.lib().pko_eq_accumulate(O.p64(w), nv, O.p64(pack([v for p in pts for v in p])),
                                     O.p64(pack(cf)), npts) == 0

    def eq(p, b):
        acc = 1
        for i in range(nv):
            bit = (b >> (nv - 1 - i)) & 1
            acc = acc * (p[i] if bit else (1 - p[i])) % P
        return acc
    exp = [(w0[b] + sum(cf[j] * eq(pts[j], b) for j in range(npts))) % P for b in range(1 << nv)]
    assert unpack(w) == exp
