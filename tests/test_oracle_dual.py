"""The oracle's dual-commitment prover (R1CS with verifier challenges) on CPU:
sizing with the witness split at w1_size, the synthetic instance's solver,
the verifier's acceptance (both commitments, the challenges between them,
both WHIR proofs, the claimed values, the challenge binding) and its
rejections.  Follows provekit/prover/src/lib.rs:145-232 and
provekit/prover/src/whir_r1cs.rs:302-425; the reference's own proof bytes
need the un-vendored whir and spongefish crates, so acceptance is by the
restated verifier."""
import ctypes

import numpy as np
import pytest

import oracle_lib as O


def ceil_log2(n):
    k = 0
    while (1 << k) < n:
        k += 1
    return k


def sizing_formula(nc, nw, w1):
    """WhirR1CSScheme::new_for_r1cs (r1cs-compiler/src/whir_r1cs.rs:48-92)."""
    m = max(ceil_log2(w1), ceil_log2(nw - w1), 13)
    m0 = max(ceil_log2(nc), 1)
    if (1 << m) - w1 < 4 * m0:
        m += 1
    return m, m0


@pytest.mark.parametrize("nc,nw,w1", [
    (1, 1, 1), (100, 300, 300), (100, 300, 150), (1 << 14, 1 << 13, 1 << 12),
    (1 << 14, (1 << 14) + 5, 5), (1 << 20, (1 << 21), 1 << 20),
    (1 << 20, (1 << 13) - 3, (1 << 13) - 3), (1 << 20, 3 << 13, (1 << 13) - 80),
])
def test_sizing_split(nc, nw, w1):
    assert O.r1cs_sizing_split(nc, nw, w1) == sizing_formula(nc, nw, w1)
    if w1 == nw:
        assert O.r1cs_sizing_split(nc, nw, w1) == O.r1cs_sizing(nc, nw)


def satisfied(h, w):
    a = np.zeros((h.num_constraints, 4), np.uint64)
    b, c = np.zeros_like(a), np.zeros_like(a)
    for k, y in enumerate((a, b, c)):
        O.lib().pko_spmv(O.p64(h.row_ptr[k]), O.p32(h.cols[k]), O.p64(h.vals[k]),
                         h.num_constraints, O.p64(np.ascontiguousarray(w)), O.p64(y))
    ab = np.zeros_like(a)
    for i in range(h.num_constraints):
        O.lib().pko_fr_mul(O.p64(ab[i]), O.p64(a[i]), O.p64(b[i]))
    return np.array_equal(ab, c)


@pytest.mark.parametrize("nchal,rows2", [(0, 0), (0, 30), (1, 0), (1, 50), (4, 77)])
def test_synthetic_instance_solves(nchal, rows2):
    h = O.SyntheticDualR1CS(3, 64, 20, nchal, rows2)
    offs = [int(o) for o in h.challenge_offsets]
    assert offs == sorted(set(offs)) and all(o < nchal + rows2 for o in offs)
    ch = O.sample_fr(99, nchal).reshape(-1, 4)
    w = h.witness.copy()
    w[h.w1_size:] = h.solve(ch)
    for j, o in enumerate(offs):
        assert np.array_equal(w[h.w1_size + o], ch[j])
    assert satisfied(h, w)
    if rows2:
        bad = w.copy()
        bad[h.w1_size + [o for o in range(nchal + rows2) if o not in offs][0], 0] ^= 1
        assert not satisfied(h, bad)


SHAPES = [  # (nc1, ni, nchal, rows2, public inputs, batch)
    (100, 30, 3, 60, 0, 1),
    (100, 30, 3, 60, 2, 2),
    (200, 40, 1, 10, 1, 2),
    (50, 10, 0, 40, 0, 2),    # two commitments, no challenge weight
    (50, 10, 5, 0, 3, 1),     # w2 holds only challenges
    (50, 10, 0, 0, 0, 2),     # w2 empty
    (300, 100, 8, 9000, 0, 2),  # w2 larger than w1: m set by w2
]


@pytest.mark.parametrize("shape", SHAPES)
def test_dual_proof_verifies(shape):
    nc1, ni, nchal, rows2, npub, nb = shape
    h = O.SyntheticDualR1CS(11, nc1, ni, nchal, rows2, num_public_inputs=npub)
    m, m0 = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, 40, 4, batch_size=nb)
    d, ch, cw1, cw2, pr1, pr2, w = O.prove_r1cs_dual(h, 5, 21, wp)
    assert (d["m"], d["m0"]) == (m, m0)
    assert satisfied(h, w)
    assert O.verify_r1cs_dual(h, wp, 21, d, ch, cw1, cw2, pr1, pr2) == 0
    # evals1 + evals2 is <M^T eq(alpha), w> over the whole witness: the value
    # the Spartan verifier's final check uses
    full = O.r1cs_covectors(h, d["alpha"], m0, h.num_witnesses).reshape(3, -1, 4)
    for k in range(3):
        want, got = np.zeros(4, np.uint64), np.zeros(4, np.uint64)
        O.lib().pko_dot(O.p64(want), O.p64(np.ascontiguousarray(full[k])), O.p64(w),
                        h.num_witnesses)
        O.lib().pko_fr_add(O.p64(got), O.p64(np.ascontiguousarray(d["evals"][k])),
                           O.p64(np.ascontiguousarray(d["evals2"][k])))
        assert np.array_equal(got, want)
    if not nchal:
        assert not d["challenge_eval"].any()


def test_dual_proof_rejections():
    h = O.SyntheticDualR1CS(12, 120, 30, 3, 80, num_public_inputs=2)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, 40, 4, batch_size=2)
    d, ch, cw1, cw2, pr1, pr2, _ = O.prove_r1cs_dual(h, 5, 21, wp)
    assert O.verify_r1cs_dual(h, wp, 21, d, ch, cw1, cw2, pr1, pr2) == 0
    # another domain: other challenges
    assert O.verify_r1cs_dual(h, wp, 22, d, ch, cw1, cw2, pr1, pr2) != 0
    # a word of either WHIR proof
    for pr, i in ((pr1, 40), (pr2, len(pr2) // 2)):
        bad = pr.copy()
        bad[i] ^= 1
        args = (pr1, bad) if pr is pr2 else (bad, pr2)
        assert O.verify_r1cs_dual(h, wp, 21, d, ch, cw1, cw2, *args) != 0
    # the second commitment's root
    bad = cw2.copy()
    bad[0] ^= 1
    assert O.verify_r1cs_dual(h, wp, 21, d, ch, cw1, bad, pr1, pr2) != 0
    # claimed Spartan messages that differ from the proofs' statement values
    d2 = dict(d, evals2=d["evals2"][[1, 0, 2]])
    assert O.verify_r1cs_dual(h, wp, 21, d2, ch, cw1, cw2, pr1, pr2) == 2


def test_challenge_binding_catches_a_wrong_challenge_value():
    """A w2 whose challenge entry is not the squeezed challenge: the proofs
    are internally consistent but the binding <[1, x, ..], challenges> fails
    (whir_r1cs.rs:340-348)."""
    h = O.SyntheticDualR1CS(13, 80, 20, 2, 40)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, 40, 4, batch_size=1)
    ctx, keep = h.solver_ctx()
    SOLVER = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                              ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64))

    def wrong(c, chal, k, w):
        O.lib().pko_synthetic_dual_solve(c, chal, k, w)
        w[4 * (h.w1_size + int(h.challenge_offsets[1]))] ^= 1

    cb = SOLVER(wrong)
    r = O._r1cs_c(h)
    out = O.DualProof()
    ch = np.zeros((2, 4), np.uint64)
    cw1 = np.zeros(O.lib().pko_whir_commit_words(ctypes.byref(wp)), np.uint64)
    cw2 = np.zeros_like(cw1)
    pr1 = np.zeros(O.lib().pko_whir_proof_words(ctypes.byref(wp), 4), np.uint64)
    pr2 = np.zeros(O.lib().pko_whir_proof_words(ctypes.byref(wp), 4), np.uint64)
    w = np.ascontiguousarray(h.witness.copy())
    offs = np.ascontiguousarray(h.challenge_offsets, dtype=np.uint64)
    rc = O.lib().pko_prove_r1cs_dual(ctypes.byref(r), h.w1_size, O.p64(offs), 2, O.p64(w),
                                     ctypes.cast(cb, ctypes.c_void_p), ctypes.byref(ctx), 5, 21,
                                     ctypes.byref(wp), ctypes.byref(out), O.p64(ch), O.p64(cw1),
                                     O.p64(cw2), O.p64(pr1), O.p64(pr2))
    del keep
    assert rc == 0
    d = O.dual_dict(out)
    assert O.verify_r1cs_dual(h, wp, 21, d, ch, cw1, cw2, pr1, pr2) == 3


def test_dual_argument_errors():
    h = O.SyntheticDualR1CS(14, 40, 10, 2, 10, num_public_inputs=3)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, 40, 4)
    r = O._r1cs_c(h)
    ctx, keep = h.solver_ctx()
    out = O.DualProof()
    buf = np.zeros(1 << 16, np.uint64)
    solve = ctypes.cast(O.lib().pko_synthetic_dual_solve, ctypes.c_void_p)

    def call(w1_size, offs, wpp=wp):
        o = np.ascontiguousarray(offs, dtype=np.uint64)
        w = np.ascontiguousarray(h.witness.copy())
        return O.lib().pko_prove_r1cs_dual(ctypes.byref(r), w1_size, O.p64(o), len(offs),
                                           O.p64(w), solve, ctypes.byref(ctx), 1, 1,
                                           ctypes.byref(wpp), ctypes.byref(out), O.p64(buf),
                                           O.p64(buf), O.p64(buf), O.p64(buf), O.p64(buf))

    assert call(h.w1_size, [1 << m]) == -1                 # offset outside 2^m
    assert call(3, [0, 1]) == -1                           # w1 without the public inputs
    assert call(h.num_witnesses + 1, [0, 1]) == -1         # w1 longer than the witness
    assert call(h.w1_size, [0, 1], O.whir_params(m + 1, 3, 2, 40, 4)) == -1  # wrong m
    del keep


def test_dual_proofs_verify_over_random_shapes():
    """Seeded random shapes (rows of w1 and w2, inputs, challenges, public
    inputs, batch, folding factor): every oracle dual proof is accepted, and
    the proof of another seed's instance is not."""
    rng = np.random.default_rng(2024)
    for case in range(12):
        nc1 = int(rng.integers(1, 300))
        ni = int(rng.integers(1, 120))
        nchal = int(rng.integers(0, 9))
        rows2 = int(rng.integers(0, 400))
        npub = int(rng.integers(0, min(ni, 4) + 1))
        nb = int(rng.integers(1, 3))
        ff = int(rng.integers(1, 5))
        h = O.SyntheticDualR1CS(100 + case, nc1, ni, nchal, rows2, num_public_inputs=npub)
        m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
        wp = O.whir_params(m, ff, 2, 40, 3, batch_size=nb)
        d, ch, cw1, cw2, pr1, pr2, w = O.prove_r1cs_dual(h, case, 7, wp)
        assert satisfied(h, w), case
        assert O.verify_r1cs_dual(h, wp, 7, d, ch, cw1, cw2, pr1, pr2) == 0, case
        if case:  # the previous case's proof does not verify against this instance
            pd, pch, pcw1, pcw2, ppr1, ppr2 = prev
            if pcw1.shape == cw1.shape and ppr1.shape == pr1.shape and ppr2.shape == pr2.shape:
                assert O.verify_r1cs_dual(h, wp, 7, pd, pch, pcw1, pcw2, ppr1, ppr2) != 0, case
        prev = (d, ch, cw1, cw2, pr1, pr2)
