"""GPU parity of the dual-commitment proof (R1CS with verifier challenges,
pkg_dual_prove_begin / _finish) against the oracle's pko_prove_r1cs_dual:
the challenges, both commitments, every Spartan message and both WHIR proofs
must be identical word for word, and the oracle's verifier must accept the
device proof (both commitments with the challenges between them, both WHIR
proofs, the claimed values, the challenge binding).  Shapes cover public
inputs, whir-ZK, no challenges, a w2 of challenges only, an empty w2, a w2
longer than w1 and the balanced transposed-product path."""
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


def assert_same(a, b):
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], k


def device_params(m, sec, pw, nb):
    from provekit_b200.whir import WhirParams
    return WhirParams.new(m, 3, 2, sec, pw, batch_size=nb)


SHAPES = [  # (nc1, ni, nchal, rows2, public inputs, batch, security, pow)
    (100, 30, 3, 60, 0, 1, 40, 3),
    (100, 30, 3, 60, 2, 2, 40, 3),
    (200, 40, 1, 10, 1, 2, 64, 4),
    (50, 10, 0, 40, 0, 2, 40, 3),      # two commitments, no challenge weight
    (50, 10, 5, 0, 3, 1, 40, 3),       # w2 holds only challenges
    (50, 10, 0, 0, 0, 2, 40, 3),       # w2 empty
    (300, 100, 8, 9000, 0, 2, 64, 5),  # w2 longer than w1: m set by w2
    (1 << 15, 1 << 13, 16, 1 << 15, 2, 2, 128, 10),  # > 2^16 nonzeros: balanced products
]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("transposes", [True, False])
def test_dual_proof_matches_oracle_and_verifies(shape, transposes):
    from provekit_b200.prover import DeviceR1CS, prove_r1cs_dual
    nc1, ni, nchal, rows2, npub, nb, sec, pw = shape
    if not transposes and nc1 > 1000:
        pytest.skip("the per-proof transposes are covered at the small shapes")
    h = O.SyntheticDualR1CS(41 + nc1, nc1, ni, nchal, rows2, num_public_inputs=npub)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, sec, pw, batch_size=nb)
    ed, ech, ecw1, ecw2, epr1, epr2, _ = O.prove_r1cs_dual(h, 9, 33, wp)
    d = DeviceR1CS(h, transposes=transposes)
    p = device_params(m, sec, pw, nb)
    assert bytes(p) == bytes(wp)
    seen = []

    def solve(ch):
        seen.append(ch)
        return h.solve(ch)

    got, ch, cw1, cw2, pr1, pr2 = prove_r1cs_dual(d, h.w1_size, h.challenge_offsets, solve, p,
                                                  blinding_seed=9, transcript_domain=33)
    assert len(seen) == 1 and np.array_equal(seen[0], ech)
    assert np.array_equal(ch, ech)
    assert_same(got, ed)
    for a, b in ((cw1, ecw1), (cw2, ecw2), (pr1, epr1), (pr2, epr2)):
        assert np.array_equal(a, b)
    assert O.verify_r1cs_dual(h, wp, 33, got, ch, cw1, cw2, pr1, pr2) == 0


def test_dual_proof_at_the_measured_configuration_matches_oracle():
    """The two-commitment instance the default bench line times: 2^20
    constraints (w1 2^19 rows over 2^18 inputs, w2 16 challenges and
    2^19 - 16 products), m = 20 per commitment, whir-ZK ff 3, rate 1/4,
    128 bits, 10 PoW bits, blinding seed 1, domain 3; generated by the
    library (pkg_synthetic_r1cs_dual, equal to the oracle's generator) and
    proved on the device, word for word equal to the oracle's proof."""
    from provekit_b200.prover import HostDualR1CS, prove_r1cs_dual
    seed = 2 + 11
    h = HostDualR1CS(seed, 1 << 19, 1 << 18, 16, (1 << 19) - 16)
    eh = O.SyntheticDualR1CS(seed, 1 << 19, 1 << 18, 16, (1 << 19) - 16)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    assert m == 20
    got, ch, cw1, cw2, pr1, pr2 = prove_r1cs_dual(h.to_device(), h.w1_size, h.challenge_offsets,
                                                  h.solve, device_params(m, 128, 10, 2),
                                                  blinding_seed=1, transcript_domain=3)
    wp = O.whir_params(m, 3, 2, 128, 10, batch_size=2)
    ed, ech, ecw1, ecw2, epr1, epr2, _ = O.prove_r1cs_dual(eh, 1, 3, wp)
    assert np.array_equal(ch, ech)
    assert_same(got, ed)
    for a, b in ((cw1, ecw1), (cw2, ecw2), (pr1, epr1), (pr2, epr2)):
        assert np.array_equal(a, b)
    assert O.verify_r1cs_dual(eh, wp, 3, got, ch, cw1, cw2, pr1, pr2) == 0


def test_dual_proof_with_a_wrong_challenge_value_fails_the_binding():
    """w2 whose challenge entry differs from the drawn challenge: the device
    proves it (the prover does not check the witness), and the verifier's
    challenge binding rejects it."""
    from provekit_b200.prover import DeviceR1CS, prove_r1cs_dual
    h = O.SyntheticDualR1CS(7, 80, 20, 2, 40)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    wp = O.whir_params(m, 3, 2, 40, 3, batch_size=2)

    def wrong(ch):
        w2 = h.solve(ch)
        w2[int(h.challenge_offsets[1]), 0] ^= 1
        return w2

    got, ch, cw1, cw2, pr1, pr2 = prove_r1cs_dual(DeviceR1CS(h), h.w1_size, h.challenge_offsets,
                                                  wrong, device_params(m, 40, 3, 2))
    assert O.verify_r1cs_dual(h, wp, 3, got, ch, cw1, cw2, pr1, pr2) == 3


def test_dual_prove_state_errors():
    """An offset outside 2^m and a second finish are errors; free is safe on
    a finished state and on NULL; a device proof run after those errors is
    unaffected."""
    import ctypes
    from provekit_b200._lib import PkgError, PKG_ERR_INVALID_ARGUMENT, check, lib
    from provekit_b200.prover import DeviceR1CS, DualProofC, prove_r1cs_dual
    h = O.SyntheticDualR1CS(8, 64, 16, 2, 20)
    m, _ = O.r1cs_sizing_split(h.num_constraints, h.num_witnesses, h.w1_size)
    d = DeviceR1CS(h)
    p = device_params(m, 40, 3, 1)
    with pytest.raises(PkgError) as e:
        prove_r1cs_dual(d, h.w1_size, [0, 1 << m], h.solve, p)
    assert e.value.code == PKG_ERR_INVALID_ARGUMENT
    st = ctypes.c_void_p()
    cw = np.zeros(p.commit_words(), np.uint64)
    ch = np.zeros((2, 4), np.uint64)
    offs = np.ascontiguousarray(h.challenge_offsets, dtype=np.uint64)
    s = torch.cuda.current_stream().cuda_stream
    check(lib().pkg_dual_prove_begin(ctypes.byref(d.c), h.w1_size, offs.ctypes.data, 2,
                                     d.witness.data_ptr(), 1, 3, ctypes.byref(p), cw.ctypes.data,
                                     ch.ctypes.data, ctypes.byref(st), s))
    w2 = torch.from_numpy(h.solve(ch).view(np.int64)).cuda()
    out = DualProofC()
    pr1 = np.zeros(p.proof_words(4), np.uint64)
    pr2 = np.zeros(p.proof_words(4), np.uint64)
    cw2 = np.zeros_like(cw)
    check(lib().pkg_dual_prove_finish(st, w2.data_ptr(), ctypes.byref(out), cw2.ctypes.data,
                                      pr1.ctypes.data, pr2.ctypes.data))
    assert lib().pkg_dual_prove_finish(st, w2.data_ptr(), ctypes.byref(out), cw2.ctypes.data,
                                       pr1.ctypes.data, pr2.ctypes.data) == PKG_ERR_INVALID_ARGUMENT
    lib().pkg_dual_prove_free(st)
    lib().pkg_dual_prove_free(None)
    wp = O.whir_params(m, 3, 2, 40, 3)
    ed = O.prove_r1cs_dual(h, 1, 3, wp)
    assert np.array_equal(pr2, ed[5]) and np.array_equal(pr1, ed[4])
