"""The oracle's Spartan zk-sumcheck driver (run_zk_sumcheck_prover,
provekit/prover/src/whir_r1cs.rs:519-621) checked against what the
reference's verifier checks (provekit/verifier/src/whir_r1cs.rs:266-321,
249-257): every round polynomial satisfies h(0) + h(1) == previous claim, the
first claim is rho * sum_g, and the final claim equals
eq(r, alpha) * (a(alpha) b(alpha) - c(alpha)) + rho * sum_i g_i(alpha_i),
with the multilinear extensions evaluated in plain Python big ints.  CPU only."""
import random

import numpy as np
import pytest

import oracle_lib as O
from fieldutil import P, pack, unpack


def mle(table, point):
    """Multilinear extension, first coordinate bound to the top index bit."""
    t = list(table)
    for x in point:
        h = len(t) // 2
        t = [(t[j] + x * (t[j + h] - t[j])) % P for j in range(h)]
    assert len(t) == 1
    return t[0]


def cubic(c, x):
    return (c[0] + x * (c[1] + x * (c[2] + x * c[3]))) % P


def run_oracle_sumcheck(a, b, c, g, w1, offset, m0, domain=7):
    L = O.lib()
    t = O.Transcript()
    L.pko_transcript_init(O.ctypes.byref(t), O.p64(np.array([domain, 0, 0, 0], np.uint64)))
    A, B, C = pack(a), pack(b), pack(c)
    r = np.zeros((m0, 4), np.uint64)
    rho = np.zeros(4, np.uint64)
    sg = np.zeros(4, np.uint64)
    coeffs = np.zeros((4 * m0, 4), np.uint64)
    alpha = np.zeros((m0, 4), np.uint64)
    be = np.zeros(4, np.uint64)
    rc = L.pko_spartan_sumcheck(O.ctypes.byref(t), O.p64(A), O.p64(B), O.p64(C), m0,
                                O.p64(pack(g)), O.p64(pack(w1)), offset, O.p64(r), O.p64(rho),
                                O.p64(sg), O.p64(coeffs), O.p64(alpha), O.p64(be))
    assert rc == 0
    return (unpack(r), unpack(rho.reshape(1, 4))[0], unpack(sg.reshape(1, 4))[0],
            unpack(coeffs), unpack(alpha), unpack(be.reshape(1, 4))[0])


@pytest.mark.parametrize("m0", [1, 2, 3, 5, 8])
def test_zk_sumcheck_satisfies_verifier_identities(m0):
    rng = random.Random(m0)
    n = 1 << m0
    a = [rng.randrange(P) for _ in range(n)]
    b = [rng.randrange(P) for _ in range(n)]
    c = [x * y % P for x, y in zip(a, b)]
    c[0] = (c[0] + 1) % P  # unsatisfied: the per-round identities still hold
    g = [rng.randrange(P) for _ in range(4 * m0)]
    offset = 3
    w1 = [rng.randrange(P) for _ in range(offset + 4 * m0 + 5)]
    r, rho, sum_g, coeffs, alpha, be = run_oracle_sumcheck(a, b, c, g, w1, offset, m0)
    gs = [g[4 * i: 4 * i + 4] for i in range(m0)]
    assert sum_g == sum(2 ** (m0 - 1) * (cubic(gi, 0) + cubic(gi, 1)) for gi in gs) % P
    # F summed over the hypercube
    eqr = []
    for x in range(n):
        v = 1
        for i in range(m0):
            bit = (x >> (m0 - 1 - i)) & 1
            v = v * (r[i] if bit else (1 - r[i])) % P
        eqr.append(v)
    total_f = sum(e * (x * y - z) for e, x, y, z in zip(eqr, a, b, c)) % P
    claim = rho * sum_g % P
    for i in range(m0):
        cf = coeffs[4 * i: 4 * i + 4]
        assert (2 * cf[0] + cf[1] + cf[2] + cf[3]) % P == claim   # prover's own assert
        claim = cubic(cf, alpha[i])
    # sum F != 0 here, so the final claim cannot match F(alpha) + rho G(alpha)
    # (the next test checks that on satisfied instances)
    assert total_f != 0
    expected_be = 0
    for i in range(m0):
        pw = 1
        for k in range(4):
            expected_be = (expected_be + pw * w1[offset + 4 * i + k]) % P
            pw = pw * alpha[i] % P
    assert be == expected_be


@pytest.mark.parametrize("m0", [1, 2, 4, 7, 10])
def test_zk_sumcheck_final_claim_on_satisfied_instance(m0):
    rng = random.Random(100 + m0)
    n = 1 << m0
    a = [rng.randrange(P) for _ in range(n)]
    b = [rng.randrange(P) for _ in range(n)]
    c = [x * y % P for x, y in zip(a, b)]
    g = [rng.randrange(P) for _ in range(4 * m0)]
    w1 = [rng.randrange(P) for _ in range(4 * m0)]
    r, rho, sum_g, coeffs, alpha, be = run_oracle_sumcheck(a, b, c, g, w1, 0, m0, domain=11)
    gs = [g[4 * i: 4 * i + 4] for i in range(m0)]
    claim = rho * sum_g % P
    for i in range(m0):
        cf = coeffs[4 * i: 4 * i + 4]
        assert (2 * cf[0] + cf[1] + cf[2] + cf[3]) % P == claim
        claim = cubic(cf, alpha[i])
    eq_ra = 1
    for ri, ai in zip(r, alpha):
        eq_ra = eq_ra * (ri * ai + (1 - ri) * (1 - ai)) % P
    f_alpha = eq_ra * (mle(a, alpha) * mle(b, alpha) - mle(c, alpha)) % P
    g_alpha = sum(cubic(gi, ai) for gi, ai in zip(gs, alpha)) % P
    assert claim == (f_alpha + rho * g_alpha) % P


@pytest.mark.parametrize("nc,ni", [(1, 1), (3, 2), (1 << 10, 1 << 8), (5000, 3000)])
def test_synthetic_r1cs_is_satisfied_and_sized_like_new_for_r1cs(nc, ni):
    """pkg_synthetic_r1cs gives A w o B w == C w, and the prove core sizes
    m, m0 as WhirR1CSScheme::new_for_r1cs does
    (provekit/r1cs-compiler/src/whir_r1cs.rs:48-92)."""
    from provekit_b200.prover import HostR1CS
    h = HostR1CS(nc + ni, nc, ni)
    ys = []
    for k in range(3):
        y = np.zeros((nc, 4), np.uint64)
        O.lib().pko_spmv(O.p64(h.row_ptr[k]), O.p32(np.ascontiguousarray(h.cols[k])),
                         O.p64(np.ascontiguousarray(h.vals[k])), nc, O.p64(h.witness), O.p64(y))
        ys.append(unpack(y))
    assert all((x * y - z) % P == 0 for x, y, z in zip(*ys))
    pr = O.spartan_prove(h, 1, 2, 3, 2)
    nw = h.num_witnesses
    clog = lambda n: max(n - 1, 0).bit_length()  # noqa: E731
    m, m0 = max(clog(nw), 13), max(clog(nc), 1)
    if (1 << m) - nw < 4 * m0:
        m += 1
    assert (pr["m"], pr["m0"]) == (m, m0)
