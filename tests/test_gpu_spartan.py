"""GPU parity of the Spartan side: eq tables, SpMV and transpose, Hadamard
witness bounds, dot products, single sumcheck rounds and the whole
zk-sumcheck driver against the C oracle, bit-exact."""
import ctypes

import numpy as np
import pytest
import torch

import oracle_lib as O
from fieldutil import P, pack, unpack

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
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("nr,entries", [(0, 1), (1, 2), (4, 16), (4, 10), (7, 100), (11, 2048), (20, 1 << 20), (20, 700001)])
def test_eq_hypercube(nr, entries):
    from provekit_b200.spartan import eq_hypercube
    r = O.sample_fr(300 + nr, nr) if nr else np.zeros((0, 4), np.uint64)
    exp = np.zeros((entries, 4), np.uint64)
    assert O.lib().pko_eq_hypercube(O.p64(r) if nr else None, nr, entries, O.p64(exp)) == 0
    got = eq_hypercube(r, entries)
    assert np.array_equal(host(got), exp)


def random_csr(rng, rows, cols, max_nnz=3):
    counts = rng.integers(0, max_nnz + 1, size=rows)
    row_ptr = np.zeros(rows + 1, np.uint64)
    row_ptr[1:] = np.cumsum(counts)
    nnz = int(row_ptr[-1])
    col = rng.integers(0, cols, size=nnz).astype(np.uint32)
    vals = O.sample_fr(int(rng.integers(1 << 30)), nnz)
    return row_ptr, col, vals


@pytest.mark.parametrize("rows,cols", [(1, 1), (3, 4), (1000, 777), (1 << 16, 1 << 15), (1 << 20, 1 << 21)])
def test_spmv_and_transpose(rows, cols):
    from provekit_b200.spartan import CsrMatrix
    rng = np.random.default_rng(rows)
    row_ptr, col, vals = random_csr(rng, rows, cols)
    x = O.sample_fr(5, cols)
    y_exp = np.zeros((rows, 4), np.uint64)
    O.lib().pko_spmv(O.p64(row_ptr), O.p32(col) if col.size else None, O.p64(vals) if vals.size else None,
                     rows, O.p64(x), O.p64(y_exp))
    m = CsrMatrix.from_host(rows, cols, row_ptr, col, vals)
    y = m.mul(dev(x))
    assert np.array_equal(host(y), y_exp)
    # transposed product == oracle product with the host transpose
    z = O.sample_fr(6, rows)
    order = np.argsort(col, kind="stable")
    row_of = np.repeat(np.arange(rows, dtype=np.uint32), np.diff(row_ptr).astype(np.int64))
    t_ptr = np.zeros(cols + 1, np.uint64)
    t_ptr[1:] = np.cumsum(np.bincount(col, minlength=cols))
    t_cols = np.ascontiguousarray(row_of[order])
    t_vals = np.ascontiguousarray(vals[order]) if vals.size else vals
    w_exp = np.zeros((cols, 4), np.uint64)
    O.lib().pko_spmv(O.p64(t_ptr), O.p32(t_cols) if t_cols.size else None,
                     O.p64(t_vals) if t_vals.size else None, cols, O.p64(z), O.p64(w_exp))
    mt = m.transpose()
    assert np.array_equal(host(mt.row_ptr), t_ptr)
    w = mt.mul(dev(z))
    assert np.array_equal(host(w), w_exp)


def test_multiply_transposed_by_eq_alpha_reference_vectors():
    """provekit/common/src/utils/sumcheck.rs:417-435 on the device."""
    import json
    import os
    from provekit_b200.spartan import CsrMatrix, eq_hypercube
    k = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))["sumcheck"]
    r1cs, exp = k["test_r1cs"], k["multiply_transposed_by_eq_alpha"]
    nw, nc = r1cs["num_witnesses"], len(r1cs["constraints"])
    eq = eq_hypercube(pack(exp["alpha"]), nc)
    for mi, name in enumerate("abc"):
        row_ptr, cols, vals = [0], [], []
        for cons in r1cs["constraints"]:
            for coef, col in cons[mi]:
                cols.append(col)
                vals.append(coef)
            row_ptr.append(len(cols))
        m = CsrMatrix.from_host(nc, nw, np.array(row_ptr, np.uint64), np.array(cols, np.uint32), pack(vals))
        got = m.transpose().mul(eq)
        assert unpack(host(got)) == [v % P for v in exp["expected"][name]]


def test_hadamard_and_dot():
    from provekit_b200.spartan import dot, hadamard_pad
    n, padded = 1000003, 1 << 20
    a, b = O.sample_fr(8, n), O.sample_fr(9, n)
    c = hadamard_pad(dev(a), dev(b), n, padded)
    ca = unpack(host(c)[:5])
    av, bv = unpack(a[:5]), unpack(b[:5])
    assert ca == [x * y % P for x, y in zip(av, bv)]
    assert not host(c)[n:].any()
    exp = np.zeros(4, np.uint64)
    O.lib().pko_dot(O.p64(exp), O.p64(a), O.p64(b), n)
    assert np.array_equal(dot(dev(a), dev(b)), exp)


@pytest.mark.parametrize("n", [1, 7, 33, 5_000_011])
def test_dot_lazy_sums_match_oracle(n):
    """pkg_dot sums its products unreduced and reduces once per thread; at
    5M entries every thread sums more than 32 terms (the carry step)."""
    from provekit_b200.spartan import dot
    a, b = O.sample_fr(30 + n % 7, n), O.sample_fr(31 + n % 5, n)
    exp = np.zeros(4, np.uint64)
    O.lib().pko_dot(O.p64(exp), O.p64(a), O.p64(b), n)
    assert np.array_equal(dot(dev(a), dev(b)), exp)


def test_dot_of_maximal_values_past_one_lazy_chunk():
    """2^28 + 3 entries of p - 1 (Montgomery limbs) in both vectors: the
    largest operands, and more than 1024 terms per thread, so each thread
    finishes several lazy sums.  The expected value is computed in Python
    integers: n (p-1)^2 2^-256 mod p."""
    from provekit_b200.spartan import dot
    n = (1 << 28) + 3
    pm1 = np.array([P - 1 >> (64 * i) & (2**64 - 1) for i in range(4)], np.uint64)
    a = torch.from_numpy(pm1.view(np.int64)).cuda().reshape(1, 4).expand(n, 4).contiguous()
    got = unpack(dot(a, a).reshape(1, 4), mont=False)[0]
    del a
    torch.cuda.empty_cache()
    assert got == n * (P - 1) ** 2 * pow(2, -256, P) % P


@pytest.mark.parametrize("size,fold", [(2, False), (4, False), (4, True), (8, True), (1 << 12, True), (1 << 20, False), (1 << 20, True)])
def test_spartan_round(size, fold):
    from provekit_b200.spartan import spartan_round
    tabs = [O.sample_fr(40 + k + size % 97, size) for k in range(4)]
    f = O.sample_fr(99, 1)[0] if fold else None
    exp_tabs = [t.copy() for t in tabs]
    exp = np.zeros((3, 4), np.uint64)
    assert O.lib().pko_spartan_round(*[O.p64(t) for t in exp_tabs], size,
                                     O.p64(np.ascontiguousarray(f)) if fold else None, O.p64(exp)) == 0
    d = [dev(t) for t in tabs]
    got = spartan_round(*d, size, fold=f)
    assert np.array_equal(got, exp)
    live = size // 2 if fold else size
    for t, e in zip(d, exp_tabs):
        assert np.array_equal(host(t)[:live], e[:live])


@pytest.mark.parametrize("m0", [1, 2, 3, 9, 16, 20])
def test_spartan_sumcheck_matches_oracle(m0):
    from provekit_b200.spartan import Transcript, spartan_sumcheck
    n = 1 << m0
    a, b = O.sample_fr(1000 + m0, n), O.sample_fr(2000 + m0, n)
    c = O.sample_fr(3000 + m0, n)
    g = O.sample_fr(4000 + m0, 4 * m0)
    offset = 5
    w1 = O.sample_fr(5000 + m0, offset + 4 * m0)
    # oracle
    t = O.Transcript()
    O.lib().pko_transcript_init(ctypes.byref(t), O.p64(np.array([42, 0, 0, 0], np.uint64)))
    ea, eb, ec = a.copy(), b.copy(), c.copy()
    r = np.zeros((m0, 4), np.uint64); rho = np.zeros(4, np.uint64); sg = np.zeros(4, np.uint64)
    cf = np.zeros((4 * m0, 4), np.uint64); al = np.zeros((m0, 4), np.uint64); be = np.zeros(4, np.uint64)
    assert O.lib().pko_spartan_sumcheck(ctypes.byref(t), O.p64(ea), O.p64(eb), O.p64(ec), m0, O.p64(g),
                                        O.p64(w1), offset, O.p64(r), O.p64(rho), O.p64(sg), O.p64(cf),
                                        O.p64(al), O.p64(be)) == 0
    # GPU
    tr = Transcript.new(42)
    out = spartan_sumcheck(dev(a), dev(b), dev(c), m0, g, w1[offset: offset + 4 * m0], tr)
    assert np.array_equal(out["r"], r)
    assert np.array_equal(out["rho"], rho) and np.array_equal(out["sum_g"], sg)
    assert np.array_equal(out["coeffs"], cf)
    assert np.array_equal(out["alpha"], al)
    assert np.array_equal(out["blinding_eval"], be)
    assert list(tr.l) == list(t.l) and list(tr.r) == list(t.r)


def test_spmv_balanced_path_rejects_out_of_range_column():
    """Above 2^16 nonzeros the product runs as two balanced passes; a column
    index past the vector is still reported, not read."""
    from provekit_b200 import PkgError
    from provekit_b200.spartan import CsrMatrix
    rng = np.random.default_rng(31)
    rows, cols = 1 << 15, 1 << 14
    row_ptr, col, vals = random_csr(rng, rows, cols, max_nnz=6)
    assert int(row_ptr[-1]) >= 1 << 16
    col[len(col) // 2] = cols + 5
    m = CsrMatrix.from_host(rows, cols, row_ptr, col, vals)
    with pytest.raises(PkgError):
        m.mul(dev(O.sample_fr(2, cols)))


def test_spmv_rejects_out_of_range_column():
    from provekit_b200 import PkgError
    from provekit_b200.spartan import CsrMatrix
    m = CsrMatrix.from_host(2, 3, np.array([0, 1, 2], np.uint64), np.array([1, 7], np.uint32),
                            O.sample_fr(1, 2))
    with pytest.raises(PkgError):
        m.mul(dev(O.sample_fr(2, 3)))
    with pytest.raises(PkgError):
        m.transpose()
