"""GPU parity of the WHIR prove-round operations against the oracle (whose
arithmetic is pinned to the reference's Go WHIR verifier on the CPU),
bit-exact, plus the protocol identities on the device: folding the
committed codeword's rows equals encoding the folded coefficients, and the
opened Merkle paths verify against the commit's root."""
import random

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


@pytest.mark.parametrize("k,logn", [(0, 5), (1, 8), (3, 16), (4, 20), (6, 14)])
def test_fold_coeffs_matches_oracle(k, logn):
    from provekit_b200.whir import fold_coeffs
    c = O.sample_fr(100 + logn, 1 << logn)
    alpha = O.sample_fr(200 + k, max(k, 1))[:k]
    exp = O.whir_fold_coeffs(c, k, alpha if k else np.zeros((1, 4), np.uint64))
    assert np.array_equal(host(fold_coeffs(dev(c), k, alpha)), exp)


@pytest.mark.parametrize("k,nrows", [(1, 1000), (3, 1 << 15), (4, 12345), (2, 1)])
def test_fold_rows_matches_oracle(k, nrows):
    from provekit_b200.whir import fold_rows
    rows = O.sample_fr(300 + k, nrows << k)
    alpha = O.sample_fr(301, k)
    assert np.array_equal(host(fold_rows(dev(rows), k, alpha)), O.whir_fold_rows(rows, k, alpha))


def test_fold_commutes_with_the_commit():
    """fold_rows(codeword of whir_commit) == RS encode of fold_coeffs, on the
    device, at the commit's shapes (2^18 coefficients, ff = 3, rate 1/4)."""
    from provekit_b200.merkle import whir_commit
    from provekit_b200.rs import RSFr
    from provekit_b200.whir import fold_coeffs, fold_rows
    n, k, lr = 1 << 18, 3, 2
    c = dev(O.sample_fr(400, n))
    alpha = O.sample_fr(401, k)
    cw, _ = whir_commit(c, k, lr)
    L = n >> k
    folded = fold_coeffs(c, k, alpha)
    enc = RSFr().interleaved_encode(folded.reshape(1, L, 4), None, L << lr)
    assert torch.equal(fold_rows(cw, k, alpha), enc.reshape(-1, 4))


@pytest.mark.parametrize("n", [1, 7, 256, 1 << 16, (1 << 20) + 3])
def test_poly_eval_matches_oracle(n):
    from provekit_b200.whir import poly_eval_many
    c = O.sample_fr(500 + n, n)
    pts = O.sample_fr(501, 3)
    got = poly_eval_many(dev(c), pts)
    for j in range(3):
        assert np.array_equal(got[j], O.poly_eval(c, pts[j]))


def test_poly_eval_of_more_points_than_fused_slots():
    """70 points (above the 64 fused result slots): the partials path."""
    from provekit_b200.whir import poly_eval_many
    c = O.sample_fr(77, 1000)
    pts = O.sample_fr(78, 70)
    got = poly_eval_many(dev(c), pts)
    for j in range(70):
        assert np.array_equal(got[j], O.poly_eval(c, pts[j]))


def test_poly_eval_at_fused_capacity_and_full_grid():
    """Exactly 64 points (every fused result slot) on 2^20 coefficients, so
    each of the 64 back-to-back launches runs the largest evaluation grid (4
    CTAs per SM at 4 coefficients per thread and up) and reuses the one
    ticket the previous launch's last CTA reset: every value equals the
    oracle's."""
    from provekit_b200.whir import poly_eval_many
    n = 1 << 20
    props = torch.cuda.get_device_properties(0)
    assert n // (256 * 4) >= 4 * props.multi_processor_count  # the grid is at its cap
    c = O.sample_fr(79, n)
    pts = O.sample_fr(80, 64)
    got = poly_eval_many(dev(c), pts)
    for j in range(64):
        assert np.array_equal(got[j], O.poly_eval(c, pts[j])), j


@pytest.mark.parametrize("n", [1, 2, 255, 256, 257, 1025, 4099, 65536 + 3, (1 << 21) + 5])
def test_poly_eval_ragged_sizes(n):
    """Sizes that leave the last CTA's chunk, or a thread's strided run,
    short: each CTA's power tree and its z^(bC) scale against the oracle."""
    from provekit_b200.whir import poly_eval_many
    c = O.sample_fr(900 + n % 97, n)
    pts = O.sample_fr(901, 2)
    got = poly_eval_many(dev(c), pts)
    for j in range(2):
        assert np.array_equal(got[j], O.poly_eval(c, pts[j])), (n, j)


def test_merkle_openings_of_the_commit_verify():
    from provekit_b200._lib import PKG_LEAF_CANONICAL
    from provekit_b200.merkle import whir_commit
    from provekit_b200.whir import gather_rows, merkle_open
    n, k, lr = 1 << 16, 3, 2
    M = 1 << k
    c = dev(O.sample_fr(600, n))
    cw, layers = whir_commit(c, k, lr, leaf_encoding=PKG_LEAF_CANONICAL)
    nl = (n >> k) << lr
    depth = nl.bit_length() - 1
    rng = random.Random(5)
    idx = [0, nl - 1] + [rng.randrange(nl) for _ in range(30)]
    paths = merkle_open(layers, nl, idx)
    rows = gather_rows(cw, M, idx)
    lay = layers.cpu().numpy().tobytes()
    root = np.frombuffer(lay[-32:], dtype=np.uint8).copy()
    for q, i in enumerate(idx):
        assert paths[q].tobytes() == O.merkle_open(lay, nl, i)
        assert np.array_equal(rows[q], host(cw)[i * M:(i + 1) * M])
        leaf = np.ascontiguousarray(rows[q]).copy()
        O.lib().pko_from_mont_many(O.p64(leaf), M)          # leaves hash canonical values
        pth = np.ascontiguousarray(paths[q]).reshape(-1).copy()
        assert O.lib().pko_merkle_verify(O.p64(leaf), M, i, O.p8(pth), depth, O.p8(root)) == 1


def test_merkle_open_rejects_out_of_range():
    from provekit_b200 import PkgError
    from provekit_b200.whir import merkle_open
    layers = torch.zeros(32 * 15, dtype=torch.uint8, device="cuda")
    with pytest.raises(PkgError):
        merkle_open(layers, 8, [8])


def test_stir_indices_match_oracle():
    from provekit_b200.whir import stir_indices
    rng = np.random.default_rng(3)
    for folded in (1 << 4, 1 << 9, 1 << 17):
        nb = ((folded.bit_length() - 1) + 7) // 8
        data = rng.integers(0, 256, size=nb * 50, dtype=np.uint8)
        exp = np.zeros(50, np.uint64)
        O.lib().pko_stir_indices(O.p8(data), folded, 50, O.p64(exp))
        assert np.array_equal(stir_indices(data.tobytes(), folded, 50), exp)


def test_sumcheck_rounds_match_oracle_to_the_end():
    from provekit_b200.whir import sumcheck_round
    nv = 18
    f, w = O.sample_fr(700, 1 << nv), O.sample_fr(701, 1 << nv)
    df, dw = dev(f), dev(w)
    size, fold = 1 << nv, None
    for r in range(nv):
        exp = O.whir_sumcheck_round(f, w, size, fold)
        got = sumcheck_round(df, dw, size, fold)
        assert np.array_equal(got, exp), r
        if fold is not None:
            size //= 2
        fold = O.sample_fr(800 + r, 1)[0]
    live = size
    assert np.array_equal(host(df)[:live], f[:live])


def test_eq_accumulate_matches_oracle():
    """Fewer than four points take a product per term; from four on the
    products are summed unreduced (fr_lazy.cuh), past 32 points with carry
    steps and past 1024 in several lazy chunks."""
    from provekit_b200.whir import eq_accumulate
    for nv, npts in ((0, 2), (1, 3), (9, 7), (17, 40), (3, 4), (6, 33), (4, 1100), (12, 119)):
        w = O.sample_fr(900 + nv, 1 << nv)
        pts = O.sample_fr(901, max(npts * nv, 1))[: npts * nv]
        cf = O.sample_fr(902, npts)
        dw = dev(w)
        eq_accumulate(dw, nv, pts if nv else np.zeros((1, 4), np.uint64), cf)
        exp = w.copy()
        assert O.lib().pko_eq_accumulate(O.p64(exp), nv, O.p64(np.ascontiguousarray(pts) if nv else
                                         np.zeros((1, 4), np.uint64)), O.p64(cf), npts) == 0
        assert np.array_equal(host(dw), exp)
