"""GPU parity: every CUDA entry point against the C oracle on the same seeded
inputs, bit-exact (exact modular integer arithmetic admits no tolerance).
Calls go through the C ABI (provekit_b200's ctypes binding)."""
import numpy as np
import pytest
import torch

import oracle_lib as O
from fieldutil import P, to_limbs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()
    from provekit_b200 import _lib as L
    return L.lib()


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(a.view(np.int64).copy()).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


# --------------------------------------------------------------------------
# NTT
# --------------------------------------------------------------------------
@pytest.mark.parametrize("logn", list(range(0, 17)))
def test_ntt_nr_sizes(logn):
    from provekit_b200.ntt import ntt_nr
    n = 1 << logn
    a = O.sample_fr(1000 + logn, n)
    d = dev(a)
    ntt_nr(d, n, 1)
    exp = a.copy()
    assert O.ntt_nr(exp, n, 1) == 0
    assert np.array_equal(host(d), exp)


@pytest.mark.parametrize("logn,cols,groups", [
    (4, 2, 1), (5, 3, 1), (6, 16, 4), (10, 8, 2), (12, 5, 1), (13, 16, 8), (14, 1, 4),
    (16, 16, 4), (11, 7, 2), (9, 12, 1), (18, 2, 2)])
def test_ntt_nr_interleaved_and_skipped_stages(logn, cols, groups):
    from provekit_b200.ntt import ntt_nr
    n = 1 << logn
    a = O.sample_fr(77 + logn * cols, n * cols)
    d = dev(a)
    ntt_nr(d, n, groups)
    exp = a.copy()
    assert O.ntt_nr(exp, n, groups) == 0
    assert np.array_equal(host(d), exp)


def test_ntt_2_16_single_vector_bit_exact_and_round_trip():
    """2^16 Fr from ChaCha seed 1, ntt_nr(v, 2^16, 1); bit-exact against the
    oracle, and intt_rn round-trips to the input."""
    from provekit_b200.ntt import intt_rn, ntt_nr
    n = 1 << 16
    a = O.sample_fr(1, n)
    d = dev(a)
    ntt_nr(d, n, 1)
    exp = a.copy()
    O.ntt_nr(exp, n, 1)
    assert np.array_equal(host(d), exp)
    intt_rn(d)
    assert np.array_equal(host(d), a)


@pytest.mark.parametrize("logn", [0, 1, 2, 5, 10, 15])
def test_intt_rn_matches_oracle(logn):
    from provekit_b200.ntt import intt_rn
    n = 1 << logn
    a = O.sample_fr(500 + logn, n)
    d = dev(a)
    intt_rn(d)
    exp = a.copy()
    assert O.intt_rn(exp) == 0
    assert np.array_equal(host(d), exp)


def test_ntt_2_22_bit_exact():
    from provekit_b200.ntt import ntt_nr
    n = 1 << 22
    a = O.sample_fr(22, n)
    d = dev(a)
    ntt_nr(d, n, 1)
    exp = a.copy()
    O.ntt_nr(exp, n, 1)
    assert np.array_equal(host(d), exp)


def test_ntt_2_24_round_trip_and_linearity():
    """Full-size properties: intt(ntt(x)) == x and ntt(x + y) == ntt(x) + ntt(y)
    checked via a sampled subset of outputs against the oracle."""
    from provekit_b200.ntt import intt_rn, ntt_nr
    n = 1 << 24
    a = O.sample_fr(24, n)
    d = dev(a)
    ntt_nr(d, n, 1)
    out = host(d)
    exp = a.copy()
    O.ntt_nr(exp, n, 1)
    assert np.array_equal(out, exp)
    intt_rn(d)
    assert np.array_equal(host(d), a)


def test_ntt_errors_raise():
    from provekit_b200 import PkgError
    from provekit_b200.ntt import ntt_nr
    d = dev(O.sample_fr(3, 8))
    with pytest.raises(PkgError):
        ntt_nr(d, 6, 1)
    with pytest.raises(PkgError):
        ntt_nr(d, 8, 0)


def test_host_forms():
    from provekit_b200.ntt import host_intt_rn, host_ntt_nr
    a = O.sample_fr(4, 1 << 10)
    got = host_ntt_nr(a.copy(), 1 << 10, 1)
    exp = a.copy()
    O.ntt_nr(exp, 1 << 10, 1)
    assert np.array_equal(got, exp)
    assert np.array_equal(host_intt_rn(got), a)


# --------------------------------------------------------------------------
# RSFr interleaved_encode
# --------------------------------------------------------------------------
@pytest.mark.parametrize("M,L,mask,cw", [
    (1, 1, 0, 1), (1, 4, 0, 16), (4, 8, 0, 32), (3, 4, 6, 32), (8, 2, 8, 16), (2, 16, 2, 64),
    (16, 64, 0, 256), (8, 1024, 8 * 16, 8192), (1, 0, 0, 8), (5, 3, 0, 16), (2, 4, 3, 8)])
def test_rs_encode_matches_oracle(M, L, mask, cw):
    from provekit_b200.rs import RSFr
    msgs = O.sample_fr(M * 1000 + L, M * L).reshape(M, L, 4) if L else np.zeros((M, 0, 4), np.uint64)
    masks = O.sample_fr(9, mask) if mask else np.zeros((0, 4), np.uint64)
    rc, exp = O.rs_interleaved_encode(msgs, masks, cw)
    assert rc == 0
    got = RSFr().interleaved_encode(dev(msgs.reshape(M, L, 4)) if L else torch.zeros((M, 0, 4), dtype=torch.int64, device="cuda"),
                                    dev(masks) if mask else None, cw)
    assert np.array_equal(host(got), exp)


def test_rs_encode_commit_shape_bit_exact():
    """2^20 coefficients as 16 messages of 2^16, rate 1/4 -> 2^22 evaluations."""
    from provekit_b200.rs import RSFr
    M, L, cw = 16, 1 << 16, 1 << 18
    msgs = O.sample_fr(2, M * L).reshape(M, L, 4)
    rc, exp = O.rs_interleaved_encode(msgs, np.zeros((0, 4), np.uint64), cw)
    got = RSFr().interleaved_encode(dev(msgs), None, cw)
    assert np.array_equal(host(got), exp)


def test_rs_host_form_with_message_list():
    from provekit_b200.rs import RSFr
    M, L, cw = 3, 8, 32
    msgs = [O.sample_fr(40 + j, L) for j in range(M)]
    masks = O.sample_fr(41, 6)
    rc, exp = O.rs_interleaved_encode(np.stack(msgs), masks, cw)
    got = RSFr().host_interleaved_encode(msgs, masks, cw)
    assert np.array_equal(got, exp)


# --------------------------------------------------------------------------
# Skyscraper
# --------------------------------------------------------------------------
def edge_messages():
    vals = [0, 1, P - 1, P, P + 1, 2 * P - 1, 2 * P, 5 * P, 2**256 - 1, 2**255, 2**254]
    rows = []
    for l in vals:
        for r in vals:
            rows.append(to_limbs(l) + to_limbs(r))
    return np.array(rows, dtype=np.uint64)


def test_compress_many_edges_and_random():
    from provekit_b200.skyscraper import compress_many
    rng = np.random.default_rng(5)
    msgs = np.concatenate([edge_messages(), rng.integers(0, 2**63, size=(5000, 8), dtype=np.uint64) * 2 + 1])
    raw = np.ascontiguousarray(msgs).view(np.uint8).reshape(-1)
    exp = np.zeros(32 * msgs.shape[0], np.uint8)
    O.lib().pko_sky_compress_many(O.p8(raw), msgs.shape[0], O.p8(exp))
    got = compress_many(torch.from_numpy(raw.copy()).cuda())
    assert np.array_equal(got.cpu().numpy(), exp)


@pytest.mark.parametrize("size", [32, 64, 96, 128, 256, 512, 1024])
def test_hash_many_matches_oracle(size):
    from provekit_b200.skyscraper import SkyscraperHashEngine
    rng = np.random.default_rng(size)
    count = 1000
    data = rng.integers(0, 256, size=size * count, dtype=np.uint8)
    exp = O.hash_many(size, data.tobytes(), count)
    got = SkyscraperHashEngine().hash_many(size, torch.from_numpy(data.copy()).cuda())
    assert got.cpu().numpy().tobytes() == exp
    assert SkyscraperHashEngine().host_hash_many(size, data.tobytes()) == exp


def test_hash_many_rejects_unsupported_size():
    from provekit_b200 import PkgError
    from provekit_b200.skyscraper import SkyscraperHashEngine
    with pytest.raises(PkgError):
        SkyscraperHashEngine().hash_many(48, torch.zeros(96, dtype=torch.uint8, device="cuda"))


# --------------------------------------------------------------------------
# Merkle trees and the commit
# --------------------------------------------------------------------------
@pytest.mark.parametrize("count,leaf", [(1, 64), (2, 32), (8, 128), (256, 64), (512, 32), (1024, 256),
                                        (2048, 64), (4096, 512), (1 << 15, 64), (1 << 16, 32),
                                        (1 << 17, 64)])
def test_merkle_tree_bytes(count, leaf):
    """Leaf counts on both sides of the tree's launch thresholds: the top
    kernel alone (<= 256 nodes), the 256-node subtree kernel from 512 nodes,
    and per-level launches above 2^15 nodes."""
    from provekit_b200.merkle import merkle_tree
    rng = np.random.default_rng(count + leaf)
    data = rng.integers(0, 256, size=count * leaf, dtype=np.uint8)
    exp = O.merkle_tree(data.tobytes(), leaf, count)
    got = merkle_tree(torch.from_numpy(data.copy()).cuda(), leaf)
    assert got.cpu().numpy().tobytes() == exp


@pytest.mark.parametrize("encoding", [0, 1])
def test_merkle_tree_fr_encodings(encoding):
    from provekit_b200.merkle import merkle_tree_fr
    M, count = 8, 4096
    cw = O.sample_fr(11, M * count)
    leaves = cw.copy()
    if encoding == 0:
        O.lib().pko_from_mont_many(O.p64(leaves), leaves.shape[0])
    exp = O.merkle_tree(leaves.tobytes(), 32 * M, count)
    got = merkle_tree_fr(dev(cw), M, encoding)
    assert got.cpu().numpy().tobytes() == exp


@pytest.mark.parametrize("ff", [3, 4])
def test_whir_commit_2_20_bit_exact(ff):
    """Config-2 commit: 2^20 coefficients, 2^ff messages, rate 1/4, 2^22
    evaluations, leaves of 2^ff Fr; codeword and every tree layer bit-exact."""
    from provekit_b200.merkle import whir_commit
    n, M = 1 << 20, 1 << ff
    coeffs = O.sample_fr(2, n)
    L = n // M
    rc, cw_exp = O.rs_interleaved_encode(coeffs.reshape(M, L, 4), np.zeros((0, 4), np.uint64), 4 * L)
    canon = cw_exp.copy()
    O.lib().pko_from_mont_many(O.p64(canon), canon.shape[0])
    layers_exp = O.merkle_tree(canon.tobytes(), 32 * M, 4 * L)
    cw, layers = whir_commit(dev(coeffs), ff, 2)
    assert np.array_equal(host(cw), cw_exp)
    assert layers.cpu().numpy().tobytes() == layers_exp


def test_pow_solve_matches_oracle():
    from provekit_b200.skyscraper import pow_solve
    challenge = [42, 43, 44, 45]
    threshold = [0, 0, 0, 1 << 52]  # ~10 bits of work
    exp = O.lib().pko_sky_pow_solve(O.p64(np.array(challenge, np.uint64)), O.p64(np.array(threshold, np.uint64)))
    assert pow_solve(challenge, threshold) == exp
