"""Pin the C oracle against the reference's own known-answer vectors
(tests/golden/reference_kats.json, extracted from the reference test modules by
tests/golden/extract_reference_kats.py) and against independent plain-Python
big-int restatements.  CPU only."""
import ctypes
import json
import os
import random

import numpy as np
import pytest

from fieldutil import P, R, RINV, bitrev, from_limbs, pack, root_of_unity, to_limbs, unpack
import oracle_lib as O

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def limbs(x):
    return np.array(to_limbs(x % P), dtype=np.uint64)


# --------------------------------------------------------------------------
# Skyscraper (skyscraper/core/src/reference.rs:104-188)
# --------------------------------------------------------------------------
def test_sbox_table():
    for v, e in KATS["skyscraper"]["test_sbox"]:
        assert O.lib().pko_sky_sbox(v) == e


@pytest.mark.parametrize("name", ["test_ss_2", "test_bb_6", "test_zero", "test_random"])
def test_skyscraper_kat(name):
    k = KATS["skyscraper"][name]
    l, r = limbs(int(k["l"])), limbs(int(k["r"]))
    if k["op"] == "ss":
        O.lib().pko_sky_ss(k["round"], O.p64(l), O.p64(r))
    elif k["op"] == "bb":
        O.lib().pko_sky_bb(k["round"], O.p64(l), O.p64(r))
    else:
        O.lib().pko_sky_permute(O.p64(l), O.p64(r))
    assert from_limbs(l) == int(k["el"])
    assert from_limbs(r) == int(k["er"])


def _compress_via_permute(l, r):
    """reference::compress (reference.rs:41-46): permute(l, r).0 + l."""
    a, b = limbs(l), limbs(r)
    O.lib().pko_sky_permute(O.p64(a), O.p64(b))
    return (from_limbs(a) + l) % P


def test_generic_compress_equals_reference_compress():
    """simple::compress == reference::compress for arbitrary 256-bit inputs
    (skyscraper/core/src/lib.rs tests, test_eq_ref)."""
    rng = random.Random(1)
    cases = [(0, 0), (P - 1, P - 1), (2**256 - 1, 2**256 - 1), (P, 2 * P)]
    cases += [(rng.getrandbits(256), rng.getrandbits(256)) for _ in range(200)]
    for l, r in cases:
        got = O.compress(to_limbs(l), to_limbs(r))
        assert from_limbs(got) == _compress_via_permute(l % P, r % P)


def test_hash_many_left_fold():
    """hash_many(32k) == left fold of compress (skyscraper/whir.rs:139-204)."""
    rng = random.Random(2)
    for size in (32, 64, 128, 256, 512):
        count = 5
        data = bytes(rng.getrandbits(8) for _ in range(size * count))
        out = O.hash_many(size, data, count)
        for i in range(count):
            chunks = [list(np.frombuffer(data[i * size + 32 * k: i * size + 32 * k + 32], dtype=np.uint64))
                      for k in range(size // 32)]
            acc = chunks[0]
            for c in chunks[1:]:
                acc = O.compress(acc, c)
            assert bytes(np.array(acc, dtype=np.uint64).tobytes()) == out[32 * i: 32 * i + 32]


def test_merkle_tree_layers():
    rng = random.Random(3)
    count, leaf = 8, 128
    data = bytes(rng.getrandbits(8) for _ in range(leaf * count))
    layers = O.merkle_tree(data, leaf, count)
    leaves = O.hash_many(leaf, data, count)
    assert layers[: 32 * count] == leaves
    level = [leaves[32 * i: 32 * i + 32] for i in range(count)]
    off = count
    while len(level) > 1:
        nxt = [O.hash_many(64, level[2 * i] + level[2 * i + 1], 1) for i in range(len(level) // 2)]
        assert layers[32 * off: 32 * (off + len(nxt))] == b"".join(nxt)
        off += len(nxt)
        level = nxt


# --------------------------------------------------------------------------
# Field / sampler / NTT
# --------------------------------------------------------------------------
def test_fr_mul_matches_bigint():
    rng = random.Random(4)
    for _ in range(500):
        a, b = rng.randrange(P), rng.randrange(P)
        out = np.zeros(4, np.uint64)
        O.lib().pko_fr_mul(O.p64(out), O.p64(limbs(a)), O.p64(limbs(b)))
        assert from_limbs(out) == a * b * RINV % P


def test_sampler_is_uniform_range_and_deterministic():
    x = O.sample_fr(1, 1000, mont=False)
    vals = [from_limbs(r) for r in x]
    assert all(v < P for v in vals)
    assert len(set(vals)) == 1000
    y = O.sample_fr(1, 1000, mont=True)
    assert [from_limbs(r) for r in y] == [v * R % P for v in vals]
    assert np.array_equal(O.sample_fr(1, 10), O.sample_fr(1, 10))
    assert not np.array_equal(O.sample_fr(1, 10), O.sample_fr(2, 10))


def test_roots_table():
    for order in (2, 4, 16, 1024):
        t = unpack(O.roots(order))
        w = root_of_unity(order)
        bits = (order // 2).bit_length() - 1
        for i in range(order // 2):
            assert t[bitrev(i, bits) if bits else 0] == pow(w, i, P)
    # prefix property (ntt/src/ntt.rs:515-522 roots_direct_vs_extended)
    big, small = O.roots(1 << 12), O.roots(1 << 6)
    assert np.array_equal(big[: small.shape[0]], small)


def py_ntt_nr(vals, codeword_size, num_groups):
    """Independent big-int restatement of interleaved_ntt_nr (ntt/src/ntt.rs:150-248)."""
    vals = list(vals)
    n = len(vals)
    w = root_of_unity(codeword_size)
    half_order = codeword_size // 2
    bits = max(half_order.bit_length() - 1, 0)
    roots = [0] * max(half_order, 1)
    for i in range(half_order):
        roots[bitrev(i, bits) if bits else 0] = pow(w, i, P)
    eig = n // num_groups
    g = num_groups
    while g < codeword_size:
        h = eig // 2
        for k in range(g):
            for i in range(h):
                e, o = vals[k * eig + i], vals[k * eig + h + i]
                t = roots[k] * o % P
                vals[k * eig + i], vals[k * eig + h + i] = (e + t) % P, (e - t) % P
        eig //= 2
        g *= 2
    return vals


def test_ntt_matches_dft_definition():
    """Output[j] = sum_i x_i w^(i * bitrev(j)): normal in, bit-reversed out."""
    rng = random.Random(5)
    for logn in range(0, 7):
        n = 1 << logn
        x = [rng.randrange(P) for _ in range(n)]
        a = pack(x)
        assert O.ntt_nr(a, n, 1) == 0
        got = unpack(a)
        w = root_of_unity(n)
        for j in range(n):
            exp = sum(x[i] * pow(w, i * bitrev(j, logn), P) for i in range(n)) % P
            assert got[j] == exp


@pytest.mark.parametrize("logn,cols,groups", [(4, 1, 1), (5, 3, 1), (6, 4, 2), (7, 2, 8), (8, 1, 4)])
def test_ntt_matches_python_restatement(logn, cols, groups):
    rng = random.Random(logn * 100 + cols)
    n = 1 << logn
    x = [rng.randrange(P) for _ in range(n * cols)]
    a = pack(x)
    assert O.ntt_nr(a, n, groups) == 0
    assert unpack(a) == py_ntt_nr(x, n, groups)


def test_ntt_round_trip():
    """ntt/src/ntt.rs:415-430 round_trip_ntt for sizes 2^0..2^14."""
    for logn in range(0, 15):
        n = 1 << logn
        a = O.sample_fr(100 + logn, n)
        b = a.copy()
        assert O.ntt_nr(b, n, 1) == 0
        assert O.intt_rn(b) == 0
        assert np.array_equal(a, b)


def test_ntt_interleaved_equals_transposed():
    """ntt/src/ntt.rs:488-505 test_interleaved."""
    for rows, cols in [(16, 1), (8, 4), (32, 2), (4, 8), (1, 16)]:
        a = O.sample_fr(rows * 31 + cols, rows * cols)
        ref = a.reshape(rows, cols, 4).transpose(1, 0, 2).copy()
        for c in range(cols):
            col = np.ascontiguousarray(ref[c])
            O.ntt_nr(col, rows, 1)
            ref[c] = col
        b = a.copy()
        O.ntt_nr(b, rows, 1)
        assert np.array_equal(b.reshape(rows, cols, 4), ref.transpose(1, 0, 2))


def test_ntt_edge_cases():
    v = np.zeros((0, 4), np.uint64)
    assert O.ntt_nr(np.zeros((1, 4), np.uint64), 0, 1) == 0  # ntt_empty
    a = O.sample_fr(7, 8)
    assert O.ntt_nr(a.copy(), 8, 0) != 0      # num_groups = 0 panics in the reference
    assert O.ntt_nr(a.copy(), 6, 1) != 0      # non power of two
    assert O.ntt_nr(a.copy()[:6], 4, 1) != 0  # len not a multiple of codeword_size
    b = a.copy()
    assert O.ntt_nr(b, 8, 8) == 0 and np.array_equal(a, b)  # all stages skipped


# --------------------------------------------------------------------------
# RSFr (provekit/common/src/ntt.rs)
# --------------------------------------------------------------------------
def py_rs_encode(msgs, masks, codeword_length):
    M, L = len(msgs), len(msgs[0])
    res = [0] * (M * codeword_length)
    for col in range(L):
        for row in range(M):
            res[col * M + row] = msgs[row][col]
    res[L * M: L * M + len(masks)] = masks
    mlen = len(masks) // M
    cs = 1
    while cs < L + mlen:
        cs *= 2
    while codeword_length % cs:
        cs *= 2
    nc = codeword_length // cs
    chunk = cs * M
    for k in range(1, nc):
        res[k * chunk:(k + 1) * chunk] = res[:chunk]
    return py_ntt_nr(res, codeword_length, nc)


@pytest.mark.parametrize("M,L,mask,cw", [(1, 4, 0, 16), (4, 8, 0, 32), (3, 4, 6, 32), (8, 2, 8, 16), (2, 16, 2, 64)])
def test_rs_encode_matches_python(M, L, mask, cw):
    rng = random.Random(M * 1000 + L * 10 + mask)
    msgs = [[rng.randrange(P) for _ in range(L)] for _ in range(M)]
    masks = [rng.randrange(P) for _ in range(mask)]
    arr = np.stack([pack(m) for m in msgs])
    rc, out = O.rs_interleaved_encode(arr, pack(masks) if masks else np.zeros((0, 4), np.uint64), cw)
    assert rc == 0
    assert unpack(out) == py_rs_encode(msgs, masks, cw)


def test_rs_encode_is_evaluation_at_points():
    """Row i of the codeword holds each message evaluated at w^bitrev(i)
    (provekit/common/src/ntt.rs:22-42 evaluation_points)."""
    rng = random.Random(9)
    M, L, cw = 2, 8, 32
    msgs = [[rng.randrange(P) for _ in range(L)] for _ in range(M)]
    rc, out = O.rs_interleaved_encode(np.stack([pack(m) for m in msgs]), np.zeros((0, 4), np.uint64), cw)
    vals = unpack(out)
    idx = (ctypes_sz := __import__("ctypes").c_size_t * cw)(*range(cw))
    pts = np.zeros((cw, 4), np.uint64)
    O.lib().pko_rs_evaluation_points(cw, idx, cw, O.p64(pts))
    pts = unpack(pts)
    for i in range(cw):
        for m in range(M):
            assert vals[i * M + m] == sum(c * pow(pts[i], k, P) for k, c in enumerate(msgs[m])) % P


# --------------------------------------------------------------------------
# Sumcheck helpers (provekit/common/src/utils/sumcheck.rs:229-436)
# --------------------------------------------------------------------------
def test_calculate_eq_kat():
    k = KATS["sumcheck"]["calculate_eq"]
    r, a = pack(k["r"]), pack(k["alpha"])
    out = np.zeros(4, np.uint64)
    O.lib().pko_calculate_eq(O.p64(out), O.p64(r), O.p64(a), 4)
    assert unpack(out) == [k["expected"] % P]


def test_eq_hypercube_kats():
    r = pack([2, 3, 4, 5])
    out = np.zeros((16, 4), np.uint64)
    assert O.lib().pko_eq_hypercube(O.p64(r), 4, 16, O.p64(out)) == 0
    vals = unpack(out)
    for i in range(16):
        pt = pack([(i >> (3 - j)) & 1 for j in range(4)])
        e = np.zeros(4, np.uint64)
        O.lib().pko_calculate_eq(O.p64(e), O.p64(r), O.p64(pt), 4)
        assert vals[i] == unpack(e)[0]
    t = np.zeros((10, 4), np.uint64)
    O.lib().pko_eq_hypercube(O.p64(r), 4, 10, O.p64(t))
    assert np.array_equal(t, out[:10])
    k = KATS["sumcheck"]["eval_eq_left_only"]
    one = np.zeros((1, 4), np.uint64)
    O.lib().pko_eq_hypercube(O.p64(pack(k["r"])), 3, 1, O.p64(one))
    assert unpack(one) == [k["expected"] % P]
    one2 = np.zeros((1, 4), np.uint64)
    O.lib().pko_eq_hypercube(O.p64(pack([2, 3])), 2, 1, O.p64(one2))
    assert unpack(one2) == [2]


def test_multiply_transposed_by_eq_alpha_kat():
    k = KATS["sumcheck"]
    r1cs = k["test_r1cs"]
    nw = r1cs["num_witnesses"]
    nc = len(r1cs["constraints"])
    exp = k["multiply_transposed_by_eq_alpha"]
    eq = np.zeros((nc, 4), np.uint64)
    O.lib().pko_eq_hypercube(O.p64(pack(exp["alpha"])), len(exp["alpha"]), nc, O.p64(eq))
    for mi, name in enumerate("abc"):
        # transpose: CSR over witnesses (rows of M^T)
        entries = [[] for _ in range(nw)]
        for row, cons in enumerate(r1cs["constraints"]):
            for coef, col in cons[mi]:
                entries[col].append((row, coef))
        row_ptr = np.zeros(nw + 1, np.uint64)
        cols, vals = [], []
        for w in range(nw):
            for row, coef in entries[w]:
                cols.append(row)
                vals.append(coef)
            row_ptr[w + 1] = len(cols)
        y = np.zeros((nw, 4), np.uint64)
        O.lib().pko_spmv(O.p64(row_ptr), O.p32(np.array(cols, np.uint32)), O.p64(pack(vals)), nw,
                         O.p64(eq), O.p64(y))
        assert unpack(y) == [v % P for v in exp["expected"][name]]


# --------------------------------------------------------------------------
# Poseidon2 (poseidon2/src/permutation.rs:182-195, hash.rs:53-70)
# --------------------------------------------------------------------------
def test_poseidon2_permutation_kat():
    k = KATS["poseidon2"]["permutation_zero"]
    st = np.zeros((4, 4), np.uint64)
    O.lib().pko_poseidon2_permutation(O.p64(st))
    assert unpack(st) == [int(x) for x in k["expected"]]


@pytest.mark.parametrize("name", ["hash_single", "hash_two"])
def test_poseidon2_hash_kat(name):
    k = KATS["poseidon2"][name]
    inp = pack([int(x) for x in k["input"]])
    out = np.zeros(4, np.uint64)
    O.lib().pko_poseidon2_hash(O.p64(out), O.p64(inp), inp.shape[0])
    assert unpack(out.reshape(1, 4))[0] == int(k["expected"])


# --------------------------------------------------------------------------
# The NTT's root of unity, pinned to the reference's own constant
# (noir-examples/babyjubjub/src/hash_to_curve.nr: Z = 5, C1 = 28, C5 =
# Z^((p-1)/2^28), the 2^28-th root of unity that ark-bn254's
# Fr::get_root_of_unity squares down to each NTT order).
# --------------------------------------------------------------------------
def test_two_adic_root_matches_the_reference_constant():
    k = KATS["root_of_unity"]
    c5, z, c1 = int(k["two_adic_root"]), int(k["generator"]), int(k["two_adicity"])
    assert c1 == 28 and (P - 1) % (1 << c1) == 0 and ((P - 1) >> c1) % 2 == 1
    assert c5 == pow(z, (P - 1) >> c1, P)
    assert pow(c5, 1 << 27, P) == P - 1          # order exactly 2^28
    assert root_of_unity(1 << 28) == c5            # the tests' helper
    out = np.zeros(4, np.uint64)
    O.lib().pko_fr_root_of_unity.argtypes = [O._u64p, ctypes.c_uint64]
    for logn in (28, 24, 16, 1):
        O.lib().pko_fr_root_of_unity(O.p64(out), 1 << logn)
        assert unpack(out.reshape(1, 4))[0] == pow(c5, 1 << (28 - logn), P)
