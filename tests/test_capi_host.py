"""CPU-side checks of the C ABI: the library loads, exports every symbol the
header declares, and its host-only logic (sampler, RS planning, argument
validation) agrees with the oracle.  No GPU compute is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

from fieldutil import root_of_unity, unpack
import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    from provekit_b200 import build
    build.build()
    from provekit_b200 import _lib
    return _lib.lib()


def header_symbols():
    src = open(os.path.join(ROOT, "include", "provekit_b200.h")).read()
    return sorted(set(re.findall(r"\b(pkg_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(L):
    from provekit_b200 import _lib
    declared = header_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(L, name), f"{name} declared but not exported"
    # the Python binding covers every declared entry point
    assert set(declared) <= set(_lib.exported_symbols())


def test_sampler_matches_oracle(L):
    for seed, n in [(1, 1), (2, 100), (3, 4097)]:
        a = np.zeros((n, 4), np.uint64)
        assert L.pkg_sample_fr(seed, n, a.ctypes.data, 1) == 0
        assert np.array_equal(a, O.sample_fr(seed, n, mont=True))
        b = np.zeros((n, 4), np.uint64)
        assert L.pkg_sample_fr(seed, n, b.ctypes.data, 0) == 0
        assert np.array_equal(b, O.sample_fr(seed, n, mont=False))


def test_rs_host_helpers_match_oracle(L):
    from provekit_b200.rs import RSFr
    rs = RSFr()
    assert rs.next_order(0) == 1 and rs.next_order(5) == 8 and rs.next_order(1 << 28) == 1 << 28
    assert rs.next_order((1 << 28) + 1) is None
    for n in (1, 2, 1024, 1 << 20, 1 << 28):
        g = rs.generator(n)
        assert unpack(g.reshape(1, 4))[0] == root_of_unity(n)
    rng = np.random.default_rng(5)
    for cw in (1, 2, 16, 64, 1 << 19, 1 << 20, 1 << 23, 1 << 28):
        idx = list(range(min(cw, 64))) + [cw + 3, cw - 1]
        idx += [int(x) for x in rng.integers(0, cw, 40)]
        got = rs.evaluation_points(0, cw, idx)
        exp = np.zeros((len(idx), 4), np.uint64)
        arr = (ctypes.c_size_t * len(idx))(*idx)
        O.lib().pko_rs_evaluation_points(cw, arr, len(idx), O.p64(exp))
        assert np.array_equal(got, exp)


@pytest.mark.parametrize("len_,cw,groups", [(8, 6, 1), (8, 8, 0), (8, 8, 3), (6, 4, 1), (0, 4, 1)])
def test_ntt_validation_rejects_like_reference(L, len_, cw, groups):
    """Contract violations the reference panics on come back as
    PKG_ERR_INVALID_ARGUMENT before any device work."""
    assert L.pkg_ntt_nr(None, len_, cw, groups, None) == -1
    assert L.pkg_last_error()


def test_ntt_noop_cases_need_no_device(L):
    assert L.pkg_ntt_nr(None, 0, 0, 1, None) == 0   # ntt_empty
    assert L.pkg_ntt_nr(None, 4, 1, 1, None) == 0   # codeword_size <= 1


def test_hash_many_rejects_bad_sizes(L):
    for size in (0, 1, 31, 33):
        assert L.pkg_skyscraper_hash_many(size, None, 1, None, None) == -1
        assert b"unsupported message size" in L.pkg_last_error()


def test_rs_encode_validation(L):
    assert L.pkg_rs_interleaved_encode(None, 0, 4, None, 0, 16, None, None) == 0  # no messages
    assert L.pkg_rs_interleaved_encode(None, 2, 32, None, 0, 16, None, None) == -1
    assert L.pkg_rs_interleaved_encode(None, 2, 8, None, 32, 16, None, None) == -1
    assert L.pkg_rs_interleaved_encode(None, 3, 4, None, 0, 12, None, None) == -1


def test_merkle_requires_power_of_two_leaves(L):
    assert L.pkg_merkle_tree_fr(None, 4, 6, 0, None, None) == -1
    assert L.pkg_merkle_tree_fr(None, 4, 8, 7, None, None) == -1


def test_transcript_matches_oracle(L):
    """The library's host transcript (pkg_transcript_*) and the oracle's agree
    message by message; both run the KAT-pinned Skyscraper permutation."""
    from provekit_b200.spartan import Transcript
    for domain in (0, 42, (1 << 255) + 12345):
        t = Transcript.new(domain)
        o = O.Transcript()
        d = np.array([(domain >> (64 * i)) & (2**64 - 1) for i in range(4)], np.uint64)
        O.lib().pko_transcript_init(ctypes.byref(o), O.p64(d))
        assert list(t.l) == list(o.l) and list(t.r) == list(o.r)
        xs = O.sample_fr(domain % 1000 + 1, 6)
        for x in xs:
            t.absorb(x)
            O.lib().pko_transcript_absorb(ctypes.byref(o), O.p64(np.ascontiguousarray(x)))
            a = t.squeeze()
            b = np.zeros(4, np.uint64)
            O.lib().pko_transcript_squeeze(ctypes.byref(o), O.p64(b))
            assert np.array_equal(a, b)


def test_whir_schedule_and_sizes_match_oracle(L):
    """pkg_whir_params_init / pkg_whir_proof_words (host only) agree with the
    oracle for every shape, and bad shapes are refused."""
    from provekit_b200.whir import WhirParams
    from provekit_b200._lib import PkgError
    for n in range(1, 25):
        for k in range(1, 7):
            if k > n:
                continue
            for lr, sec, pw in ((1, 40, 0), (2, 128, 10), (3, 100, 20)):
                try:
                    p = WhirParams.new(n, k, lr, sec, pw)
                except PkgError:
                    po = O.WhirParams()
                    assert O.lib().pko_whir_params_init(ctypes.byref(po), n, k, lr, sec, pw) != 0
                    continue
                po = O.whir_params(n, k, lr, sec, pw)
                assert bytes(p) == bytes(po)
                for ncov in (0, 3):
                    assert p.proof_words(ncov) == O.lib().pko_whir_proof_words(
                        ctypes.byref(po), ncov)
                assert p.commit_words() == O.lib().pko_whir_commit_words(ctypes.byref(po))
    bad = WhirParams.new(12, 3, 2, 64, 4)
    bad.final_vars += 1
    assert L.pkg_whir_proof_words(ctypes.byref(bad), 1) == 0
    with pytest.raises(PkgError):
        WhirParams.new(8, 7, 2, 64, 4)


def test_transcript_bytes_match_oracle(L):
    from provekit_b200.spartan import Transcript
    from provekit_b200.whir import squeeze_bytes
    for n in (0, 1, 30, 31, 32, 62, 100):
        t = Transcript.new(9)
        o = O.transcript(9)
        out = np.zeros(max(n, 1), np.uint8)
        O.lib().pko_transcript_squeeze_bytes(ctypes.byref(o), O.p8(out), n)
        assert squeeze_bytes(t, n) == out[:n].tobytes()
        assert list(t.l) == list(o.l) and list(t.r) == list(o.r)


def test_whir_prove_validation_needs_no_device(L):
    """Invalid parameters and null pointers are refused before any device work."""
    from provekit_b200.whir import WhirParams
    from provekit_b200._lib import PKG_ERR_INVALID_ARGUMENT
    from provekit_b200.spartan import Transcript
    p = WhirParams.new(10, 3, 2, 64, 4)
    t = Transcript.new(1)
    proof = np.zeros(p.proof_words(0), np.uint64)
    assert L.pkg_whir_prove(ctypes.byref(p), ctypes.byref(t), None, None, None, None, None, 0,
                            proof.ctypes.data, None) == PKG_ERR_INVALID_ARGUMENT
    p.queries[0] = 0
    assert L.pkg_whir_prove(ctypes.byref(p), ctypes.byref(t), 16, 16, 16, None, None, 0,
                            proof.ctypes.data, None) == PKG_ERR_INVALID_ARGUMENT
    assert L.pkg_subset_transform(None, 4, 0, None) == PKG_ERR_INVALID_ARGUMENT
    assert L.pkg_subset_transform(16, 4, 7, None) == PKG_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("nc,nw", [(1, 1), (3, 5), (1 << 10, 1 << 9), (1000, 70000),
                                   (1 << 20, (1 << 18) + (1 << 20) + 1), (5, 4 * 13 + 8200)])
def test_r1cs_sizing_matches_oracle(nc, nw):
    """new_for_r1cs sizing (m, m0), with the blinding slots' extra variable."""
    from provekit_b200.prover import r1cs_sizing
    assert r1cs_sizing(nc, nw) == O.r1cs_sizing(nc, nw)


def test_prove_r1cs_validation_needs_no_device(L):
    """pkg_prove_r1cs refuses bad arguments before any device work: no WHIR
    parameters, parameters for another variable count, a batch other than
    1 or 2, as many public inputs as witnesses, null outputs."""
    from provekit_b200.prover import R1csC, SpartanProofC, r1cs_sizing
    from provekit_b200.whir import WhirParams
    from provekit_b200._lib import PKG_ERR_INVALID_ARGUMENT
    nc, nw = 1 << 10, (1 << 9) + (1 << 10) + 1
    m, _ = r1cs_sizing(nc, nw)
    r = R1csC(nc, nw)
    out = SpartanProofC()
    w = np.zeros(4 * 16, np.uint64)
    wptr = (w.ctypes.data + 15) // 16 * 16
    cw = np.zeros(64, np.uint64)

    def prove(p, r1cs=r, words=cw.ctypes.data, proof=cw.ctypes.data):
        return L.pkg_prove_r1cs(ctypes.byref(r1cs), wptr, 1, 2,
                                None if p is None else ctypes.byref(p), ctypes.byref(out),
                                words, proof, None)

    assert prove(None) == PKG_ERR_INVALID_ARGUMENT
    assert prove(WhirParams.new(m + 1, 3, 2, 64, 4)) == PKG_ERR_INVALID_ARGUMENT
    assert prove(WhirParams.new(m, 3, 2, 64, 4, batch_size=4)) == PKG_ERR_INVALID_ARGUMENT
    good = WhirParams.new(m, 3, 2, 64, 4, batch_size=2)
    assert prove(good, words=None) == PKG_ERR_INVALID_ARGUMENT
    assert prove(good, proof=None) == PKG_ERR_INVALID_ARGUMENT
    many = R1csC(nc, nw)
    many.num_public_inputs = nw
    assert prove(good, r1cs=many) == PKG_ERR_INVALID_ARGUMENT
    assert L.pkg_prove_r1cs(ctypes.byref(r), w.ctypes.data + 8, 1, 2, ctypes.byref(good),
                            ctypes.byref(out), cw.ctypes.data, cw.ctypes.data,
                            None) == PKG_ERR_INVALID_ARGUMENT  # unaligned witness


@pytest.mark.parametrize("nc,nw,w1", [(1, 1, 1), (100, 300, 150), (1 << 14, 1 << 13, 1 << 12),
                                      (1 << 14, (1 << 14) + 5, 5), (1 << 20, 1 << 21, 1 << 20),
                                      (1 << 20, 3 << 13, (1 << 13) - 80), (1000, 5000, 5000)])
def test_r1cs_sizing_split_matches_oracle(L, nc, nw, w1):
    from provekit_b200.prover import r1cs_sizing, r1cs_sizing_split
    assert r1cs_sizing_split(nc, nw, w1) == O.r1cs_sizing_split(nc, nw, w1)
    if w1 == nw:
        assert r1cs_sizing_split(nc, nw, w1) == r1cs_sizing(nc, nw)


def test_dual_prove_validation_needs_no_device(L):
    """pkg_dual_prove_begin refuses bad arguments before any device work: a
    w1 without the public inputs or longer than the witness, an offset
    outside 2^m, parameters for another m, a batch of 4, null outputs, an
    unaligned w1; finish refuses a null state; free accepts NULL."""
    from provekit_b200._lib import PKG_ERR_INVALID_ARGUMENT
    from provekit_b200.prover import DualProofC, R1csC, r1cs_sizing_split
    from provekit_b200.whir import WhirParams
    nc, nw, w1 = 1 << 10, 3000, 2000
    m, _ = r1cs_sizing_split(nc, nw, w1)
    r = R1csC(nc, nw)
    r.num_public_inputs = 2
    w = np.zeros(4 * 16, np.uint64)
    wptr = (w.ctypes.data + 15) // 16 * 16
    buf = np.zeros(64, np.uint64)
    good = WhirParams.new(m, 3, 2, 64, 4, batch_size=2)

    def begin(w1_size=w1, offs=(0, 5), p=good, wp=wptr, words=buf.ctypes.data,
              chal=buf.ctypes.data, state=True):
        o = np.array(offs, np.uint64)
        st = ctypes.c_void_p(1)
        rc = L.pkg_dual_prove_begin(ctypes.byref(r), w1_size, o.ctypes.data if len(o) else None,
                                    len(o), wp, 1, 2, None if p is None else ctypes.byref(p),
                                    words, chal, ctypes.byref(st) if state else None, None)
        assert st.value is None or not state  # the state output is reset on entry
        return rc

    assert begin(w1_size=2) == PKG_ERR_INVALID_ARGUMENT          # public inputs outside w1
    assert begin(w1_size=nw + 1) == PKG_ERR_INVALID_ARGUMENT     # w1 longer than the witness
    assert begin(offs=(0, 1 << m)) == PKG_ERR_INVALID_ARGUMENT   # offset outside 2^m
    assert begin(p=WhirParams.new(m + 1, 3, 2, 64, 4)) == PKG_ERR_INVALID_ARGUMENT
    assert begin(p=WhirParams.new(m, 3, 2, 64, 4, batch_size=4)) == PKG_ERR_INVALID_ARGUMENT
    assert begin(p=None) == PKG_ERR_INVALID_ARGUMENT
    assert begin(words=None) == PKG_ERR_INVALID_ARGUMENT
    assert begin(chal=None) == PKG_ERR_INVALID_ARGUMENT
    assert begin(wp=wptr + 8) == PKG_ERR_INVALID_ARGUMENT        # unaligned w1
    assert begin(state=False) == PKG_ERR_INVALID_ARGUMENT
    out = DualProofC()
    assert L.pkg_dual_prove_finish(None, wptr, ctypes.byref(out), buf.ctypes.data,
                                   buf.ctypes.data, buf.ctypes.data) == PKG_ERR_INVALID_ARGUMENT
    L.pkg_dual_prove_free(None)


@pytest.mark.parametrize("seed,log_nc,log_ni,npub", [(1, 0, 0, 0), (3, 6, 4, 2), (7, 12, 10, 0),
                                                     (1003, 16, 14, 5)])
def test_synthetic_r1cs_matches_oracle_generator(L, seed, log_nc, log_ni, npub):
    """pkg_synthetic_r1cs (the library's host-side generator of the prove
    workload) and the oracle's pko_synthetic_r1cs produce the same matrices
    and witness entry for entry, so a CPU arm can build the instance without
    loading the CUDA library; the instance is satisfiable."""
    from provekit_b200.prover import HostR1CS
    nc, ni = 1 << log_nc, 1 << log_ni
    got = HostR1CS(seed, nc, ni, num_public_inputs=npub)
    exp = O.SyntheticR1CS(seed, nc, ni, num_public_inputs=npub)
    assert got.num_witnesses == exp.num_witnesses and got.nnz == exp.nnz
    for k in range(3):
        assert np.array_equal(got.row_ptr[k], exp.row_ptr[k]), k
        assert np.array_equal(got.cols[k], exp.cols[k]), k
        assert np.array_equal(got.vals[k], exp.vals[k]), k
    assert np.array_equal(got.witness, exp.witness)
    # satisfiable: (A w) o (B w) == C w, checked with the oracle's SpMV
    w = np.ascontiguousarray(exp.witness)
    ys = []
    for k in range(3):
        y = np.zeros((nc, 4), np.uint64)
        O.lib().pko_spmv(O.p64(exp.row_ptr[k]), O.p32(exp.cols[k]), O.p64(exp.vals[k]), nc,
                         O.p64(w), O.p64(y))
        ys.append(y)
    for i in range(nc):
        ab = np.zeros(4, np.uint64)
        O.lib().pko_fr_mul(O.p64(ab), O.p64(np.ascontiguousarray(ys[0][i])),
                           O.p64(np.ascontiguousarray(ys[1][i])))
        assert np.array_equal(ab, ys[2][i]), i


@pytest.mark.parametrize("nc1,ni,nchal,rows2", [(1, 1, 0, 0), (64, 20, 3, 77), (100, 30, 0, 50),
                                                (50, 10, 5, 0), (4096, 1024, 16, 5000)])
def test_synthetic_dual_matches_oracle_generator(L, nc1, ni, nchal, rows2):
    """pkg_synthetic_r1cs_dual and pkg_synthetic_dual_solve (the library's
    generator and w2 solve of the two-commitment workload) equal the
    oracle's entry for entry, for the same challenges."""
    from provekit_b200.prover import HostDualR1CS
    got = HostDualR1CS(9, nc1, ni, nchal, rows2)
    exp = O.SyntheticDualR1CS(9, nc1, ni, nchal, rows2)
    assert (got.w1_size, got.num_witnesses, got.nnz) == (exp.w1_size, exp.num_witnesses, exp.nnz)
    assert np.array_equal(got.challenge_offsets, exp.challenge_offsets)
    for k in range(3):
        assert np.array_equal(got.row_ptr[k], exp.row_ptr[k]), k
        assert np.array_equal(got.cols[k], exp.cols[k]), k
        assert np.array_equal(got.vals[k], exp.vals[k]), k
    assert np.array_equal(got.witness, exp.witness)
    ch = O.sample_fr(5, nchal).reshape(-1, 4)
    assert np.array_equal(got.solve(ch), exp.solve(ch))


def prover_bytes(h, folding_factor=3, log_inv_rate=2, security_bits=128, pow_bits=10, zk=1,
                 domain=0) -> bytes:
    """The pkg_prover_serialize layout written independently from the header's
    description (a test of the loader and of the serializer on the GPU)."""
    import struct
    out = [b"PKGPROVR", struct.pack("<II", 1, 0),
           struct.pack("<6Q", h.num_constraints, h.num_witnesses,
                       getattr(h, "num_public_inputs", 0), *h.nnz),
           struct.pack("<6I", folding_factor, log_inv_rate, security_bits, pow_bits, zk, 0),
           struct.pack("<QQ", domain, 0)]
    for k in range(3):
        out.append(np.ascontiguousarray(h.row_ptr[k], np.uint64).tobytes())
        c = np.ascontiguousarray(h.cols[k][: h.nnz[k]], np.uint32).tobytes()
        out.append(c + b"\0" * (-len(c) % 8))
        out.append(np.ascontiguousarray(h.vals[k][: h.nnz[k]], np.uint64).tobytes())
    return b"".join(out)


def test_get_last_error_takes_and_clears(L):
    from provekit_b200.handle import last_error_taken
    assert L.pkg_ntt_nr(None, 6, 4, 1, None) == -1
    msg = last_error_taken()
    assert msg  # the validation message, as UTF-8 bytes in a library-owned buffer
    assert last_error_taken() == ""  # cleared by the first take


P_LIMBS = [0x43e1f593f0000001, 0x2833e84879b97091, 0xb85045b68181585d, 0x30644e72e131a029]


def _bad_variants(h):
    """(description, mutated HostR1CS-like copy) with one malformed matrix each."""
    import copy
    out = []
    for what in ("start", "decrease", "end", "column", "coefficient p", "coefficient max"):
        g = copy.deepcopy(h)
        if what == "start":
            g.row_ptr[1] = g.row_ptr[1].copy()
            g.row_ptr[1][0] = 1
        elif what == "decrease":
            g.row_ptr[0] = g.row_ptr[0].copy()
            g.row_ptr[0][2] = g.row_ptr[0][1] - 1 if g.row_ptr[0][1] else 5
        elif what == "end":
            g.nnz = list(g.nnz)
            g.nnz[2] += 1
        elif what == "column":
            g.cols[0] = g.cols[0].copy()
            g.cols[0][3] = g.num_witnesses
        else:  # a coefficient that is not a canonical field element
            k = 1 if what == "coefficient p" else 2
            g.vals[k] = g.vals[k].copy()
            g.vals[k][-1] = P_LIMBS if what == "coefficient p" else [2**64 - 1] * 4
        out.append((what, g))
    return out


def test_prover_create_rejects_malformed_circuits_before_device_work(L):
    """Row pointers that do not start at 0, decrease or do not end at nnz,
    columns that are not witness indices and coefficients that are not
    canonical field elements (p itself, 2^256 - 1) are rejected on the host:
    the kernels that walk the rows never see them."""
    from provekit_b200._lib import PkgError
    from provekit_b200.handle import Prover
    h = O.SyntheticR1CS(5, 64, 16)
    for what, g in _bad_variants(h):
        with pytest.raises(PkgError) as e:
            Prover.create(g)
        assert e.value.code == -1, what


def test_prover_load_bytes_validates_the_layout(L):
    """Bad magic, an unknown version, truncation anywhere, trailing bytes and
    malformed matrices are rejected before any device work; a well-formed
    string gets as far as the device (which this machine lacks)."""
    import ctypes
    h = O.SyntheticR1CS(6, 64, 16, num_public_inputs=2)
    good = prover_bytes(h)

    def load(b):
        out = ctypes.c_void_p()
        buf = (ctypes.c_uint8 * max(len(b), 1)).from_buffer_copy(b or b"\0")
        return L.pkg_prover_load_bytes(buf, len(b), ctypes.byref(out)), out

    assert load(b"XKGPROVR" + good[8:])[0] == -1
    assert load(good[:8] + b"\2" + good[9:])[0] == -1
    for cut in (4, 20, 60, 104, 300, len(good) - 1):
        rc, out = load(good[:cut])
        assert rc == -1 and not out.value, cut
    assert load(good + b"\0")[0] == -1
    for what, g in _bad_variants(h):
        assert load(prover_bytes(g))[0] == -1, what
    rc, out = load(good)
    if rc == 0:  # a device is present after all
        L.pkg_prover_free(out)
    else:
        assert rc == -2 and not out.value  # CUDA: past every host check


def test_batch_plan_entry_points_reject_null_batch(L):
    """The batch plan setters and getter validate their handle before any
    device work."""
    from provekit_b200._lib import PKG_ERR_INVALID_ARGUMENT
    assert L.pkg_batch_set_params(None, 8, 8) == PKG_ERR_INVALID_ARGUMENT
    assert L.pkg_batch_set_butterflies_per_thread(None, 1) == PKG_ERR_INVALID_ARGUMENT
    k = ctypes.c_int()
    assert L.pkg_batch_get_params(None, ctypes.byref(k), None, None) == PKG_ERR_INVALID_ARGUMENT
