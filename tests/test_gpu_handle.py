"""Prover handles (pkg_prover_*): the reference FFI's PKProver / PKBuf
conventions (tooling/provekit-ffi/src/ffi.rs) over the device prover.

A handle made from a host R1CS proves a solved witness into a library-owned
buffer whose bytes decode to exactly the proof of pkg_prove_r1cs and of the
oracle for the same instance and seeds; its serialized form is the layout
the header documents, and a handle loaded from it proves the same bytes."""
import threading

import numpy as np
import pytest
import torch

import oracle_lib as O
from test_capi_host import prover_bytes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def same(a, b):
    for k in b:
        if isinstance(b[k], np.ndarray):
            assert np.array_equal(np.asarray(a[k]), b[k]), k
        else:
            assert a[k] == b[k], k


@pytest.mark.parametrize("log_nc,log_ni,npub,zk", [(10, 8, 0, 1), (12, 10, 3, 1), (11, 9, 0, 0)])
def test_handle_proof_equals_the_oracle(log_nc, log_ni, npub, zk):
    from provekit_b200.handle import Prover, config, parse_proof
    from provekit_b200.prover import HostR1CS
    h = HostR1CS(600 + log_nc, 1 << log_nc, 1 << log_ni, num_public_inputs=npub)
    cfg = config(transcript_domain=17, security_bits=64, pow_bits=4, zk=zk)
    pv = Prover.create(h, cfg)
    info = pv.info()
    data = pv.prove(h.witness, blinding_seed=9)
    assert len(data) == info.proof_bytes
    got = parse_proof(data)
    assert bytes(got["whir"]) == bytes(info.whir)
    wp = O.whir_params(info.m, 3, 2, 64, 4, batch_size=2 if zk else 1)
    assert bytes(wp) == bytes(got["whir"])
    esp, ecw, eproof = O.prove_r1cs(h, 9, 17, wp)
    same(got["spartan"], esp)
    assert np.array_equal(got["commit_words"], ecw)
    assert np.array_equal(got["proof"], eproof)
    assert O.verify_r1cs_whir(h, wp, 17, got["spartan"], got["commit_words"], got["proof"]) == 0
    # the same handle again, another seed: a fresh proof, the first unchanged
    again = pv.prove(h.witness, blinding_seed=9)
    assert again == data
    assert pv.prove(h.witness, blinding_seed=10) != data
    pv.close()


def test_serialize_load_and_prove_again():
    from provekit_b200.handle import Prover, config
    from provekit_b200.prover import HostR1CS
    h = HostR1CS(611, 1 << 12, 1 << 10, num_public_inputs=2)
    cfg = config(transcript_domain=4, security_bits=40, pow_bits=3)
    pv = Prover.create(h, cfg)
    ser = pv.serialize()
    assert ser == prover_bytes(h, security_bits=40, pow_bits=3, domain=4)
    pv2 = Prover.load_bytes(ser)
    assert pv2.serialize() == ser
    assert pv2.prove(h.witness, 3) == pv.prove(h.witness, 3)
    pv.close()
    pv2.close()


def test_handle_matches_resident_prove_at_2p16_constraints():
    """The handle (witness from host memory through the stager, cached
    transposes) and pkg_prove_r1cs on a resident circuit give the same proof."""
    from provekit_b200.handle import Prover, config, parse_proof
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(612, 1 << 16, 1 << 14)
    pv = Prover.create(h, config(transcript_domain=3))
    got = parse_proof(pv.prove(h.witness, 1))
    d = h.to_device(transposes=False)
    sp, cw, proof = prove_r1cs(d, whir_params_for(d), blinding_seed=1, transcript_domain=3)
    same(got["spartan"], sp)
    assert np.array_equal(got["commit_words"], cw) and np.array_equal(got["proof"], proof)
    pv.close()


def test_two_handles_prove_concurrently():
    from provekit_b200.handle import Prover, config
    from provekit_b200.prover import HostR1CS
    hs = [HostR1CS(620 + i, 1 << 11, 1 << 9) for i in range(2)]
    pvs = [Prover.create(h, config(transcript_domain=i, security_bits=40, pow_bits=3))
           for i, h in enumerate(hs)]
    alone = [[pv.prove(h.witness, s) for s in range(4)] for pv, h in zip(pvs, hs)]
    got = [[None] * 4 for _ in range(2)]

    def worker(j):
        torch.cuda.set_device(0)
        for s in range(4):
            got[j][s] = pvs[j].prove(hs[j].witness, s)

    th = [threading.Thread(target=worker, args=(j,)) for j in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert got == alone
    for pv in pvs:
        pv.close()


def test_cached_transposes_give_the_same_proof():
    """DeviceR1CS with the transposes built once, and without (every proof
    transposes): identical proofs, equal to the oracle's."""
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(630, 1 << 13, 1 << 11, num_public_inputs=1)
    a = h.to_device(transposes=True)
    b = h.to_device(transposes=False)
    assert a.c.row_ptr_t[0] and not b.c.row_ptr_t[0]
    p = whir_params_for(a, 3, 2, 64, 5)
    ra = prove_r1cs(a, p, blinding_seed=2, transcript_domain=8)
    rb = prove_r1cs(b, p, blinding_seed=2, transcript_domain=8)
    same(ra[0], rb[0])
    assert np.array_equal(ra[1], rb[1]) and np.array_equal(ra[2], rb[2])
    wp = O.whir_params(ra[0]["m"], 3, 2, 64, 5, batch_size=2)
    esp, ecw, eproof = O.prove_r1cs(h, 2, 8, wp)
    same(ra[0], esp)
    assert np.array_equal(ra[2], eproof)
