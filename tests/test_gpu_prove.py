"""GPU parity of the Spartan prove core (pkg_spartan_prove) against the
oracle's pko_spartan_prove on synthetic satisfiable R1CS instances, up to the
2^20-constraint prove workload: root, every sumcheck message and challenge,
covector evaluations and the final transcript state must be identical.  The
whole proof (pkg_prove_r1cs, with the WHIR rounds) must equal the oracle's
word for word and its WHIR part verify."""
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


@pytest.mark.parametrize("log_nc,log_ni,ff", [(1, 1, 3), (10, 8, 3), (12, 10, 4), (16, 14, 3), (20, 18, 3)])
def test_spartan_prove_matches_oracle(log_nc, log_ni, ff):
    from provekit_b200.prover import HostR1CS, spartan_prove
    h = HostR1CS(100 + log_nc, 1 << log_nc, 1 << log_ni)
    exp = O.spartan_prove(h, 5, 9, ff, 2)
    got = spartan_prove(h.to_device(), blinding_seed=5, transcript_domain=9, folding_factor=ff,
                        log_inv_rate=2)
    assert_same(got, exp)


def test_stage_timers_and_memory_trim_keep_results():
    """pkg_last_prove_stages reports the calling thread's last prove; returning
    the library pool's memory (pkg_trim_memory) between proves changes no
    output."""
    import ctypes
    from provekit_b200._lib import check, lib
    from provekit_b200.prover import HostR1CS, spartan_prove
    h = HostR1CS(77, 1 << 14, 1 << 12)
    d = h.to_device()
    first = spartan_prove(d, blinding_seed=3, transcript_domain=4)
    stages = (ctypes.c_double * 6)()
    check(lib().pkg_last_prove_stages(stages))
    assert all(v > 0 for v in stages[:5]) and stages[5] == 0, list(stages)
    check(lib().pkg_trim_memory(0))
    again = spartan_prove(d, blinding_seed=3, transcript_domain=4)
    assert_same(again, first)


@pytest.mark.parametrize("log_nc,log_ni,sec,pw,zk,npub", [(10, 8, 40, 3, False, 0),
                                                         (12, 11, 64, 5, False, 0),
                                                         (14, 12, 128, 10, False, 0),
                                                         (10, 8, 40, 3, True, 0),
                                                         (13, 11, 64, 5, True, 0),
                                                         (11, 9, 40, 3, False, 1),
                                                         (12, 10, 64, 4, True, 2),
                                                         (12, 10, 40, 3, True, 300)])
def test_whole_proof_matches_oracle_and_verifies(log_nc, log_ni, sec, pw, zk, npub):
    import ctypes
    from provekit_b200._lib import check, lib
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(300 + log_nc, 1 << log_nc, 1 << log_ni, num_public_inputs=npub)
    d = h.to_device()
    p = whir_params_for(d, 3, 2, sec, pw, zk=zk)
    sp, cw, proof = prove_r1cs(d, p, blinding_seed=6, transcript_domain=12)
    stages = (ctypes.c_double * 6)()
    check(lib().pkg_last_prove_stages(stages))
    assert all(v > 0 for v in stages), list(stages)
    wp = O.whir_params(sp["m"], 3, 2, sec, pw, batch_size=2 if zk else 1)
    assert bytes(wp) == bytes(p)
    esp, ecw, eproof = O.prove_r1cs(h, 6, 12, wp)
    assert_same(sp, esp)
    assert np.array_equal(cw, ecw)
    assert np.array_equal(proof, eproof)
    assert O.verify_r1cs_whir(h, wp, 12, sp, cw, proof) == 0


def test_whole_proof_at_2p20_constraints_matches_oracle():
    """The headline bench instance itself -- the synthetic R1CS of seed 2
    with 2^20 constraints and 2^18 inputs (m = 21, m0 = 20), whir-ZK (batch
    of 2), ff 3, rate 1/4, 128 bits, 10 PoW bits, blinding seed 1, domain 3:
    the device proof equals the oracle's in every Spartan field, every
    commitment word and every WHIR proof word, and the oracle verifier
    accepts it."""
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(2, 1 << 20, 1 << 18)
    d = h.to_device()
    p = whir_params_for(d)
    assert (p.num_variables, p.folding_factor, p.log_inv_rate, p.pow_bits, p.batch_size) == \
        (21, 3, 2, 10, 2)
    sp, cw, proof = prove_r1cs(d, p, blinding_seed=1, transcript_domain=3)
    del d
    torch.cuda.empty_cache()
    wp = O.whir_params(21, 3, 2, 128, 10, batch_size=2)
    assert bytes(wp) == bytes(p)
    esp, ecw, eproof = O.prove_r1cs(h, 1, 3, wp)
    assert_same(sp, esp)
    assert np.array_equal(cw, ecw)
    assert proof.shape == eproof.shape
    if not np.array_equal(proof, eproof):
        first = int(np.nonzero(proof != eproof)[0][0])
        pytest.fail(f"proofs differ first at word {first} of {proof.shape[0]}")
    assert O.verify_r1cs_whir(h, wp, 3, sp, cw, proof) == 0


def test_concurrent_whole_proofs_equal_sequential():
    """Four host threads with their own streams prove the same resident
    circuit at once (the batched bench's pattern); each proof equals the
    same call made alone."""
    import threading
    from provekit_b200._lib import check, lib
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(41, 1 << 13, 1 << 11)
    d = h.to_device()
    p = whir_params_for(d, 3, 2, 64, 4)
    alone = [prove_r1cs(d, p, blinding_seed=10 + i, transcript_domain=20 + i) for i in range(8)]
    check(lib().pkg_reserve_memory(1 << 30))
    streams = [torch.cuda.Stream() for _ in range(4)]
    got = [None] * 8

    def worker(j):
        for i in range(j, 8, 4):
            got[i] = prove_r1cs(d, p, blinding_seed=10 + i, transcript_domain=20 + i,
                                stream=streams[j])

    th = [threading.Thread(target=worker, args=(j,)) for j in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for (sp, cw, pr), (esp, ecw, epr) in zip(got, alone):
        assert_same(sp, esp)
        assert np.array_equal(cw, ecw) and np.array_equal(pr, epr)


@pytest.mark.parametrize("seed,start,n", [(1, 0, 1), (5, 0, 1000), (0xfeedface12345678, 1 << 33, 4097)])
def test_indexed_sampler_matches_oracle(seed, start, n):
    """pkg_sample_fr_indexed (the whir-ZK blinding polynomial's source)."""
    from provekit_b200._lib import check, lib
    d = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    check(lib().pkg_sample_fr_indexed(seed, start, n, d.data_ptr(), None))
    torch.cuda.synchronize()
    exp = np.zeros((n, 4), np.uint64)
    O.lib().pko_sample_fr_indexed(seed, start, n, O.p64(exp))
    assert np.array_equal(d.cpu().numpy().view(np.uint64), exp)
