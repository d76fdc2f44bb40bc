"""Served form: requests of different sizes submitted together to a server
whose HBM budget and slots force queueing and overlap; every proof equals the
same request proved alone with pkg_spartan_prove."""
import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def same(a, b):
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], k


def test_served_results_equal_alone_results():
    from provekit_b200.prover import HostR1CS, spartan_prove
    from provekit_b200.server import ProofServer
    sizes = [(12, 10), (10, 8), (14, 12), (11, 9), (13, 11), (10, 8), (14, 12), (12, 10)]
    reqs = [HostR1CS(500 + i, 1 << lc, 1 << li) for i, (lc, li) in enumerate(sizes)]
    alone = [spartan_prove(h.to_device(), blinding_seed=7 + i, transcript_domain=100 + i)
             for i, h in enumerate(reqs)]
    # budget: room for about two of the largest requests at once
    srv = ProofServer(hbm_budget_bytes=2 * 96 << 20, max_inflight=3)
    ids = [srv.submit(h, blinding_seed=7 + i, transcript_domain=100 + i) for i, h in enumerate(reqs)]
    results = [srv.wait(rid) for rid in ids]
    for (proof, times), ref in zip(results, alone):
        same(proof, ref)
        assert times["submit_ns"] <= times["admit_ns"] <= times["done_ns"]
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["p50_ms"] > 0
    assert st["peak_reserved_bytes"] <= 2 * 96 << 20
    srv.close()


def test_submit_from_threads_and_overlap():
    """Requests submitted from several host threads while others run."""
    from provekit_b200.prover import HostR1CS, spartan_prove
    from provekit_b200.server import ProofServer
    reqs = [HostR1CS(900 + i, 1 << 12, 1 << 10) for i in range(6)]
    srv = ProofServer(hbm_budget_bytes=1 << 30, max_inflight=4)
    out = {}

    def client(i):
        rid = srv.submit(reqs[i], blinding_seed=i, transcript_domain=i)
        out[i] = srv.wait(rid)[0]

    th = [threading.Thread(target=client, args=(i,)) for i in range(len(reqs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, h in enumerate(reqs):
        same(out[i], spartan_prove(h.to_device(), blinding_seed=i, transcript_domain=i))
    srv.close()


def test_request_above_budget_is_rejected():
    from provekit_b200 import PkgError
    from provekit_b200.prover import HostR1CS
    from provekit_b200.server import ProofServer
    srv = ProofServer(hbm_budget_bytes=64 << 20, max_inflight=1)
    with pytest.raises(PkgError):
        srv.submit(HostR1CS(1, 1 << 16, 1 << 14))
    srv.close()


def test_served_whole_proofs_equal_alone_results():
    """Whole proofs (pkg_prove_r1cs) through the server: Spartan part, WHIR
    commitment words and WHIR proof equal the same request proved alone."""
    from provekit_b200.prover import HostR1CS, prove_r1cs
    from provekit_b200.server import ProofServer
    sizes = [(12, 10), (14, 12), (13, 11), (15, 13), (12, 10)]
    reqs = [HostR1CS(700 + i, 1 << lc, 1 << li) for i, (lc, li) in enumerate(sizes)]
    alone = [prove_r1cs(h.to_device(), blinding_seed=3 + i, transcript_domain=40 + i)
             for i, h in enumerate(reqs)]
    srv = ProofServer(hbm_budget_bytes=1 << 30, max_inflight=3)
    ids = [srv.submit(h, whole_proof=True, blinding_seed=3 + i, transcript_domain=40 + i)
           for i, h in enumerate(reqs)]
    for rid, (sp, cw, proof) in zip(ids, alone):
        got, times = srv.wait(rid)
        assert np.array_equal(got.pop("whir_commit_words"), cw)
        assert np.array_equal(got.pop("whir_proof"), proof)
        same(got, sp)
        assert times["submit_ns"] <= times["admit_ns"] <= times["done_ns"]
    srv.close()


def test_served_mix_of_public_inputs_and_zk_equals_alone_results():
    """A mix of whole proofs with 0, 1 and 3 public inputs, committed with
    a blinding polynomial (whir-ZK) or alone, served together: each equals
    the same request proved alone."""
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    from provekit_b200.server import ProofServer
    spec = [(12, 10, 0, True), (13, 11, 1, False), (12, 10, 3, True), (14, 12, 1, True),
            (11, 9, 3, False), (13, 11, 0, False)]
    reqs = [HostR1CS(800 + i, 1 << lc, 1 << li, num_public_inputs=npub)
            for i, (lc, li, npub, _) in enumerate(spec)]
    params = [whir_params_for(h, zk=zk) for h, (_, _, _, zk) in zip(reqs, spec)]
    alone = [prove_r1cs(h.to_device(), whir=p, blinding_seed=5 + i, transcript_domain=60 + i)
             for i, (h, p) in enumerate(zip(reqs, params))]
    srv = ProofServer(hbm_budget_bytes=1 << 30, max_inflight=3)
    ids = [srv.submit(h, whir=p, blinding_seed=5 + i, transcript_domain=60 + i)
           for i, (h, p) in enumerate(zip(reqs, params))]
    for rid, (sp, cw, proof) in zip(ids, alone):
        got, _ = srv.wait(rid)
        assert np.array_equal(got.pop("whir_commit_words"), cw)
        assert np.array_equal(got.pop("whir_proof"), proof)
        same(got, sp)
    srv.close()


def test_served_large_whole_proofs_equal_alone_results():
    """Requests of 2^18 and 2^20 constraints (the latter the headline's size)
    with a small one, served two at a time under a budget that admits both
    large ones together: whole whir-ZK proofs equal to the same requests
    proved alone."""
    from provekit_b200.prover import HostR1CS, prove_r1cs
    from provekit_b200.server import ProofServer
    sizes = [(20, 18), (18, 16), (14, 12), (18, 17)]
    reqs = [HostR1CS(900 + i, 1 << lc, 1 << li) for i, (lc, li) in enumerate(sizes)]
    alone = [prove_r1cs(h.to_device(), blinding_seed=7 + i, transcript_domain=70 + i)
             for i, h in enumerate(reqs)]
    srv = ProofServer(hbm_budget_bytes=24 << 30, max_inflight=2)
    ids = [srv.submit(h, whole_proof=True, blinding_seed=7 + i, transcript_domain=70 + i)
           for i, h in enumerate(reqs)]
    for rid, (sp, cw, proof) in zip(ids, alone):
        got, _ = srv.wait(rid)
        assert np.array_equal(got.pop("whir_commit_words"), cw)
        assert np.array_equal(got.pop("whir_proof"), proof)
        same(got, sp)
    srv.close()


def test_malformed_request_is_rejected_at_submit():
    """Row pointers that decrease or do not end at nnz are refused by
    pkg_server_submit before the request is queued (device walks over a
    row's entries are bounded by them); a well-formed request on the same
    server still proves."""
    import copy

    from provekit_b200._lib import PKG_ERR_INVALID_ARGUMENT, PkgError
    from provekit_b200.prover import HostR1CS, spartan_prove
    from provekit_b200.server import ProofServer
    h = HostR1CS(950, 1 << 10, 1 << 8)
    srv = ProofServer(hbm_budget_bytes=1 << 30, max_inflight=1)
    dec = copy.deepcopy(h)
    dec.row_ptr[1] = dec.row_ptr[1].copy()
    dec.row_ptr[1][3] = dec.row_ptr[1][4] + 1  # row 3 starts after row 4 does
    end = copy.deepcopy(h)
    end.row_ptr[2] = end.row_ptr[2].copy()
    end.row_ptr[2][-1] += 1  # past nnz
    for bad in (dec, end):
        with pytest.raises(PkgError) as e:
            srv.submit(bad, blinding_seed=2, transcript_domain=5)
        assert e.value.code == PKG_ERR_INVALID_ARGUMENT
    got, _ = srv.wait(srv.submit(h, blinding_seed=2, transcript_domain=5))
    same(got, spartan_prove(h.to_device(), blinding_seed=2, transcript_domain=5))
    srv.close()
