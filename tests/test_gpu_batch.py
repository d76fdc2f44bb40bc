"""Batched form: every job's NTT output, codeword, Merkle layers and
zk-sumcheck transcript from one grouped batch (direct launches, a captured
CUDA graph and its replay, and after autotuning) equal the plain entry points
run one job at a time, bit-exact."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SIZES = [4, 10, 5, 12, 7, 14, 6, 11, 9, 13, 8, 10]


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def plain_job(job):
    """Job j through pkg_ntt_nr, pkg_whir_commit and pkg_spartan_sumcheck."""
    from provekit_b200.batch import Batch
    from provekit_b200.merkle import whir_commit
    from provekit_b200.ntt import ntt_nr
    from provekit_b200.spartan import Transcript, spartan_sumcheck
    n = job.n
    coeffs = torch.from_numpy(Batch.read_fr(job.coeffs, n).view(np.int64)).cuda()
    ntt = coeffs.clone()
    ntt_nr(ntt, n, 1)
    cw, layers = whir_commit(coeffs, 3, 2)
    m0 = job.log_n
    g = np.array(job.g[: 16 * m0], np.uint64).reshape(-1, 4)
    wb = np.array(job.w1_blinding[: 16 * m0], np.uint64).reshape(-1, 4)
    t = Transcript.new(job.transcript_domain)
    sc = spartan_sumcheck(coeffs.clone(), ntt.clone(), cw[:n].clone(), m0, g, wb, t)
    sc["transcript"] = (list(t.l), list(t.r))
    return ntt, cw, layers, sc


def check_batch(b):
    from provekit_b200.batch import Batch
    for j in range(len(b.log_sizes)):
        job = b.job(j)
        ntt, cw, layers, sc = plain_job(job)
        n = job.n
        assert np.array_equal(Batch.read_fr(job.ntt, n), ntt.cpu().numpy().view(np.uint64)), j
        assert np.array_equal(Batch.read_fr(job.codeword, 4 * n), cw.cpu().numpy().view(np.uint64)), j
        assert Batch.read(job.layers, 32 * (2 * job.num_leaves - 1)) == layers.cpu().numpy().tobytes(), j
        got = b.sumcheck_result(j)
        for k in ("r", "coeffs", "alpha", "rho", "sum_g", "blinding_eval"):
            assert np.array_equal(got[k], sc[k]), (j, k)
        assert got["transcript"] == sc["transcript"], j


def test_batch_direct_matches_plain():
    from provekit_b200.batch import Batch
    b = Batch(SIZES, seed=11)
    b.run(use_graph=False)
    torch.cuda.synchronize()
    check_batch(b)
    b.close()


def test_batch_graph_replay_and_params():
    from provekit_b200.batch import Batch
    b = Batch(SIZES, seed=12)
    s = torch.cuda.Stream()
    b.run(use_graph=True, stream=s)   # capture + launch
    b.run(use_graph=True, stream=s)   # replay
    s.synchronize()
    check_batch(b)
    b.set_params(4, 8)                # radix 2^4, 256 elements per CTA
    b.run(use_graph=False, stream=s)
    s.synchronize()
    check_batch(b)
    b.set_params(11, 11)              # radix 2^11 (64 KiB shared memory)
    b.run(use_graph=True, stream=s)
    s.synchronize()
    check_batch(b)
    for lb in (1, 2):                 # 2 and 4 butterflies per thread per stage
        b.set_params(8, 10, log_bpt=lb)
        assert b.params() == (8, 10, lb)
        b.run(use_graph=False, stream=s)
        s.synchronize()
        check_batch(b)
    b.close()


def test_batch_autotune_keeps_results():
    from provekit_b200.batch import Batch
    b = Batch([10, 12, 9, 11], seed=13)
    k, e, ms = b.tune()
    assert 4 <= k <= 11 and k <= e <= 11 and ms > 0
    kk, ee, lb = b.params()
    assert (kk, ee) == (k, e) and 0 <= lb <= 2
    b.run(use_graph=False)
    torch.cuda.synchronize()
    check_batch(b)
    b.close()


def test_batch_rejects_bad_sizes():
    from provekit_b200 import PkgError
    from provekit_b200.batch import Batch
    with pytest.raises(PkgError):
        Batch([3], seed=1)
    with pytest.raises(PkgError):
        Batch([25], seed=1)
