"""GPU parity of the Spartan prove core (pkg_spartan_prove) against the
oracle's pko_spartan_prove on synthetic satisfiable R1CS instances, up to the
2^20-constraint prove workload: root, every sumcheck message and challenge,
covector evaluations and the final transcript state must be identical."""
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
    stages = (ctypes.c_double * 5)()
    check(lib().pkg_last_prove_stages(stages))
    assert all(v > 0 for v in stages), list(stages)
    check(lib().pkg_trim_memory(0))
    again = spartan_prove(d, blinding_seed=3, transcript_domain=4)
    assert_same(again, first)
