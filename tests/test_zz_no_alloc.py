"""pkg_intt_rn_noalloc: the inverse NTT for callers that cannot let the
library allocate device memory (a service that reserves all HBM for its own
admission control, or an application whose framework allocator owns the free
memory).  Its scratch is a fixed __device__ array inside the library, so it
must give exactly what pkg_intt_rn gives -- the field arithmetic is exact, so
the tolerance is zero -- on consecutive calls that reuse that array.

Kept in a file that sorts last so a failure here cannot hide other results;
it passes both on its own in a fresh process and after the other tests."""
import numpy as np
import pytest
import torch

import oracle_lib as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()
    from provekit_b200 import _lib
    return _lib.lib()


def _run(L, fn, values: np.ndarray) -> np.ndarray:
    d = torch.from_numpy(values.view(np.int64).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(d.data_ptr(), values.shape[0], stream)
    assert rc == 0, L.pkg_last_error()
    torch.cuda.synchronize()
    return d.cpu().numpy().view(np.uint64)


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(L):
    # Two calls in a row share (and overwrite) the fixed scratch array: a
    # larger size first, then a smaller one whose twiddles and gather buffer
    # reuse the same words.
    for seed, logn in [(71, 16), (72, 10), (73, 16)]:
        x = O.sample_fr(seed, 1 << logn)
        want = _run(L, L.pkg_intt_rn, x)
        got = _run(L, L.pkg_intt_rn_noalloc, x)
        assert np.array_equal(got, want), f"mismatch at 2^{logn}"


@pytest.mark.parametrize("logn", [0, 1, 2, 5, 9, 10, 16])
def test_noalloc_small_and_edge_lengths(L, logn):
    # Below 2^10 the allocating path uses a padded order-1024 twiddle table
    # while this one builds a table of exactly len/2 entries (len 2: one
    # entry, a kernel with log_half = 0); len 1 is the identity.  Compared
    # with pkg_intt_rn and, independently, with the oracle's intt_rn.
    x = O.sample_fr(800 + logn, 1 << logn)
    want = _run(L, L.pkg_intt_rn, x)
    got = _run(L, L.pkg_intt_rn_noalloc, x)
    assert np.array_equal(got, want), f"mismatch at 2^{logn}"
    exp = x.copy()
    assert O.intt_rn(exp) == 0
    assert np.array_equal(got.reshape(-1, 4), exp)


def test_noalloc_on_a_non_default_stream(L):
    x = O.sample_fr(901, 1 << 12)
    want = _run(L, L.pkg_intt_rn, x)
    s = torch.cuda.Stream()
    d = torch.from_numpy(x.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    for _ in range(2):  # the second call must not see the first one's scratch
        d.copy_(torch.from_numpy(x.view(np.int64).copy()))
        torch.cuda.synchronize()
        assert L.pkg_intt_rn_noalloc(d.data_ptr(), x.shape[0], s.cuda_stream) == 0
        s.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint64), want)


def test_noalloc_rejects_lengths_beyond_its_scratch(L):
    d = torch.zeros((1 << 17, 4), dtype=torch.int64, device="cuda")
    rc = L.pkg_intt_rn_noalloc(d.data_ptr(), 1 << 17, None)
    assert rc == -1
    assert b"exceeds the fixed scratch maximum" in L.pkg_last_error()
