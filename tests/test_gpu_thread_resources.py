"""Per-thread resources are released when their thread ends.

A host thread that proves keeps a mapped pinned buffer for reduction results,
a pinned bounce buffer for small reads, and per device a small device block
and a pinned staging buffer for STIR openings.  These belong to the thread:
a proving server's worker threads (joined when the server is destroyed) and
short-lived caller threads must not leave them behind.  The library's live
totals (pkg_thread_resource_bytes) and the device's free memory must come
back to where they started after many such threads."""
import ctypes
import threading

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def settled(base, timeout_s=10.0):
    """Python's Thread.join() returns when the thread's interpreter state is
    gone, a moment before the OS thread runs its C++ thread_local
    destructors: wait (bounded) for the totals to come back."""
    import time
    t_end = time.monotonic() + timeout_s
    while totals() != base and time.monotonic() < t_end:
        time.sleep(0.01)
    return totals()


def totals():
    from provekit_b200._lib import check, lib
    h, d = ctypes.c_size_t(0), ctypes.c_size_t(0)
    check(lib().pkg_thread_resource_bytes(ctypes.byref(h), ctypes.byref(d)))
    return h.value, d.value


def test_server_create_destroy_cycles_release_worker_resources():
    from provekit_b200._lib import check, lib
    from provekit_b200.prover import HostR1CS
    from provekit_b200.server import ProofServer
    h = HostR1CS(71, 1 << 10, 1 << 8)
    # one cycle first: the pool, twiddles and stager reach their sizes
    srv = ProofServer(hbm_budget_bytes=256 << 20, max_inflight=4)
    srv.wait(srv.submit(h, whole_proof=True, blinding_seed=1, transcript_domain=1))
    srv.close()
    torch.cuda.synchronize()
    check(lib().pkg_trim_memory(0))
    base = totals()
    free0, _ = torch.cuda.mem_get_info()
    for i in range(50):
        srv = ProofServer(hbm_budget_bytes=256 << 20, max_inflight=4)
        ids = [srv.submit(h, whole_proof=True, blinding_seed=i, transcript_domain=j)
               for j in range(4)]
        for rid in ids:
            srv.wait(rid)
        assert totals()[0] > base[0]  # the workers hold their buffers while alive
        srv.close()
    check(lib().pkg_trim_memory(0))
    assert totals() == base
    free1, _ = torch.cuda.mem_get_info()
    # 50 cycles x 4 workers leaking one device block each would be ~12 MB
    assert free1 >= free0 - (4 << 20), (free0, free1)


def test_short_lived_proving_threads_release_their_resources():
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(72, 1 << 10, 1 << 8)
    d = h.to_device()
    p = whir_params_for(d, 3, 2, 40, 3)
    first = prove_r1cs(d, p, blinding_seed=2, transcript_domain=5)
    torch.cuda.synchronize()
    base = totals()
    seen = []

    def worker(i):
        torch.cuda.set_device(0)
        sp, cw, pr = prove_r1cs(d, p, blinding_seed=2, transcript_domain=5)
        seen.append(totals()[0] > base[0])
        assert (cw == first[1]).all() and (pr == first[2]).all()

    for batch in range(10):
        th = [threading.Thread(target=worker, args=(j,)) for j in range(8)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    assert len(seen) == 80 and all(seen)
    assert settled(base) == base


def test_explicit_release_then_reuse():
    """pkg_release_thread_resources frees the calling thread's buffers; the
    next call re-creates them and gives the same proof."""
    from provekit_b200._lib import check, lib
    from provekit_b200.prover import HostR1CS, prove_r1cs, whir_params_for
    h = HostR1CS(73, 1 << 11, 1 << 9)
    d = h.to_device()
    p = whir_params_for(d, 3, 2, 40, 3)
    a = prove_r1cs(d, p, blinding_seed=4, transcript_domain=6)
    torch.cuda.synchronize()
    before = totals()
    check(lib().pkg_release_thread_resources())
    after = totals()
    assert after[0] < before[0] and after[1] < before[1]
    b = prove_r1cs(d, p, blinding_seed=4, transcript_domain=6)
    assert (a[1] == b[1]).all() and (a[2] == b[2]).all()
    # re-created for this proof: the device block at its fixed size; the
    # staging buffer at this proof's size (earlier, larger proofs of this
    # thread had grown it)
    again = totals()
    assert again[1] == before[1] and after[0] < again[0] <= before[0]
