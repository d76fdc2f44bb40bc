"""GPU tests of the host-slice entry points at sizes that cross the staging
chunks (8 MiB): pinned, pipelined copies must deliver exactly the bytes the
device-resident entry points see.  Each host form is compared bit for bit
with the device form (itself checked against the oracle elsewhere) on the
same inputs, including message lists whose boundaries fall inside a chunk,
sizes that are not a multiple of the chunk, workspace growth and shrink,
and back-to-back calls."""
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


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).copy()).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("logn", [19, 21, 12])
def test_host_ntt_matches_device(logn):
    from provekit_b200.ntt import host_intt_rn, host_ntt_nr, ntt_nr
    n = 1 << logn
    a = O.sample_fr(70 + logn, n)
    d = dev(a)
    ntt_nr(d, n, 1)
    got = host_ntt_nr(a.copy(), n, 1)
    assert np.array_equal(got, host(d).reshape(-1, 4))
    assert np.array_equal(host_intt_rn(got), a)


def test_host_rs_encode_message_list_crossing_chunks():
    from provekit_b200.rs import RSFr
    M, L, cw = 3, 1 << 17, 1 << 19          # 4 MiB per message, 48 MiB out
    msgs = [O.sample_fr(80 + j, L) for j in range(M)]
    masks = O.sample_fr(89, 5)
    exp = RSFr().interleaved_encode(dev(np.stack(msgs)), dev(masks), cw)
    got = RSFr().host_interleaved_encode(msgs, masks, cw)
    assert np.array_equal(got, host(exp).reshape(-1, 4))


@pytest.mark.parametrize("size,count", [(512, 1 << 16), (96, 100_003), (64, 5), (32 * 16, 1 << 14)])
def test_host_hash_many_matches_device(size, count):
    from provekit_b200.skyscraper import SkyscraperHashEngine
    rng = np.random.default_rng(size + count)
    data = rng.integers(0, 256, size=size * count, dtype=np.uint8)
    eng = SkyscraperHashEngine()
    exp = eng.hash_many(size, torch.from_numpy(data.copy()).cuda()).cpu().numpy().tobytes()
    assert eng.host_hash_many(size, data.tobytes()) == exp
    assert eng.host_hash_many(size, data.tobytes()) == exp  # back to back, same workspace


def test_host_commit_through_the_trait_calls():
    """The plugin-shaped commit (RS encode, leaf hashing, one call per tree
    level) equals the resident pkg_whir_commit root."""
    from provekit_b200.merkle import whir_commit
    from provekit_b200.rs import RSFr
    from provekit_b200.skyscraper import SkyscraperHashEngine
    from provekit_b200._lib import PKG_LEAF_MONTGOMERY
    n, ff, lr = 1 << 18, 3, 2
    M = 1 << ff
    L = n // M
    coeffs = O.sample_fr(91, n)
    cw = L << lr
    msgs = [coeffs[j * L:(j + 1) * L] for j in range(M)]
    code = RSFr().host_interleaved_encode(msgs, None, cw)
    eng = SkyscraperHashEngine()
    level = eng.host_hash_many(32 * M, code.tobytes())
    while len(level) > 32:
        level = eng.host_hash_many(64, level)
    _, layers = whir_commit(dev(coeffs), ff, lr, leaf_encoding=PKG_LEAF_MONTGOMERY)
    assert level == layers[-32:].cpu().numpy().tobytes()


def test_concurrent_host_calls_match_sequential():
    """Host-slice calls from several threads at once (the stager serialises
    them per device and shares its pinned chunks) return exactly what the
    same calls return one at a time."""
    import threading
    from provekit_b200.ntt import host_ntt_nr
    from provekit_b200.skyscraper import SkyscraperHashEngine
    eng = SkyscraperHashEngine()
    rng = np.random.default_rng(42)
    blobs = [rng.integers(0, 256, size=512 * (1 << 14), dtype=np.uint8).tobytes() for _ in range(4)]
    polys = [O.sample_fr(500 + i, 1 << 18) for i in range(4)]
    exp_h = [eng.host_hash_many(512, b) for b in blobs]
    exp_n = [host_ntt_nr(p.copy(), 1 << 18, 1) for p in polys]
    got_h, got_n, errors = [None] * 4, [None] * 4, []

    def work(i):
        try:
            for _ in range(3):
                got_h[i] = eng.host_hash_many(512, blobs[i])
                got_n[i] = host_ntt_nr(polys[i].copy(), 1 << 18, 1)
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    assert got_h == exp_h
    assert all(np.array_equal(g, e) for g, e in zip(got_n, exp_n))
