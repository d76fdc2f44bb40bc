"""GPU Poseidon2 against the reference KATs and the oracle, bit-exact."""
import json
import os

import numpy as np
import pytest
import torch

import oracle_lib as O
from fieldutil import pack, unpack

pytestmark = pytest.mark.gpu
KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).copy()).cuda()


def test_permutation_kat_and_batch():
    from provekit_b200.poseidon2 import poseidon2_permutation_many
    n = 4097
    st = O.sample_fr(77, 4 * n)
    st[:4] = 0  # the reference's smoke_test input
    d = dev(st)
    poseidon2_permutation_many(d)
    got = d.cpu().numpy().view(np.uint64)
    assert unpack(got[:4]) == [int(x) for x in KATS["poseidon2"]["permutation_zero"]["expected"]]
    for i in range(0, n, 409):
        e = np.ascontiguousarray(st[4 * i: 4 * i + 4])
        O.lib().pko_poseidon2_permutation(O.p64(e))
        assert np.array_equal(got[4 * i: 4 * i + 4], e)


@pytest.mark.parametrize("length", [1, 2, 3, 4, 7])
def test_hash_many(length):
    from provekit_b200.poseidon2 import poseidon2_hash_many
    n = 1000
    x = O.sample_fr(length, n * length)
    got = poseidon2_hash_many(dev(x), length).cpu().numpy().view(np.uint64)
    for i in range(0, n, 97):
        e = np.zeros(4, np.uint64)
        O.lib().pko_poseidon2_hash(O.p64(e), O.p64(np.ascontiguousarray(x[i * length:(i + 1) * length])), length)
        assert np.array_equal(got[i], e)


@pytest.mark.parametrize("name", ["hash_single", "hash_two"])
def test_hash_kats(name):
    from provekit_b200.poseidon2 import poseidon2_hash_many
    k = KATS["poseidon2"][name]
    inp = pack([int(v) for v in k["input"]])
    got = poseidon2_hash_many(dev(inp), inp.shape[0]).cpu().numpy().view(np.uint64)
    assert unpack(got)[0] == int(k["expected"])
