"""GPU parity of the field arithmetic itself: the FP64-pipe Montgomery
product, square and Montgomery->canonical conversion (the routines inside
the NTT and Skyscraper kernels) and the integer-pipe ones, through the C ABI
(pkg_fr_mul_batch), against Python big-int a*b*2^-256 mod p.  Bit-exact:
exact modular arithmetic admits no tolerance.  Edge values cover the digit
and carry extremes: 0, 1, p-1, [p, 2p) where the contract allows it, and
all-ones words."""
import random

import numpy as np
import pytest
import torch

from fieldutil import P, from_limbs, to_limbs

pytestmark = pytest.mark.gpu

RINV = pow(2, -256, P)
TOP = (1 << 256) - 1


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def dev(vals):
    a = np.array([to_limbs(v) for v in vals], dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64).copy()).cuda()


def ints(t):
    return [from_limbs(r) for r in t.cpu().numpy().view(np.uint64).reshape(-1, 4)]


def edge_below(bound):
    e = [0, 1, 2, 3, P - 1, P - 2, (P - 1) // 2, 1 << 253, (1 << 253) - 1, 1 << 24, (1 << 24) - 1,
         (1 << 48) - 1, 0xFFFFFF << 240, bound - 1, bound - 2]
    e += [sum(0xFFFFFF << (24 * k) for k in range(j)) for j in range(1, 11)]
    return [v for v in e if v < bound]


def operands(bound, n, seed):
    rnd = random.Random(seed)
    edge = edge_below(bound)
    a = edge * len(edge) + [rnd.randrange(bound) for _ in range(n)]
    b = [x for x in edge for _ in edge] + [rnd.randrange(bound) for _ in range(n)]
    return a, b


@pytest.mark.parametrize("pipe,bound", [("fp64", 2 * P), ("int", P)])
def test_mul(pipe, bound):
    from provekit_b200.field import fr_op
    a, b = operands(bound, 20000, 11)
    got = ints(fr_op("mul", dev(a), dev(b), pipe=pipe))
    want = [x * y * RINV % P for x, y in zip(a, b)]
    bad = [i for i, (g, w) in enumerate(zip(got, want)) if g != w]
    assert not bad, (pipe, bad[:5], [(hex(a[i]), hex(b[i])) for i in bad[:3]])


@pytest.mark.parametrize("pipe,bound", [("fp64", 2 * P), ("int", P)])
def test_sqr(pipe, bound):
    from provekit_b200.field import fr_op
    a, _ = operands(bound, 20000, 12)
    got = ints(fr_op("sqr", dev(a), pipe=pipe))
    assert got == [x * x * RINV % P for x in a]


@pytest.mark.parametrize("pipe,bound", [("fp64", 1 << 256), ("int", 1 << 256)])
def test_from_mont(pipe, bound):
    from provekit_b200.field import fr_op
    a, _ = operands(bound, 20000, 13)
    a += [TOP, TOP - 1, 1 << 255] if bound > TOP else []
    got = ints(fr_op("from_mont", dev(a), pipe=pipe))
    assert got == [x * RINV % P for x in a]


def test_pipes_agree_on_canonical_inputs():
    from provekit_b200.field import fr_op
    a, b = operands(P, 50000, 14)
    A, B = dev(a), dev(b)
    assert torch.equal(fr_op("mul", A, B, pipe="fp64"), fr_op("mul", A, B, pipe="int"))
    assert torch.equal(fr_op("sqr", A, pipe="fp64"), fr_op("sqr", A, pipe="int"))


def test_rejects_bad_arguments():
    from provekit_b200._lib import PkgError, lib
    a = dev([1, 2])
    assert lib().pkg_fr_mul_batch(a.data_ptr(), a.data_ptr(), a.data_ptr(), 2, 9, None) == -1
    assert lib().pkg_fr_mul_batch(a.data_ptr(), None, a.data_ptr(), 2, 0, None) == -1
    assert lib().pkg_fr_mul_batch(None, None, None, 0, 1, None) == 0
    _ = PkgError
