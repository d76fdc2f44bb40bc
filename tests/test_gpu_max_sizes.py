"""GPU checks at the largest sizes, where the oracle would take too long:
size-independent properties instead of element-wise parity.

* ntt_nr at 2^28 (the largest order the twiddle table supports): intt_rn
  brings the input back exactly, and sampled outputs equal the polynomial
  evaluated at omega^bitrev(k) by the independent Horner kernel.
* The WHIR commit of 2^24 coefficients (a 2^26-Fr codeword): its root equals
  the root of a tree built from the same codeword by the byte-path kernels
  (Montgomery -> canonical, hash_many leaves, tree levels)."""
import numpy as np
import pytest
import torch

from fieldutil import P, from_limbs, root_of_unity, to_limbs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib():
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from provekit_b200 import build
    build.build()


def random_fr_device(n, seed):
    """n uniform-ish Fr below p (top limb masked), built on the host in chunks."""
    rng = np.random.default_rng(seed)
    out = torch.empty((n, 4), dtype=torch.int64, device="cuda")
    chunk = 1 << 24
    for i in range(0, n, chunk):
        m = min(chunk, n - i)
        h = rng.integers(0, 2**63, size=(m, 4), dtype=np.uint64) * 2 + 1
        h[:, 3] &= np.uint64(0x2FFFFFFFFFFFFFFF)
        out[i:i + m] = torch.from_numpy(h.view(np.int64)).cuda()
    return out


def test_ntt_2_28_round_trip_and_sampled_evaluations():
    from provekit_b200.ntt import intt_rn, ntt_nr
    from provekit_b200.whir import poly_eval_many
    n, logn = 1 << 28, 28
    x = random_fr_device(n, 28)
    d = x.clone()
    ntt_nr(d, n, 1)
    # output k is x(omega^bitrev(k)) (evaluation points of RSFr / ntt_nr)
    w = root_of_unity(n)
    ks = [0, 1, 2, 12345, n - 1]
    pts = []
    for k in ks:
        e = int(format(k, f"0{logn}b")[::-1], 2)
        z = pow(w, e, P) * pow(2, 256, P) % P  # Montgomery form
        pts.append(to_limbs(z))
    got = poly_eval_many(x, np.array(pts, dtype=np.uint64))
    out = d[torch.tensor(ks, device="cuda")].cpu().numpy().view(np.uint64)
    for j in range(len(ks)):
        assert from_limbs(got[j]) == from_limbs(out[j]), ks[j]
    intt_rn(d)
    assert torch.equal(d, x)


def test_commit_2_24_root_equals_the_byte_path_tree():
    from provekit_b200._lib import PKG_LEAF_CANONICAL
    from provekit_b200.field import fr_op
    from provekit_b200.merkle import merkle_tree, whir_commit
    n, ff, lr = 1 << 24, 4, 2
    M = 1 << ff
    c = random_fr_device(n, 24)
    cw, layers = whir_commit(c, ff, lr, leaf_encoding=PKG_LEAF_CANONICAL)
    canon = fr_op("from_mont", cw, pipe="fp64")
    byte_layers = merkle_tree(canon.view(torch.uint8).reshape(-1), 32 * M)
    assert torch.equal(byte_layers[-32:], layers[-32:])
    assert torch.equal(byte_layers, layers)
