"""Plain-Python BN254 Fr helpers shared by the tests (big-int arithmetic and
limb packing).  Fr values travel as little-endian 4 x u64 limbs; "mont" is the
arkworks in-memory form x * 2^256 mod p."""
import numpy as np

P = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
R = pow(2, 256, P)
RINV = pow(R, P - 2, P)


def to_limbs(x: int):
    return [(x >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(4)]


def from_limbs(l) -> int:
    return sum(int(v) << (64 * i) for i, v in enumerate(l))


def pack(values, mont=True) -> np.ndarray:
    """List of ints -> (n, 4) uint64 array (Montgomery form when mont)."""
    out = np.zeros((len(values), 4), dtype=np.uint64)
    for i, v in enumerate(values):
        v %= P
        if mont:
            v = v * R % P
        out[i] = to_limbs(v)
    return out


def unpack(arr, mont=True):
    arr = np.asarray(arr, dtype=np.uint64).reshape(-1, 4)
    res = []
    for row in arr:
        v = from_limbs(row)
        res.append(v * RINV % P if mont else v)
    return res


def fe(v: int) -> int:
    return v % P


def root_of_unity(n: int) -> int:
    """ark-ff Fr::get_root_of_unity for n = 2^k: 5^((p-1)/2^28) squared 28-k times."""
    k = n.bit_length() - 1
    assert 1 << k == n and k <= 28
    w = pow(5, (P - 1) >> 28, P)
    for _ in range(28 - k):
        w = w * w % P
    return w


def bitrev(v: int, bits: int) -> int:
    r = 0
    for i in range(bits):
        r |= ((v >> i) & 1) << (bits - 1 - i)
    return r
