"""The ntt crate's API (ntt/src/ntt.rs) over the CUDA implementation."""
import numpy as np

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib


def ntt_nr(values, codeword_size: int, num_groups: int, stream=None):
    """In-place NTT, normal order -> bit-reversed order, over
    len(values) / codeword_size interleaved columns, skipping the first
    log2(num_groups) stages (ntt/src/ntt.rs:105-108).  values: CUDA int64
    tensor (n, 4)."""
    fr_tensor(values)
    check(lib().pkg_ntt_nr(ptr(values), values.shape[0], codeword_size, num_groups,
                           stream_handle(stream)))
    return values


def intt_rn(values, stream=None):
    """In-place inverse NTT, bit-reversed -> normal order (ntt/src/ntt.rs:326-330)."""
    fr_tensor(values)
    check(lib().pkg_intt_rn(ptr(values), values.shape[0], stream_handle(stream)))
    return values


def host_ntt_nr(values: np.ndarray, codeword_size: int, num_groups: int):
    """Host-slice form (copy in, transform on the GPU, copy out)."""
    v = np.ascontiguousarray(values, dtype=np.uint64).reshape(-1, 4)
    check(lib().pkg_host_ntt_nr(v.ctypes.data, v.shape[0], codeword_size, num_groups))
    return v


def host_intt_rn(values: np.ndarray):
    v = np.ascontiguousarray(values, dtype=np.uint64).reshape(-1, 4)
    check(lib().pkg_host_intt_rn(v.ctypes.data, v.shape[0]))
    return v


class NTTEngine:
    """Device-resident twiddle table (ntt/src/ntt.rs:24-95).  The table is
    per device and grow-only; this object only reserves capacity."""

    def __init__(self, order: int = 1024):
        check(lib().pkg_ntt_engine_reserve(order))
        self._order = order

    @classmethod
    def with_order(cls, order: int):
        return cls(order)

    def order(self) -> int:
        return self._order
