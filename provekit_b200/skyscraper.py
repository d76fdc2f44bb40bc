"""Skyscraper compression and provekit's SkyscraperHashEngine
(provekit/common/src/skyscraper/whir.rs) on the GPU."""
import ctypes

import numpy as np
import torch

from ._dev import byte_tensor, ptr, stream_handle
from ._lib import check, lib

WIDTH_LCM = 12  # skyscraper/core/src/lib.rs:26

# SHA3-256("whir::hash" || "skyscraper") (provekit/common/src/skyscraper/whir.rs:17-20)
SKYSCRAPER_ENGINE_ID = bytes([
    0xa5, 0x0d, 0x5e, 0xe2, 0xa3, 0xfc, 0x52, 0xe9, 0x6f, 0x11, 0x10, 0x3c, 0xbb, 0x8a, 0x65, 0xa3,
    0x77, 0xb5, 0x82, 0xb0, 0xb2, 0xdd, 0x42, 0x1c, 0x66, 0x19, 0x13, 0xe6, 0xa5, 0x63, 0xf8, 0xa1])


def compress_many(messages, hashes=None, stream=None):
    """messages: CUDA uint8 tensor of n*64 bytes -> n*32-byte hashes."""
    byte_tensor(messages, "messages")
    if messages.numel() % 64:
        raise ValueError("Message length not a multiple of 64")
    n = messages.numel() // 64
    if hashes is None:
        hashes = torch.empty(32 * n, dtype=torch.uint8, device=messages.device)
    check(lib().pkg_skyscraper_compress_many(ptr(messages), n, ptr(hashes), stream_handle(stream)))
    return hashes


class SkyscraperHashEngine:
    """Mirror of `impl HashEngine for SkyscraperHashEngine`."""

    def name(self):
        return "skyscraper"

    def engine_id(self):
        return SKYSCRAPER_ENGINE_ID

    def supports_size(self, size: int) -> bool:
        return size > 0 and size % 32 == 0

    def preferred_batch_size(self) -> int:
        return WIDTH_LCM

    def hash_many(self, size: int, input, output=None, stream=None):
        """input: CUDA uint8 tensor of count*size bytes; output: count*32 bytes."""
        byte_tensor(input)
        count = input.numel() // size if size else 0
        if output is None:
            output = torch.empty(32 * count, dtype=torch.uint8, device=input.device)
        if size == 0 or input.numel() != size * (output.numel() // 32):
            raise ValueError(f"skyscraper: input length {input.numel()} != size {size} * count")
        check(lib().pkg_skyscraper_hash_many(size, ptr(input), output.numel() // 32, ptr(output),
                                             stream_handle(stream)))
        return output

    def host_hash_many(self, size: int, data: bytes) -> bytes:
        if size == 0 or len(data) % size:
            raise ValueError("input length is not a multiple of size")
        count = len(data) // size
        inp = np.frombuffer(data, dtype=np.uint8).copy()
        out = np.zeros(max(32 * count, 1), np.uint8)
        check(lib().pkg_host_skyscraper_hash_many(size, inp.ctypes.data, count, out.ctypes.data))
        return out[: 32 * count].tobytes()


def pow_solve(challenge, threshold) -> int:
    """Smallest nonce with compress(challenge, [nonce, 0, 0, 0]) < threshold
    (skyscraper/core/src/generic.rs:42-71).  challenge/threshold: 4 u64 limbs."""
    c = np.ascontiguousarray(np.asarray(challenge, dtype=np.uint64))
    t = np.ascontiguousarray(np.asarray(threshold, dtype=np.uint64))
    out = ctypes.c_uint64(0)
    check(lib().pkg_skyscraper_pow_solve(c.ctypes.data, t.ctypes.data, ctypes.byref(out)))
    return out.value
