"""RSFr -- provekit's whir ReedSolomon<Fr> plugin (provekit/common/src/ntt.rs)
on the GPU."""
import ctypes

import numpy as np
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib


class RSFr:
    """Same methods, argument meaning and error behaviour as the reference's
    `impl ReedSolomon<Fr> for RSFr` (contract violations raise PkgError)."""

    def next_order(self, size: int):
        out = ctypes.c_size_t(0)
        rc = lib().pkg_rs_next_order(size, ctypes.byref(out))
        return None if rc else out.value

    def generator(self, codeword_length: int) -> np.ndarray:
        out = np.zeros(4, np.uint64)
        check(lib().pkg_rs_generator(codeword_length, out.ctypes.data))
        return out

    def evaluation_points(self, masked_message_length: int, codeword_length: int, indices):
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
        out = np.zeros((max(len(idx), 1), 4), np.uint64)
        check(lib().pkg_rs_evaluation_points(codeword_length, idx.ctypes.data, len(idx),
                                             out.ctypes.data))
        return out[: len(idx)]

    def interleaved_encode(self, messages, masks, codeword_length: int, out=None, stream=None):
        """messages: CUDA int64 tensor (M, L, 4) (message-major) or a list of
        (L, 4) tensors; masks: (k, 4) tensor or None.  Returns the
        (codeword_length * M, 4) codeword."""
        if isinstance(messages, (list, tuple)):
            if len(messages) == 0:
                return torch.zeros((0, 4), dtype=torch.int64, device="cuda")
            L = messages[0].shape[0]
            for m in messages:
                if m.shape[0] != L:
                    raise ValueError("messages must all have the same length")
            messages = torch.stack(list(messages))
        M, L = messages.shape[0], messages.shape[1]
        flat = messages.reshape(M * L, 4) if M * L else None
        if masks is not None and masks.shape[0] == 0:
            masks = None
        if masks is not None:
            fr_tensor(masks, "masks")
        if out is None:
            out = torch.empty((M * codeword_length, 4), dtype=torch.int64, device=messages.device)
        check(lib().pkg_rs_interleaved_encode(
            ptr(flat), M, L, ptr(masks), 0 if masks is None else masks.shape[0],
            codeword_length, ptr(out), stream_handle(stream)))
        return out

    def host_interleaved_encode(self, messages, masks, codeword_length: int) -> np.ndarray:
        """Host-slice form with the trait's message list (list of (L, 4) uint64
        arrays)."""
        M = len(messages)
        if M == 0:
            return np.zeros((0, 4), np.uint64)
        msgs = [np.ascontiguousarray(m, dtype=np.uint64).reshape(-1, 4) for m in messages]
        L = msgs[0].shape[0]
        ptrs = (ctypes.c_void_p * M)(*[m.ctypes.data for m in msgs])
        mk = None if masks is None or len(masks) == 0 else np.ascontiguousarray(masks, dtype=np.uint64)
        out = np.zeros((M * codeword_length, 4), np.uint64)
        check(lib().pkg_host_rs_interleaved_encode(
            ctypes.cast(ptrs, ctypes.c_void_p), M, L, None if mk is None else mk.ctypes.data,
            0 if mk is None else mk.reshape(-1, 4).shape[0], codeword_length, out.ctypes.data))
        return out
