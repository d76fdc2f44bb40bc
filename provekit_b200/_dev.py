"""Device-buffer helpers: torch tensors as plain device pointers."""
import torch


def ptr(t):
    """Device (or host) address of a tensor, or None for an absent buffer."""
    if t is None:
        return None
    return t.data_ptr()


def stream_handle(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def fr_tensor(t, name="values"):
    if t.dtype != torch.int64 or t.dim() != 2 or t.shape[1] != 4:
        raise ValueError(f"{name} must be an int64 tensor of shape (n, 4)")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def byte_tensor(t, name="input"):
    if t.dtype != torch.uint8 or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous uint8 tensor")
    return t
