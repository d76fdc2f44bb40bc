"""BN254 Poseidon2 (t = 4) over the CUDA implementation (poseidon2/src)."""
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib


def poseidon2_permutation_many(states, stream=None):
    """In place: states is a CUDA int64 tensor of shape (n*4, 4) (n states of
    4 Fr, Montgomery form)."""
    fr_tensor(states, "states")
    if states.shape[0] % 4:
        raise ValueError("states must hold a multiple of 4 field elements")
    check(lib().pkg_poseidon2_permutation_many(ptr(states), states.shape[0] // 4,
                                               stream_handle(stream)))
    return states


def poseidon2_hash_many(inputs, length: int, out=None, stream=None):
    """inputs: (n*length, 4) CUDA tensor -> (n, 4) hashes (poseidon2_hash)."""
    fr_tensor(inputs, "inputs")
    n = inputs.shape[0] // length if length else 0
    if out is None:
        out = torch.empty((n, 4), dtype=torch.int64, device=inputs.device)
    check(lib().pkg_poseidon2_hash_many(ptr(inputs), length, n, ptr(out), stream_handle(stream)))
    return out
