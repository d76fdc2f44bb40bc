"""Skyscraper Merkle trees and the WHIR commit of one polynomial on the GPU."""
import torch

from ._dev import byte_tensor, fr_tensor, ptr, stream_handle
from ._lib import PKG_LEAF_CANONICAL, PKG_LEAF_MONTGOMERY, check, lib  # noqa: F401


def merkle_tree(leaves, leaf_size: int, layers=None, stream=None):
    """Binary tree over count = len(leaves)/leaf_size leaves (power of two).
    Returns the (2*count-1)*32-byte layer array: leaf digests first, root last."""
    byte_tensor(leaves, "leaves")
    count = leaves.numel() // leaf_size
    if layers is None:
        layers = torch.empty(32 * (2 * count - 1), dtype=torch.uint8, device=leaves.device)
    check(lib().pkg_merkle_tree(ptr(leaves), leaf_size, count, ptr(layers), stream_handle(stream)))
    return layers


def merkle_tree_fr(codeword, fr_per_leaf: int, leaf_encoding=PKG_LEAF_CANONICAL, layers=None,
                   stream=None):
    """Tree whose leaf i is codeword row i (fr_per_leaf Fr)."""
    fr_tensor(codeword, "codeword")
    count = codeword.shape[0] // fr_per_leaf
    if layers is None:
        layers = torch.empty(32 * (2 * count - 1), dtype=torch.uint8, device=codeword.device)
    check(lib().pkg_merkle_tree_fr(ptr(codeword), fr_per_leaf, count, leaf_encoding, ptr(layers),
                                   stream_handle(stream)))
    return layers


def whir_commit(coeffs, folding_factor: int, log_inv_rate: int, masks=None,
                leaf_encoding=PKG_LEAF_CANONICAL, codeword=None, layers=None, stream=None):
    """RS-encode 2^folding_factor contiguous messages of the coefficient vector
    at rate 2^-log_inv_rate and commit the rows.  Returns (codeword, layers);
    the root is layers[-32:]."""
    fr_tensor(coeffs, "coeffs")
    n = coeffs.shape[0]
    M = 1 << folding_factor
    cw_len = (n // M) << log_inv_rate
    if codeword is None:
        codeword = torch.empty((cw_len * M, 4), dtype=torch.int64, device=coeffs.device)
    if layers is None:
        layers = torch.empty(32 * (2 * cw_len - 1), dtype=torch.uint8, device=coeffs.device)
    check(lib().pkg_whir_commit(ptr(coeffs), n, folding_factor, log_inv_rate, ptr(masks),
                                0 if masks is None else masks.shape[0], leaf_encoding,
                                ptr(codeword), ptr(layers), stream_handle(stream)))
    return codeword, layers
