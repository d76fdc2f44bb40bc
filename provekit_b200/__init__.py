"""provekit_b200 -- B200-native (sm_100a) ProveKit Spartan+WHIR prover hot path.

Host mirror of the reference's call surfaces over the C ABI of
libprovekit_b200.so:

* ``provekit_b200.ntt``        -- the ntt crate: ntt_nr, intt_rn, NTTEngine
* ``provekit_b200.rs``         -- RSFr, whir's ReedSolomon<Fr> plugin
* ``provekit_b200.skyscraper`` -- compress_many, SkyscraperHashEngine, PoW
* ``provekit_b200.merkle``     -- Merkle trees and the WHIR commit

Field elements are BN254 Fr in arkworks' in-memory layout: int64 tensors of
shape (n, 4) (4 little-endian u64 limbs, Montgomery form) on a CUDA device.
"""
from ._lib import PkgError, lib  # noqa: F401

__all__ = ["PkgError", "lib", "ntt", "rs", "skyscraper", "merkle"]
