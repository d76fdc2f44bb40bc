"""Element-wise BN254 Fr arithmetic on device tensors (pkg_fr_mul_batch): the
Montgomery product, square and Montgomery->canonical conversion on the FP64
pipe (the routines inside the NTT and Skyscraper kernels) or the integer pipe.
Mirrors skyscraper/bn254-multiplier/src/scalar.rs:12-132 (scalar_mul,
scalar_sqr) up to the residue (results here are fully reduced)."""
import torch

from ._dev import fr_tensor, ptr, stream_handle
from ._lib import check, lib

OPS = {("mul", "fp64"): 0, ("sqr", "fp64"): 1, ("from_mont", "fp64"): 2,
       ("mul", "int"): 3, ("sqr", "int"): 4, ("from_mont", "int"): 5}


def fr_op(op: str, a: torch.Tensor, b: torch.Tensor = None, pipe: str = "fp64", out=None,
          stream=None) -> torch.Tensor:
    """out[i] = op(a[i], b[i]); op in {"mul", "sqr", "from_mont"}, pipe in
    {"fp64", "int"}.  Inputs are (n, 4) int64 device tensors of Fr limbs."""
    code = OPS[(op, pipe)]
    fr_tensor(a, "a")
    if op == "mul":
        fr_tensor(b, "b")
        if b.shape != a.shape:
            raise ValueError("a and b must have the same shape")
    if out is None:
        out = torch.empty_like(a)
    check(lib().pkg_fr_mul_batch(ptr(a), ptr(b) if op == "mul" else None, ptr(out), a.shape[0],
                                 code, stream_handle(stream)))
    return out
