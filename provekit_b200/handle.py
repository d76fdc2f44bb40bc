"""Prover handles: the reference FFI's PKProver / PKBuf conventions
(tooling/provekit-ffi/src/ffi.rs) over the device prover (pkg_prover_* in
the C header).  A Prover holds a circuit resident on the device with its
transposes built once; prove() returns the proof bytes the library wrote
into a buffer it owns, copied out and released with pkg_free_buf."""
import ctypes
import struct

import numpy as np

from ._lib import PkgBuf, check, lib
from .whir import WhirParams


class ProverConfigC(ctypes.Structure):
    _fields_ = [("folding_factor", ctypes.c_uint), ("log_inv_rate", ctypes.c_uint),
                ("security_bits", ctypes.c_uint), ("pow_bits", ctypes.c_uint),
                ("zk", ctypes.c_int), ("transcript_domain", ctypes.c_uint64)]


class ProverInfoC(ctypes.Structure):
    _fields_ = [("num_constraints", ctypes.c_size_t), ("num_witnesses", ctypes.c_size_t),
                ("num_public_inputs", ctypes.c_size_t), ("m", ctypes.c_size_t),
                ("m0", ctypes.c_size_t), ("num_statements", ctypes.c_size_t),
                ("proof_bytes", ctypes.c_size_t), ("device", ctypes.c_int),
                ("whir", WhirParams)]


def config(transcript_domain=0, **over) -> ProverConfigC:
    """The reference's configuration (ff 3, rate 1/4, 128 bits, 10 PoW
    bits, whir-ZK) with the given fields replaced."""
    c = ProverConfigC()
    check(lib().pkg_prover_config_default(ctypes.byref(c)))
    c.transcript_domain = transcript_domain
    for k, v in over.items():
        setattr(c, k, v)
    return c


def _take(buf: PkgBuf) -> bytes:
    """Copy a library-owned buffer out and release it (exactly once)."""
    try:
        return ctypes.string_at(buf.ptr, buf.len) if buf.len else b""
    finally:
        lib().pkg_free_buf(buf)


def last_error_taken() -> str:
    """pkg_get_last_error: the thread's message, then cleared."""
    b = PkgBuf()
    check(lib().pkg_get_last_error(ctypes.byref(b)))
    return _take(b).decode()


class Prover:
    def __init__(self, handle):
        self._h = handle

    @classmethod
    def create(cls, h, cfg: ProverConfigC = None):
        """From a HostR1CS-like object (host CSR arrays and its public-input
        count)."""
        cfg = cfg if cfg is not None else config()
        rp = (ctypes.c_void_p * 3)(*[np.ascontiguousarray(a).ctypes.data for a in h.row_ptr])
        cl = (ctypes.c_void_p * 3)(*[np.ascontiguousarray(a).ctypes.data for a in h.cols])
        vl = (ctypes.c_void_p * 3)(*[np.ascontiguousarray(a).ctypes.data for a in h.vals])
        nnz = (ctypes.c_size_t * 3)(*h.nnz)
        out = ctypes.c_void_p()
        check(lib().pkg_prover_create(h.num_constraints, h.num_witnesses,
                                      getattr(h, "num_public_inputs", 0), rp, cl, vl, nnz,
                                      ctypes.byref(cfg), ctypes.byref(out)))
        return cls(out)

    @classmethod
    def load_bytes(cls, data: bytes):
        out = ctypes.c_void_p()
        buf = (ctypes.c_uint8 * len(data)).from_buffer_copy(data)
        check(lib().pkg_prover_load_bytes(buf, len(data), ctypes.byref(out)))
        return cls(out)

    def info(self) -> ProverInfoC:
        i = ProverInfoC()
        check(lib().pkg_prover_get_info(self._h, ctypes.byref(i)))
        return i

    def prove(self, witness: np.ndarray, blinding_seed: int = 1) -> bytes:
        w = np.ascontiguousarray(witness, dtype=np.uint64)
        b = PkgBuf()
        check(lib().pkg_prover_prove(self._h, w.ctypes.data, blinding_seed, ctypes.byref(b)))
        return _take(b)

    def serialize(self) -> bytes:
        b = PkgBuf()
        check(lib().pkg_prover_serialize(self._h, ctypes.byref(b)))
        return _take(b)

    def close(self):
        if self._h:
            lib().pkg_prover_free(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def parse_proof(data: bytes) -> dict:
    """The pkg_prover_prove layout -> the fields of prove_r1cs: a dict of
    Spartan fields (as provekit_b200.prover returns them), the WHIR
    commitment words and the WHIR proof words."""
    if data[:8] != b"PKGPROOF":
        raise ValueError("not a proof (bad magic)")
    version, _ = struct.unpack_from("<II", data, 8)
    if version != 1:
        raise ValueError(f"unsupported proof version {version}")
    m, m0, npub, nstm, cwords, pwords, domain = struct.unpack_from("<7Q", data, 16)
    whir = WhirParams.from_buffer_copy(data[72:176])
    at = 176
    root = bytes(data[at:at + 32])
    at += 32

    def fr(n):
        nonlocal at
        a = np.frombuffer(data, np.uint64, 4 * n, at).reshape(n, 4).copy()
        at += 32 * n
        return a

    sp = {"m": m, "m0": m0, "root": root, "r": fr(m0), "coeffs": fr(4 * m0), "alpha": fr(m0)}
    for k in ("rho", "sum_g", "blinding_eval", "public_x"):
        sp[k] = fr(1)[0]
    sp["evals"] = fr(3)
    sp["public_hash"] = fr(1)[0]
    sp["public_eval"] = fr(1)[0]
    t = fr(2)
    sp["transcript"] = (list(t[0]), list(t[1]))
    cw = np.frombuffer(data, np.uint64, cwords, at).copy()
    at += 8 * cwords
    proof = np.frombuffer(data, np.uint64, pwords, at).copy()
    at += 8 * pwords
    if at != len(data):
        raise ValueError(f"{len(data) - at} trailing bytes")
    return {"spartan": sp, "commit_words": cw, "proof": proof, "whir": whir,
            "num_public_inputs": npub, "num_statements": nstm, "transcript_domain": domain}
