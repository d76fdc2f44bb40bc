"""Generate the BN254 t=4 Poseidon2 constants header from the reference's
constant tables (poseidon2/src/constants.rs: load_diag, load_rc_full1,
load_rc_partial, load_rc_full2 for t = 4), laid out as the reference's
Poseidon2Config builds them (poseidon2/src/permutation.rs:29-65): 64 rounds x 4
lanes, partial rounds only in lane 0.

    python tests/golden/gen_poseidon2_constants.py <reference checkout>

Writes provekit_b200/csrc/poseidon2_t4_constants.h and
oracle/poseidon2_t4_constants.h (same content: canonical and Montgomery u64
limbs).  The reference checkout is read only here; the headers are committed.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
P = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
R = pow(2, 256, P)


def arm(src, fn, t=4):
    m = re.search(r"pub fn " + fn + r"\(t: u32\).*?match t \{(.*?)\n    \}\n\}", src, re.S)
    body = m.group(1)
    a = re.search(r"\b%d => vec!\[(.*?)\n        \],\n" % t, body, re.S)
    return a.group(1)


def hexes(text):
    return [int(h, 16) % P for h in re.findall(r'fe\("(?:0x)?([0-9a-fA-F]+)"\)', text)]


def rows(text):
    return [hexes(v) for v in re.findall(r"vec!\[(.*?)\]", text, re.S)]


def limbs(x):
    return ", ".join("0x%016xULL" % ((x >> (64 * i)) & (2**64 - 1)) for i in range(4))


def main(ref):
    src = open(os.path.join(ref, "poseidon2/src/constants.rs")).read()
    diag = hexes(arm(src, "load_diag"))
    full1 = rows(arm(src, "load_rc_full1"))
    partial = hexes(arm(src, "load_rc_partial"))
    full2 = rows(arm(src, "load_rc_full2"))
    assert len(diag) == 4 and len(full1) == 4 and len(full2) == 4 and len(partial) == 56
    rc = [r for r in full1] + [[v, 0, 0, 0] for v in partial] + [r for r in full2]
    assert len(rc) == 64 and all(len(r) == 4 for r in rc)
    out = ["// Generated by tests/golden/gen_poseidon2_constants.py from the reference's",
           "// poseidon2/src/constants.rs (t = 4).  Do not edit.",
           "#pragma once", "#include <stdint.h>", ""]
    for name, conv in (("", lambda v: v), ("_MONT", lambda v: v * R % P)):
        out.append("static const uint64_t POSEIDON2_T4_DIAG%s[4][4] = {" % name)
        out += ["    {%s}," % limbs(conv(v)) for v in diag]
        out.append("};")
        out.append("static const uint64_t POSEIDON2_T4_RC%s[64][4][4] = {" % name)
        for r in rc:
            out.append("    {" + ", ".join("{%s}" % limbs(conv(v)) for v in r) + "},")
        out.append("};")
        out.append("")
    text = "\n".join(out)
    for path in (os.path.join(ROOT, "provekit_b200", "csrc", "poseidon2_t4_constants.h"),
                 os.path.join(ROOT, "oracle", "poseidon2_t4_constants.h")):
        with open(path, "w") as f:
            f.write(text)
        print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: gen_poseidon2_constants.py <reference checkout directory>")
    main(sys.argv[1])
