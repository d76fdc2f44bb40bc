"""Extract the known-answer vectors that the reference's own tests hold for
the prover hot path, and write them to ``reference_kats.json`` beside this
script.

The vectors are read as text from the reference's Rust test modules:

* Skyscraper: ``skyscraper/core/src/reference.rs`` tests ``test_ss_2``,
  ``test_bb_6``, ``test_zero``, ``test_random`` (sage-derived) and the sbox
  table in ``test_sbox``.
* Spartan sumcheck helpers: ``provekit/common/src/utils/sumcheck.rs`` tests
  (``calculate_eq`` = 2 289 441, the eq-hypercube cross checks, the 3x4 R1CS
  of ``make_test_r1cs`` and the expected ``multiply_transposed_by_eq_alpha``
  vectors).
* Poseidon2: ``poseidon2/src/permutation.rs`` ``smoke_test`` and
  ``poseidon2/src/hash.rs`` single/two-element hashes.
* The field's two-adic root of unity: the square-root constants of
  ``noir-examples/babyjubjub/src/hash_to_curve.nr`` (Z = 5, C1 = 28 = the
  two-adicity, C5 = Z^((p-1)/2^28)), i.e. the 2^28-th root of unity that
  ark-bn254's ``Fr::get_root_of_unity`` raises to the NTT's order.

Run from the repository root:  python tests/golden/extract_reference_kats.py <reference checkout>
(the reference checkout is only needed to regenerate the JSON; the tests read
the committed JSON).
"""
import json
import os
import re
import sys

REF = ""  # the reference checkout, set from the command line
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def fn_body(src: str, name: str) -> str:
    """Return the text of `fn name(...) { ... }` by brace matching."""
    m = re.search(r"fn\s+" + re.escape(name) + r"\s*\(", src)
    if not m:
        raise KeyError(name)
    i = src.index("{", m.end())
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i : j + 1]
    raise ValueError(name)


def quoted_decimals(body: str):
    return [int(s) for s in re.findall(r'"(\d+)"', body)]


def fe_list(text: str):
    """fe(N) / fe(-N) calls in order."""
    return [int(v) for v in re.findall(r"fe\((-?\d[\d_]*)\)", text.replace("_", ""))]


def skyscraper_kats():
    path = os.path.join(REF, "skyscraper/core/src/reference.rs")
    src = open(path).read()
    out = {"source": "skyscraper/core/src/reference.rs"}
    for test, op, rnd in [("test_ss_2", "ss", 2), ("test_bb_6", "bb", 6), ("test_random", "permute", None)]:
        l, r, el, er = quoted_decimals(fn_body(src, test))
        out[test] = {"op": op, "round": rnd, "l": str(l), "r": str(r), "el": str(el), "er": str(er)}
    el, er = quoted_decimals(fn_body(src, "test_zero"))
    out["test_zero"] = {"op": "permute", "round": None, "l": "0", "r": "0", "el": str(el), "er": str(er)}
    pairs = re.findall(r"sbox\((0x[0-9a-fA-F]+)\),\s*(0x[0-9a-fA-F]+)\)", fn_body(src, "test_sbox"))
    out["test_sbox"] = [[int(a, 16), int(b, 16)] for a, b in pairs]
    return out


def sumcheck_kats():
    path = os.path.join(REF, "provekit/common/src/utils/sumcheck.rs")
    src = open(path).read()
    out = {"source": "provekit/common/src/utils/sumcheck.rs"}
    body = fn_body(src, "test_calculate_eq_non_boolean")
    r, alpha = re.findall(r"\[(fe\([^\]]*)\]", body)[:2]
    expected = fe_list(body.split("assert_eq!")[1])
    out["calculate_eq"] = {"r": fe_list(r), "alpha": fe_list(alpha), "expected": expected[-1]}
    body = fn_body(src, "test_eval_eq_truncated_left_only")
    out["eval_eq_left_only"] = {"r": [2, 3, 5], "subtree_size": 8, "expected": fe_list(body.split("assert_eq!")[1])[-1]}
    body = fn_body(src, "test_eq_hypercube_single_entry")
    out["eq_single_entry"] = {"r": fe_list(re.search(r"let r = \[(.*?)\];", body).group(1))}
    # make_test_r1cs: add_constraint(&[(coef, col), ...], &[...], &[...])
    body = fn_body(src, "make_test_r1cs")
    cons = []
    for m in re.finditer(r"add_constraint\((.*?)\);", body, re.S):
        groups = re.findall(r"&\[(.*?)\]", m.group(1), re.S)
        parsed = []
        for g in groups:
            terms = re.findall(r"\(fe\((-?\d+)\),\s*(\d+)\)", g)
            parsed.append([[int(c), int(col)] for c, col in terms])
        cons.append(parsed)
    nw = int(re.search(r"add_witnesses\((\d+)\)", body).group(1))
    out["test_r1cs"] = {"num_witnesses": nw, "constraints": cons}
    body = fn_body(src, "test_multiply_transposed_by_eq_alpha")
    alpha = fe_list(re.search(r"let alpha = \[(.*?)\];", body).group(1))
    exp = {}
    for k in "abc":
        exp[k] = fe_list(re.search(r"let expected_%s = vec!\[(.*?)\];" % k, body).group(1))
    out["multiply_transposed_by_eq_alpha"] = {"alpha": alpha, "expected": exp}
    return out


def poseidon2_kats():
    perm = open(os.path.join(REF, "poseidon2/src/permutation.rs")).read()
    body = fn_body(perm, "smoke_test")
    exp = [int(h, 16) for h in re.findall(r'fe\("([0-9A-Fa-f]+)"\)', body)]
    out = {"source": "poseidon2/src/permutation.rs, poseidon2/src/hash.rs",
           "permutation_zero": {"input": [0, 0, 0, 0], "expected": [str(x) for x in exp]}}
    hsrc = open(os.path.join(REF, "poseidon2/src/hash.rs")).read()
    b1 = fn_body(hsrc, "test_poseidon2_hash_single_element")
    h1 = [int(h, 16) for h in re.findall(r'fe\("0x([0-9a-fA-F]+)"\)', b1)]
    out["hash_single"] = {"input": ["1"], "expected": str(h1[-1])}
    b2 = fn_body(hsrc, "test_poseidon2_hash_two_elements")
    h2 = [int(h, 16) for h in re.findall(r'fe\("0x([0-9a-fA-F]+)"\)', b2)]
    out["hash_two"] = {"input": [str(h2[0]), str(h2[0])], "expected": str(h2[-1])}
    return out


def root_of_unity_kats():
    path = "noir-examples/babyjubjub/src/hash_to_curve.nr"
    src = open(os.path.join(REF, path)).read()
    consts = {}
    for name in ("Z", "C1", "C5"):
        m = re.search(r"global\s+" + name + r"\s*:\s*\w+\s*=\s*(\d+)\s*;", src)
        consts[name] = m.group(1)
    return {"source": path, "generator": consts["Z"], "two_adicity": consts["C1"],
            "two_adic_root": consts["C5"]}


def main():
    global REF
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: extract_reference_kats.py <reference checkout directory>")
    REF = sys.argv[1]
    kats = {"skyscraper": skyscraper_kats(), "sumcheck": sumcheck_kats(), "poseidon2": poseidon2_kats(),
            "root_of_unity": root_of_unity_kats()}
    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
