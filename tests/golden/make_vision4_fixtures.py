"""Extracts the reference's Vision-4 known answers into vision4_kat.json.

Sources (read as text; nothing of the reference is executed):
  verifier/verifier/src/hash/vision_4/permutation.rs  test_permutation: the two cases with fixed
      inputs (the third draws its input from StdRng, which is not restated here)
  verifier/verifier/src/hash/vision_4/constants.rs    ROUND_CONSTANTS (checked against the
      derivation in test_round_constants) and B_INV_COEFFS (the linearized polynomial of B^-1,
      checked against B^-1 o B = id in test_b_inverse_coeffs)

Usage: python tests/golden/make_vision4_fixtures.py <reference root>
"""
import json
import os
import re
import sys

HEX = re.compile(r"Ghash::new\((0x[0-9a-fA-F]+)\)")


def block(text, start, end_pat=r"\n\];"):
    i = text.index(start)
    j = re.compile(end_pat).search(text, i).start()
    return [int(h, 16) for h in HEX.findall(text[i:j])]


def main():
    if len(sys.argv) != 2:
        print(__doc__)
        return 2
    base = os.path.join(sys.argv[1], "verifier/verifier/src/hash/vision_4")
    consts = open(os.path.join(base, "constants.rs")).read()
    perm = open(os.path.join(base, "permutation.rs")).read()
    round_constants = block(consts, "pub static ROUND_CONSTANTS")
    b_inv = block(consts, "pub static B_INV_COEFFS")
    assert len(round_constants) == 4 * 17 and len(b_inv) == 129
    t = perm[perm.index("fn test_permutation"):]
    t = t[:t.index("for (input, expected) in cases")]
    vals = [int(h, 16) for h in HEX.findall(t)]
    # case 1: all-zero input (array::from_fn(|_| Ghash::new(0x0))) then 4 outputs;
    # case 2: 4 inputs then 4 outputs; case 3 (random input): 4 outputs, dropped
    cases = [
        {"input": [0, 0, 0, 0], "output": vals[1:5]},
        {"input": vals[5:9], "output": vals[9:13]},
    ]
    hx = lambda v: "%032x" % v  # noqa: E731
    out = {
        "source": "verifier/verifier/src/hash/vision_4/{permutation.rs,constants.rs}",
        "permutation": [{"input": [hx(v) for v in c["input"]],
                         "output": [hx(v) for v in c["output"]]} for c in cases],
        "round_constants": [[hx(v) for v in round_constants[4 * r:4 * r + 4]] for r in range(17)],
        "b_inv_coeffs": [hx(v) for v in b_inv],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vision4_kat.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print("wrote", dst)


if __name__ == "__main__":
    main()
