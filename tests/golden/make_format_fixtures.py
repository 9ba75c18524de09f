"""Writes tests/golden/formats_v1.json: the reference's binary serialization fixtures
(verifier/core/test_data/{constraint_system_v2,witness_v1,proof_v1}.bin) as hex, with the contents
its own tests assert (verifier/core/src/constraint_system.rs:1465-1500, 1579-1600, 1775-1800).

Usage: python tests/golden/make_format_fixtures.py <reference root>
Run where the reference tree exists; the GPU box and the tests read only the committed JSON.
"""
import json
import os
import sys



def main():
    if len(sys.argv) != 2:
        print(__doc__)
        return 2
    data = os.path.join(sys.argv[1], "verifier", "core", "test_data")
    out = {}
    for name in ("constraint_system_v2", "witness_v1", "proof_v1"):
        with open(os.path.join(data, name + ".bin"), "rb") as f:
            out[name] = f.read().hex()
    out["expect"] = {
        "constraint_system_v2": {
            "layout": {"n_const": 3, "n_inout": 2, "n_witness": 10, "n_internal": 3,
                       "offset_inout": 4, "offset_witness": 8, "committed_total_len": 16,
                       "n_scratch": 0},
            "constants": [1, 42, 0xDEADBEEF], "n_and": 2, "n_mul": 1},
        "witness_v1": {"words": [1, 42, 0xDEADBEEF, 0x1234567890ABCDEF]},
        "proof_v1": {"challenger": "HasherChallenger<Sha256>",
                     "data": "0123456789abcdeffedcba9876543210deadbeefcafebabe"},
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "formats_v1.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")
    print("wrote", path)


if __name__ == "__main__":
    sys.exit(main())
