"""Extracts the reference's own Poseidon2 constants fixture.

The reference ships, in
integration_test/zkc/riscv/zkc/lib/poseidon2/constants.zkc, the width-16
Poseidon2 round keys (27 rows of 16, partial rows zero-padded) and internal
diagonal of gnark-crypto's KoalaBear permutation.  The prover itself uses
width 24, whose keys are not in the tree; reproducing these width-16 keys
pins the key-derivation procedure that produces the width-24 ones.

Run in a container that has the reference checked out:
    python tests/golden/make_fixtures.py /path/to/loom
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_fixtures.py <path of the loom checkout>")
ref = sys.argv[1]
path = os.path.join(ref, "integration_test/zkc/riscv/zkc/lib/poseidon2/constants.zkc")
txt = open(path).read()
keys_txt = txt[txt.index("static round_keys"):txt.index("static internal_diag")]
diag_txt = txt[txt.index("static internal_diag"):]
keys = [int(h, 16) for h in re.findall(r"0x[0-9a-fA-F]{8}", keys_txt)]
diag = [int(h, 16) for h in re.findall(r"0x[0-9a-fA-F]{8}", diag_txt)]
assert len(keys) == 27 * 16 and len(diag) == 16
out = {
    "source": "integration_test/zkc/riscv/zkc/lib/poseidon2/constants.zkc",
    "width": 16, "full_rounds": 6, "partial_rounds": 21,
    "round_keys": [keys[16 * r:16 * r + 16] for r in range(27)],
    "internal_diag": diag,
}
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "poseidon2_w16_zkc.json")
with open(dst, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", dst)
