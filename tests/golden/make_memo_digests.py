"""Writes tests/golden/memo_digests.json from the reference's shipped Golomb-Rice table.

Reads include/function/golombRiceMemo.hpp of ByteHamster/GpuRecSplit (23 rows of 3000
uint32 for leaf sizes 2..24, AbstractParallelRecSplit.hpp:191-227 generates them) and
records, per leaf size, the SHA-256 of the row as little-endian uint32 plus a few spot
values. Run once where the reference source tree is present, giving its path:

    python tests/golden/make_memo_digests.py <GpuRecSplit source tree>
"""
import hashlib
import json
import os
import re
import sys

import numpy as np


def main(ref_root: str) -> None:
    path = os.path.join(ref_root, "include", "function", "golombRiceMemo.hpp")
    text = open(path).read()
    body = text[text.index("golomb_rice_memo{{"):text.index("}};")]
    rows = re.findall(r"\{([^{}]*)\}", body)
    assert len(rows) == 23, len(rows)
    out = {"source": "include/function/golombRiceMemo.hpp", "leaf": {}}
    for i, row in enumerate(rows):
        vals = np.array([int(v, 16) for v in re.findall(r"0x[0-9A-Fa-f]+", row)], dtype="<u4")
        assert vals.size == 3000
        leaf = i + 2
        out["leaf"][str(leaf)] = {
            "sha256": hashlib.sha256(vals.tobytes()).hexdigest(),
            "spot": {str(m): int(vals[m]) for m in (2, leaf, leaf + 1, 100, 112, 560, 1000, 2000, 2999)},
        }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "memo_digests.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_memo_digests.py <path of the GpuRecSplit source tree>")
    main(sys.argv[1])
