"""Generate the golden fixtures of tests/golden/ from the reference's own tests.

Run with the path of a checkout of the reference:

    python tests/golden/make_golden.py REFERENCE_DIR

Writes
  - reference_N64.npz: the regression fixture test/data/reference_N64.txt
    (output of the original C++ code by N. Saito and S. Ishihara, Zenodo
    doi:10.5281/zenodo.10356125, CC BY 4.0; see the file's own header),
    parsed the way test/test_dynamics.jl:5-20 parses it: `init` (3 x 64:
    x, y, θ) and the snapshots after 1001 and 4001 steps (15 x 64 each:
    x y θ xc yc a2..a6 b2..b6);
  - philox_kat.json: the Philox4x32-10 known-answer vectors asserted by
    test/test_random.jl:4-11 (Random123's KATs).
The tests read only these files, never the reference itself.
"""

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_reference(path):
    """test/test_dynamics.jl:5-20: '#T=t' blocks hold the state after t+1 steps."""
    init, snaps, current = [], {}, None
    with open(path) as f:
        for line in f:
            if line.startswith("#init"):
                init.append([float(v) for v in line.split()[1:]])
            elif line.startswith("#T="):
                current = int(line[3:].split()[0]) + 1
                snaps[current] = []
            elif line.startswith("#cell"):
                snaps[current].append([float(v) for v in line.split()[1:]])
    return np.array(init).T, {k: np.array(v).T for k, v in snaps.items()}


def philox_kats(path):
    text = open(path).read()
    block = text[text.index("known-answer vectors"): text.index("standard normal noise")]
    vecs = []
    pat = re.compile(r"philox4x32\(\((.*?)\)(?: \.% UInt32)?, \((.*?)\)(?: \.% UInt32)?\) ==\s*\((.*?)\)", re.S)
    for m in pat.finditer(block):
        ints = lambda s: [int(v.strip(), 16) for v in s.split(",")]
        vecs.append({"ctr": ints(m.group(1)), "key": ints(m.group(2)), "out": ints(m.group(3))})
    return vecs


def main(ref):
    init, snaps = read_reference(os.path.join(ref, "test", "data", "reference_N64.txt"))
    np.savez_compressed(os.path.join(HERE, "reference_N64.npz"), init=init,
                        steps=np.array(sorted(snaps)), **{f"snap_{k}": v for k, v in snaps.items()})
    kats = philox_kats(os.path.join(ref, "test", "test_random.jl"))
    assert len(kats) == 3, kats
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump({"source": "test/test_random.jl:4-11 (Random123 Philox4x32-10 KATs)", "vectors": kats}, f, indent=1)
    print("init", init.shape, "snapshots", {k: v.shape for k, v in snaps.items()}, "kats", len(kats))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_DIR")
    main(sys.argv[1])
