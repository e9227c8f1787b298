"""Generates tests/golden/prep/prep.npz: outputs of the reference's own data-prep
scripts (software/scripts/tvtensor.py and stensor.py) on a seeded input.

The scripts are run unmodified except for three lines: their hard-coded
`tensordir` / `tensorname` now point at a temporary directory, and
`random.seed(SEED)` follows their imports (tvtensor.py draws from an
unseeded generator).  The fixture holds the input file and every output
file as bytes; tests/test_prep.py checks that cutc_b200.prep writes the same
bytes.  Test infrastructure only:

    python tests/golden/prep/make_prep_golden.py [reference root]
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEEDS = (7, 20240611)


def make_input(rng) -> str:
    """~1500 lines "i j k v": repeated (i, j) pairs (the stable sort keeps
    their file order), values with 1-17 significant digits, halfway cases of
    the %.1f rounding, negative values, and large indices."""
    lines = []
    for _ in range(1500):
        i = int(rng.integers(1, 40))
        j = int(rng.integers(1, 12))
        k = int(rng.integers(1, 300))
        r = rng.random()
        if r < 0.5:
            v = "%.3f" % rng.uniform(-2, 7)
        elif r < 0.7:
            v = repr(float(rng.uniform(0, 5)))
        elif r < 0.8:
            v = ["0.05", "0.15", "0.25", "0.35", "2.45", "-0.05", "1e3", "4.0"][int(rng.integers(8))]
        else:
            v = "%d" % int(rng.integers(1, 6))
        if rng.random() < 0.01:
            i = int(rng.integers(1, 1 << 40))
        lines.append(f"{i} {j} {k} {v}\n")
    return "".join(lines)


def patch(src: str, tensordir: str, name: str, seed: int | None) -> str:
    src = re.sub(r'^tensordir = .*$', f'tensordir = "{tensordir}/"', src, count=1, flags=re.M)
    src = re.sub(r'^tensorname = .*$', f'tensorname = "{name}"', src, count=1, flags=re.M)
    if seed is not None:
        src = src.replace("from operator import *", f"from operator import *\nrandom.seed({seed})", 1)
    return src


def main(ref_root: str):
    scripts = os.path.join(ref_root, "software", "scripts")
    tv = open(os.path.join(scripts, "tvtensor.py")).read()
    st = open(os.path.join(scripts, "stensor.py")).read()
    out = {}
    rng = np.random.default_rng(5)
    text = make_input(rng)
    out["input"] = np.frombuffer(text.encode(), dtype=np.uint8)
    out["seeds"] = np.array(SEEDS, dtype=np.uint64)
    for seed in SEEDS:
        with tempfile.TemporaryDirectory() as d:
            name = "golden"
            with open(os.path.join(d, name + ".tns"), "w") as f:
                f.write(text)
            with open(os.path.join(d, "tv.py"), "w") as f:
                f.write(patch(tv, d, name, seed))
            with open(os.path.join(d, "st.py"), "w") as f:
                f.write(patch(st, d, name, None))
            subprocess.run([sys.executable, "tv.py"], cwd=d, check=True, capture_output=True)
            subprocess.run([sys.executable, "st.py"], cwd=d, check=True, capture_output=True)
            for suffix in ("_tr", "_v", "_te", "_tr2", "_tr3"):
                data = open(os.path.join(d, name + suffix + ".tns"), "rb").read()
                out[f"{seed}{suffix}"] = np.frombuffer(data, dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "prep.npz"), **out)
    print("wrote", os.path.join(HERE, "prep.npz"), {k: v.size for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["CTC_REFERENCE_ROOT"])
