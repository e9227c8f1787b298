"""Data preparation of the reference's .tns datasets (software/scripts/
tvtensor.py and stensor.py), seeded and in native code.

tvtensor(src, out_dir, name, seed) reads `src` and writes
<out_dir>/<name>_tr.tns, _v.tns and _te.tns: the nonzeros sorted stably by
(i, j), each dealt by random.randint(0, 9) from Python's Mersenne Twister
seeded with `seed` to train (< 8), test (8) or validation (9), lines
"%d %d %d %.1f" (tvtensor.py:64-129; the script draws from an unseeded
generator).  stensor(train_path, out_dir, name) writes the mode-2 and
mode-3 copies <name>_tr2.tns (sorted stably by (j, k)) and _tr3.tns (by
(k, i)) of a training file (stensor.py:25-43).  Both go through the C ABI
(ctc_tensor_load_tns, ctc_tensor_split, ctc_tensor_sort,
ctc_tensor_write_tns).
"""
from __future__ import annotations

import os

from .api import Tensor

SCRIPT_DIGITS = 1  # the scripts' "%.1f"


def tvtensor(src: str, out_dir: str, name: str, seed: int) -> dict:
    t = Tensor.load(src)
    train, test, val = t.split(seed)
    paths = {}
    for suffix, part in (("_tr", train), ("_v", val), ("_te", test)):
        path = os.path.join(out_dir, name + suffix + ".tns")
        part.write_tns(path, SCRIPT_DIGITS)
        paths[suffix] = path
    return paths


def stensor(train_path: str, out_dir: str, name: str) -> dict:
    paths = {}
    for suffix, mode in (("_tr2", 1), ("_tr3", 2)):
        # each copy is sorted from the file's own order, as the script sorts
        # two lists read from the same file
        t = Tensor.load(train_path)
        path = os.path.join(out_dir, name + suffix + ".tns")
        t.sort(mode).write_tns(path, SCRIPT_DIGITS)
        paths[suffix] = path
        t.free()
    return paths
