"""Shared problem builders for the parity tests: the same seeded tensor and
initial factors go to the CUDA engine (through the C ABI) and to the FP64
CPU oracle."""
from __future__ import annotations

import numpy as np

import cutc_b200 as ctc
from cutc_b200 import synth
from oracle import pyoracle as po


class Problem:
    def __init__(self, nnz, dims, R, seed=0, heavy_row=0, low=1.0, high=5.0, test_frac=0.1,
                 distinct=True):
        rng = np.random.default_rng(seed + 1000)
        ind, vals = synth.random_small(nnz, dims, seed=seed, low=low, high=high, distinct=distinct)
        if heavy_row:
            # concentrate `heavy_row` extra nonzeros on row 1 of mode 0 to force
            # row pieces longer than a tile
            extra = np.stack([np.ones(heavy_row, dtype=np.uint64),
                              rng.integers(1, dims[1] + 1, heavy_row).astype(np.uint64),
                              rng.integers(1, dims[2] + 1, heavy_row).astype(np.uint64)])
            ind = np.concatenate([ind, extra], axis=1)
            vals = np.concatenate([vals, rng.uniform(low, high, heavy_row)])
            key = ind[0] * (dims[1] * dims[2] + 7) + ind[1] * (dims[2] + 3) + ind[2]
            _, first = np.unique(key, return_index=True)
            first.sort()
            ind, vals = ind[:, first], vals[first]
        n = ind.shape[1]
        is_test = rng.random(n) < test_frac
        self.dims = tuple(int(d) for d in dims)
        self.R = R
        self.train = (ind[:, ~is_test], vals[~is_test])
        self.test = (ind[:, is_test], vals[is_test])
        self.sorted = [synth.sort_for_mode(*self.train, m) for m in range(3)]
        self.U0 = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]

    # oracle side
    def o_sorted(self, m):
        return po.Tensor(*self.sorted[m], dims=self.dims)

    def o_test(self):
        return po.Tensor(*self.test, dims=self.dims)

    def o_train(self):
        return po.Tensor(*self.train, dims=self.dims)

    def factors(self):
        return [u.copy() for u in self.U0]

    # engine side
    def c_sorted(self):
        return [ctc.Tensor.from_coo(*self.sorted[m], dims=self.dims) for m in range(3)]

    def c_test(self):
        return ctc.Tensor.from_coo(*self.test, dims=self.dims)

    def c_model(self):
        m = ctc.Model(self.dims, self.R)
        m.set_factors(self.U0)
        return m


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def max_factor_rel(Ua, Ub):
    return max(rel(a, b) for a, b in zip(Ua, Ub))
