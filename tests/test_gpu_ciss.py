"""The CISS layout built on the device (ctc_ciss_build_gpu) against the
reference's own outputs (golden fixtures) and the host builder, bit for
bit, including the device-side sort."""
from __future__ import annotations

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import synth
from tests.test_golden import CASES, INDEX, load, same_ciss, sort_mode

pytestmark = pytest.mark.gpu


def identical(a, b):
    for k in ("nnz", "dlength", "size_rows", "tile_len"):
        assert a[k] == b[k], k
    assert np.array_equal(a["directory"], b["directory"])
    assert np.array_equal(a["dcounter"], b["dcounter"])
    assert np.array_equal(a["written"], b["written"])
    assert np.array_equal(a["entries"].view(np.uint64), b["entries"].view(np.uint64))


@pytest.mark.parametrize("name", [c for c in CASES if c != "zero_based"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_gpu_ciss_golden(ctx, name, mode):
    z = load(name)
    si, sv = sort_mode(z["ind"], z["vals"], mode)
    t = ctc.Tensor.from_coo(si, sv, dims=[int(x) for x in z["dims"]])
    same_ciss(ctc.ciss_alloc_gpu(ctx, t, mode + 1, 32), z, f"m{mode}_")


@pytest.mark.parametrize("T", INDEX["tile_cases"])
def test_gpu_ciss_golden_tile_lengths(ctx, T):
    z = load("n100")
    si, sv = sort_mode(z["ind"], z["vals"], 0)
    dims = [int(x) for x in z["dims"]]
    same_ciss(ctc.ciss_alloc_gpu(ctx, ctc.Tensor.from_coo(si, sv, dims=dims), 1, T, ga=True), z, f"t{T}_")


@pytest.mark.parametrize("nnz", [1, 5, 31, 32, 33, 64, 65, 1000, 4096, 50001])
@pytest.mark.parametrize("T", [1, 2, 16, 31, 32, 63, 64])
def test_gpu_ciss_equals_host(ctx, nnz, T):
    dims = (max(2, nnz // 7), 40, 30)
    ind, vals = synth.random_small(nnz, dims, seed=nnz + T, low=-3.0, high=1e3)
    for mode in (0, 1, 2):
        si, sv = sort_mode(ind, vals, mode)
        t = ctc.Tensor.from_coo(si, sv, dims=dims)
        for ga in (False, True):
            identical(ctc.ciss_alloc_gpu(ctx, t, mode + 1, T, ga=ga), ctc.ciss_alloc(t, mode + 1, T, ga=ga))


def test_gpu_ciss_one_row_and_distinct_rows(ctx):
    rng = np.random.default_rng(3)
    for ind in (np.stack([np.ones(300, dtype=np.uint64), rng.integers(1, 50, 300).astype(np.uint64),
                          rng.integers(1, 40, 300).astype(np.uint64)]),
                np.stack([np.arange(1, 301, dtype=np.uint64), rng.integers(1, 50, 300).astype(np.uint64),
                          rng.integers(1, 40, 300).astype(np.uint64)])):
        vals = rng.uniform(-5, 5, 300)
        si, sv = sort_mode(ind, vals, 0)
        t = ctc.Tensor.from_coo(si, sv, dims=[300, 50, 40])
        for T in (1, 32, 64):
            identical(ctc.ciss_alloc_gpu(ctx, t, 1, T), ctc.ciss_alloc(t, 1, T))


def test_gpu_ciss_device_sort(ctx):
    """Unsorted input with sort=True: the stable (mode, next mode) order of
    the reference's traina/b/c files, then the same layout."""
    rng = np.random.default_rng(9)
    ind = np.stack([rng.integers(1, 60, 20000), rng.integers(1, 70, 20000),
                    rng.integers(1, 80, 20000)]).astype(np.uint64)  # duplicates: ties keep input order
    vals = rng.uniform(0, 10, 20000)
    t = ctc.Tensor.from_coo(ind, vals, dims=[60, 70, 80])
    for mode in (0, 1, 2):
        si, sv = sort_mode(ind, vals, mode)  # numpy lexsort is stable
        ts = ctc.Tensor.from_coo(si, sv, dims=[60, 70, 80])
        identical(ctc.ciss_alloc_gpu(ctx, t, mode + 1, 32, sort=True), ctc.ciss_alloc(ts, mode + 1, 32))
