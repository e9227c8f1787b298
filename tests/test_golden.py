"""The oracle and the engine's host code against golden vectors made by the
reference's own tt_read / ciss_alloc / cissbasic_alloc (tests/golden/,
generated by tests/golden/make_golden.py).  CPU only."""
import glob
import json
import os

import numpy as np
import pytest

import cutc_b200 as ctc
from oracle import pyoracle as po

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
INDEX = json.load(open(os.path.join(GOLD, "index.json")))
CASES = [c["name"] for c in INDEX["cases"]]


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def sort_mode(ind, vals, m):
    o = np.lexsort((ind[(m + 1) % 3], ind[m]))
    return ind[:, o], vals[o]


def same_ciss(got, z, prefix):
    assert np.array_equal(got["directory"], z[prefix + "directory"])
    assert np.array_equal(got["dcounter"], z[prefix + "dcounter"])
    w = z[prefix + "written"]
    assert got["entries"].shape == w.shape
    # the builder must write exactly the slots the reference writes ...
    assert np.array_equal(got["written"].astype(bool), w)
    # ... with the same bits (-0.0 of tile 0's header included)
    assert np.array_equal(got["entries"].view(np.uint64)[w], z[prefix + "entries"].view(np.uint64)[w])


@pytest.mark.parametrize("name", CASES)
def test_oracle_tns_reader(name, tmp_path):
    z = load(name)
    p = tmp_path / "t.tns"
    p.write_text(str(z["tns"]))
    t = po.tns_read(str(p))
    assert np.array_equal(t.ind, z["ind"])
    assert np.array_equal(t.vals.view(np.uint64), z["vals"].view(np.uint64))
    assert t.dims == [int(x) for x in z["dims"]]


@pytest.mark.parametrize("name", CASES)
def test_engine_tns_reader(name, tmp_path):
    z = load(name)
    p = tmp_path / "t.tns"
    p.write_text(str(z["tns"]))
    t = ctc.tt_read(str(p))
    ind, vals = t.export()
    assert np.array_equal(ind, z["ind"])
    assert np.array_equal(vals.view(np.uint64), z["vals"].view(np.uint64))
    assert t.dims == [int(x) for x in z["dims"]]


@pytest.mark.parametrize("name", [c for c in CASES if c != "zero_based"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_oracle_ciss(name, mode):
    z = load(name)
    si, sv = sort_mode(z["ind"], z["vals"], mode)
    got = po.ciss_build(po.Tensor(si, sv, [int(x) for x in z["dims"]]), mode, 32)
    same_ciss(got, z, f"m{mode}_")


@pytest.mark.parametrize("name", [c for c in CASES if c != "zero_based"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_engine_ciss(name, mode):
    z = load(name)
    si, sv = sort_mode(z["ind"], z["vals"], mode)
    t = ctc.Tensor.from_coo(si, sv, dims=[int(x) for x in z["dims"]])
    got = ctc.ciss_alloc(t, mode + 1, 32)
    same_ciss(got, z, f"m{mode}_")


@pytest.mark.parametrize("T", INDEX["tile_cases"])
def test_tile_lengths(T):
    z = load("n100")
    si, sv = sort_mode(z["ind"], z["vals"], 0)
    dims = [int(x) for x in z["dims"]]
    same_ciss(po.ciss_build(po.Tensor(si, sv, dims), 0, T, ga=True), z, f"t{T}_")
    same_ciss(ctc.ciss_alloc(ctc.Tensor.from_coo(si, sv, dims=dims), 1, T, ga=True), z, f"t{T}_")


def test_golden_files_cover_edge_cases():
    names = set(CASES)
    # nnz % 32 in {0, 1, 31}, one row, all-distinct rows, a single nonzero
    assert {"n32", "n33", "n31", "one_row", "distinct_rows", "single", "n64"} <= names
    assert len(glob.glob(os.path.join(GOLD, "*.npz"))) == len(CASES)


@pytest.mark.skipif(not po.ref_host_available(), reason="reference host library not built")
def test_live_reference_ciss_random():
    """Against the live reference build, on fresh random tensors."""
    rng = np.random.default_rng(7)
    for nnz in (96, 97, 500):
        ind = np.stack([rng.integers(1, d + 1, nnz) for d in (15, 11, 7)]).astype(np.uint64)
        vals = rng.uniform(-2, 6, nnz)
        for m in range(3):
            si, sv = sort_mode(ind, vals, m)
            T = po.Tensor(si, sv, [15, 11, 7])
            a = po.ciss_build(T, m, 32)
            b = po.ref_ciss_alloc(T, m + 1)
            w = a["written"]
            assert np.array_equal(a["directory"], b["directory"])
            assert np.array_equal(a["dcounter"], b["dcounter"])
            assert np.array_equal(a["entries"].view(np.uint64)[w], b["entries"].view(np.uint64)[w])


def test_numpy_cp_grad_is_the_fd_gradient():
    """The order-d FP64 restatement of the masked CP loss gradient (the
    adjoint kernel's checker) against central finite differences."""
    rng = np.random.default_rng(5)
    dims = (5, 4, 3, 2)
    ind = np.stack([rng.integers(1, d + 1, 40) for d in dims]).astype(np.uint64)
    v = rng.uniform(1, 5, 40)
    U = [rng.uniform(0, 1, (d, 3)) for d in dims]
    G = po.cp_grad(ind, v, U, 0.2)
    h = 1e-6
    for m in range(4):
        for r in range(dims[m]):
            for c in range(3):
                Up = [u.copy() for u in U]
                Um = [u.copy() for u in U]
                Up[m][r, c] += h
                Um[m][r, c] -= h
                fd = (po.cp_objective(ind, v, Up, 0.2) - po.cp_objective(ind, v, Um, 0.2)) / (2 * h)
                assert abs(fd - G[m][r, c]) < 1e-6 * max(1.0, abs(fd))
