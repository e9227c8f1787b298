"""The reference's own CUDA kernels (sgpu/als.cu, ccd.cu, sgd.cu compiled
from source for sm_100a by oracle/build_ref.sh, rank 16) against the
oracle's lane-exact compat restatement, on the same CISS and factors.  This
pins the oracle to the reference itself; the engine is pinned to the oracle
in test_gpu_parity.py.

Inputs keep nnz % 32 == 0 for ALS/CCD (no inactive-lane reads) and
nnz % 32 != 0 for SGD (the reference SGD loops forever on a terminator-only
tile, sgpu/sgd.cu:48-50; the harness refuses that case)."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import max_factor_rel

pytestmark = pytest.mark.gpu

_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)


def _lib(name):
    path = os.path.join(po.REF_DIR, f"libref_{name}.so")
    if not os.path.exists(path):
        pytest.skip(f"{path} not built")
    L = C.CDLL(path)
    L.refh_rank.restype = C.c_int
    return L


def _tensor(nnz, dims, seed):
    rng = np.random.default_rng(seed)
    ind = np.stack([rng.integers(1, d + 1, nnz) for d in dims]).astype(np.uint64)
    vals = rng.uniform(1.0, 5.0, nnz)
    return po.Tensor(ind, vals, list(dims))


def _factors(dims, R, seed):
    rng = np.random.default_rng(seed)
    return [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]


def _p(a):
    return a.ctypes.data_as(_f64p)


def _u(a):
    return a.ctypes.data_as(_u64p)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reference_als_kernel(mode):
    L = _lib("als")
    R = L.refh_rank()
    T = _tensor(32 * 150, (80, 60, 40), 1)
    Ts = T.sorted_for_mode(mode)
    c = po.ciss_build(Ts, mode, 32)
    U = _factors(T.dims, R, 2)
    m1, m2 = (mode + 1) % 3, (mode + 2) % 3
    # reference kernels
    ft = U[mode].copy()
    dims3 = np.array(T.dims, dtype=np.uint64)
    L.refh_als_mode.argtypes = [_f64p, C.c_uint64, _u64p, C.c_uint64, C.c_uint64, _u64p, _f64p,
                                C.c_uint64, _f64p, C.c_uint64, _f64p, C.c_uint64, C.c_double]
    rc = L.refh_als_mode(_p(c["entries"]), c["size_rows"], _u(c["directory"]), c["dlength"], T.nnz, _u(dims3),
                         _p(ft), T.dims[mode], _p(U[m1]), T.dims[m1], _p(U[m2]), T.dims[m2], 10.0)
    assert rc == 0
    # oracle compat restatement
    w = po.compat_weights(Ts, mode, 0)
    Uo = [u.copy() for u in U]
    po.als_mode(Ts, mode, Uo, 10.0, w, trunc=True)
    assert max_factor_rel([ft], [Uo[mode]]) < 1e-9


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reference_ccd_kernel(mode):
    L = _lib("ccd")
    R = L.refh_rank()
    # enough tiles that the reference grid (tilenum/256+1 blocks of 8 warps)
    # leaves most of them out
    T = _tensor(32 * 600, (300, 200, 100), 3)
    Ts = T.sorted_for_mode(mode)
    c = po.ciss_build(Ts, mode, 32)
    U = _factors(T.dims, R, 4)
    m1, m2 = (mode + 1) % 3, (mode + 2) % 3
    ft = U[mode].copy()
    dims3 = np.array(T.dims, dtype=np.uint64)
    L.refh_ccd_mode.argtypes = [_f64p, C.c_uint64, _u64p, C.c_uint64, C.c_uint64, _u64p, _f64p,
                                C.c_uint64, _f64p, C.c_uint64, _f64p, C.c_uint64, C.c_double]
    rc = L.refh_ccd_mode(_p(c["entries"]), c["size_rows"], _u(c["directory"]), c["dlength"], T.nnz, _u(dims3),
                         _p(ft), T.dims[mode], _p(U[m1]), T.dims[m1], _p(U[m2]), T.dims[m2], 100.0)
    assert rc == 0
    w = po.compat_weights(Ts, mode, 1)
    assert (w == 0).mean() > 0.5  # most tiles are outside the reference grid
    Uo = [u.copy() for u in U]
    po.ccd_compat_mode(Ts, mode, Uo, 100.0, w, trunc=True)
    assert max_factor_rel([ft], [Uo[mode]]) < 1e-9


def test_reference_sgd_kernel():
    L = _lib("sgd")
    R = L.refh_rank()
    T = _tensor(32 * 200 + 7, (90, 70, 50), 5)
    Ts = T.sorted_for_mode(0)
    c = po.ciss_build(Ts, 0, 32)
    U = _factors(T.dims, R, 6)
    fa, fb, fc = (u.copy() for u in U)
    dims3 = np.array(T.dims, dtype=np.uint64)
    L.refh_sgd_epoch.argtypes = [_f64p, C.c_uint64, _u64p, _u64p, C.c_uint64, C.c_uint64, _u64p, _f64p,
                                 C.c_uint64, _f64p, C.c_uint64, _f64p, C.c_uint64, C.c_double, C.c_double]
    rc = L.refh_sgd_epoch(_p(c["entries"]), c["size_rows"], _u(c["directory"]), _u(c["dcounter"]),
                          c["dlength"], T.nnz, _u(dims3), _p(fa), T.dims[0], _p(fb), T.dims[1], _p(fc),
                          T.dims[2], 1e-3, 1e-3)
    assert rc == 0
    # reference constants: lr 1e-3, lambda 1e-3, step scale 1e-5; the
    # kernel's Hogwild order differs from the oracle's sequential order only
    # at rounding level for steps this small
    Uo = [u.copy() for u in U]
    po.sgd_epoch(Ts, Uo, 1e-3, 1e-3, 1e-5, trunc=True)
    changed = max(np.max(np.abs(a - b)) for a, b in zip(Uo, U))
    assert changed > 0
    assert max_factor_rel([fa, fb, fc], Uo) < 1e-9


def test_reference_sgd_refuses_terminator_only_tile():
    L = _lib("sgd")
    R = L.refh_rank()
    T = _tensor(32 * 10, (20, 20, 20), 7)
    c = po.ciss_build(T.sorted_for_mode(0), 0, 32)
    U = _factors(T.dims, R, 8)
    dims3 = np.array(T.dims, dtype=np.uint64)
    L.refh_sgd_epoch.argtypes = [_f64p, C.c_uint64, _u64p, _u64p, C.c_uint64, C.c_uint64, _u64p, _f64p,
                                 C.c_uint64, _f64p, C.c_uint64, _f64p, C.c_uint64, C.c_double, C.c_double]
    rc = L.refh_sgd_epoch(_p(c["entries"]), c["size_rows"], _u(c["directory"]), _u(c["dcounter"]),
                          c["dlength"], T.nnz, _u(dims3), _p(U[0]), 20, _p(U[1]), 20, _p(U[2]), 20, 1e-3, 1e-3)
    assert rc == -10
