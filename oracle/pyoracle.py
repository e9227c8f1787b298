"""ctypes front end of the FP64 CPU oracle (oracle/liboracle.so) and of the
reference's own host code built from its sources (oracle/_ref/).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, never by the engine in cutc_b200/.

Tensors are held as numpy arrays: ``ind`` (nmodes x nnz, uint64, indices as
read -- 1-based) and ``vals`` (float64); factors are lists of row-major
float64 arrays (dims[m] x R).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)


class _OrcTensor(C.Structure):
    _fields_ = [("nmodes", C.c_int), ("nnz", C.c_uint64), ("dims", C.c_uint64 * 4),
                ("ind", _u64p * 4), ("vals", _f64p)]


class _OrcCiss(C.Structure):
    _fields_ = [("nnz", C.c_uint64), ("dlength", C.c_uint64), ("size_rows", C.c_uint64),
                ("tile_len", C.c_uint64), ("directory", _u64p), ("dcounter", _u64p),
                ("entries", _f64p), ("written", C.POINTER(C.c_uint8))]


def build():
    """Compile liboracle.so (and the reference libraries when the reference
    tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    subprocess.run(["sh", os.path.join(HERE, "build_ref.sh")], check=True,
                   stdout=subprocess.DEVNULL)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(path)
        L.orc_tns_read.argtypes = [C.c_char_p, C.POINTER(_OrcTensor)]
        L.orc_tensor_free.argtypes = [C.POINTER(_OrcTensor)]
        L.orc_ciss_build.argtypes = [C.POINTER(_OrcTensor), C.c_int, C.c_int, C.POINTER(_OrcCiss)]
        L.orc_ciss_build_ga.argtypes = [C.POINTER(_OrcTensor), C.c_int, C.c_int, C.POINTER(_OrcCiss)]
        L.orc_ciss_free.argtypes = [C.POINTER(_OrcCiss)]
        L.orc_ref_value_trunc.argtypes = [C.c_double]
        L.orc_ref_value_trunc.restype = C.c_double
        L.orc_compat_weights.argtypes = [C.POINTER(_OrcCiss), C.c_int, _f64p]
        L.orc_sq_loss.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int]
        L.orc_sq_loss.restype = C.c_double
        L.orc_sq_loss_omp.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int, C.c_int]
        L.orc_sq_loss_omp.restype = C.c_double
        L.orc_frob.argtypes = [C.c_int, _u64p, C.POINTER(_f64p), C.c_int, C.c_double]
        L.orc_frob.restype = C.c_double
        L.orc_als_mode.argtypes = [C.POINTER(_OrcTensor), C.c_int, C.POINTER(_f64p), C.c_int,
                                   C.c_double, _f64p, C.c_int]
        L.orc_als_mode_omp.argtypes = [C.POINTER(_OrcTensor), C.c_int, C.POINTER(_f64p), C.c_int,
                                       C.c_double, C.c_int]
        L.orc_ccd_compat_mode.argtypes = [C.POINTER(_OrcTensor), C.c_int, C.POINTER(_f64p),
                                          C.c_int, C.c_double, _f64p, C.c_int]
        L.orc_ccdpp_outer.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int,
                                      C.c_double, C.c_int, _f64p]
        L.orc_ccdpp_outer_omp.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int,
                                          C.c_double, C.c_int, _f64p, C.c_int]
        L.orc_residual.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int, _f64p]
        L.orc_sgd_epoch.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int, C.c_double,
                                    C.c_double, C.c_double, C.c_int]
        L.orc_sgd_epoch_hogwild.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int,
                                            C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_grad.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int, C.c_double,
                               C.POINTER(_f64p)]
        L.orc_objective.argtypes = [C.POINTER(_OrcTensor), C.POINTER(_f64p), C.c_int, C.c_double]
        L.orc_objective.restype = C.c_double
        _lib = L
    return _lib


class Tensor:
    """COO tensor: ind (nmodes x nnz uint64, as read) and vals (float64)."""

    def __init__(self, ind, vals, dims=None):
        self.ind = np.ascontiguousarray(np.asarray(ind, dtype=np.uint64))
        self.vals = np.ascontiguousarray(np.asarray(vals, dtype=np.float64))
        self.nmodes, self.nnz = self.ind.shape
        if dims is None:
            dims = [int(self.ind[m].max()) if self.nnz else 0 for m in range(self.nmodes)]
        self.dims = [int(d) for d in dims]
        self._c = None

    def c(self):
        if self._c is None:
            t = _OrcTensor()
            t.nmodes = self.nmodes
            t.nnz = self.nnz
            for m in range(self.nmodes):
                t.dims[m] = self.dims[m]
                t.ind[m] = self.ind[m].ctypes.data_as(_u64p)
            t.vals = self.vals.ctypes.data_as(_f64p)
            self._c = t
        return self._c

    def sorted_for_mode(self, m):
        """Stable sort by (ind[m], ind[(m+1)%3]), as software/scripts/stensor.py:36-43."""
        n = self.nmodes
        order = np.lexsort((self.ind[(m + 1) % n], self.ind[m]))
        return Tensor(self.ind[:, order], self.vals[order], self.dims)


def _mats(U):
    arr = (_f64p * len(U))()
    for m, u in enumerate(U):
        assert u.dtype == np.float64 and u.flags.c_contiguous
        arr[m] = u.ctypes.data_as(_f64p)
    return arr


def tns_read(path):
    t = _OrcTensor()
    rc = lib().orc_tns_read(path.encode(), C.byref(t))
    if rc:
        raise OSError(f"orc_tns_read({path}) = {rc}")
    nm, nnz = t.nmodes, t.nnz
    ind = np.stack([np.ctypeslib.as_array(t.ind[m], (nnz,)).copy() for m in range(nm)])
    vals = np.ctypeslib.as_array(t.vals, (nnz,)).copy()
    dims = [t.dims[m] for m in range(nm)]
    lib().orc_tensor_free(C.byref(t))
    return Tensor(ind, vals, dims)


def ciss_build(T: Tensor, mode0: int, tile_len: int = 32, ga: bool = False):
    c = _OrcCiss()
    fn = lib().orc_ciss_build_ga if ga else lib().orc_ciss_build
    rc = fn(T.c(), mode0, tile_len, C.byref(c))
    if rc:
        raise ValueError(f"orc_ciss_build = {rc}")
    out = dict(
        nnz=c.nnz, dlength=c.dlength, size_rows=c.size_rows, tile_len=c.tile_len,
        directory=np.ctypeslib.as_array(c.directory, (c.dlength,)).copy(),
        dcounter=np.ctypeslib.as_array(c.dcounter, (c.dlength + 1,)).copy(),
        entries=np.ctypeslib.as_array(c.entries, (c.size_rows * 3,)).copy(),
        written=np.ctypeslib.as_array(c.written, (c.size_rows * 3,)).copy().astype(bool),
    )
    lib().orc_ciss_free(C.byref(c))
    return out


def compat_weights(T_sorted: Tensor, mode0: int, kernel: int):
    """Per-nonzero multiplicity of the reference ALS (kernel=0) / CCD (1) kernels."""
    c = _OrcCiss()
    rc = lib().orc_ciss_build(T_sorted.c(), mode0, 32, C.byref(c))
    if rc:
        raise ValueError(f"orc_ciss_build = {rc}")
    w = np.zeros(T_sorted.nnz, dtype=np.float64)
    rc = lib().orc_compat_weights(C.byref(c), kernel, w.ctypes.data_as(_f64p))
    lib().orc_ciss_free(C.byref(c))
    if rc:
        raise ValueError("compat weights need nnz % 32 == 0")
    return w


def value_trunc(v):
    f = lib().orc_ref_value_trunc
    return np.array([f(float(x)) for x in np.ravel(v)]).reshape(np.shape(v))


def sq_loss(T: Tensor, U, nthreads=1):
    R = U[0].shape[1]
    if nthreads > 1:
        return lib().orc_sq_loss_omp(T.c(), _mats(U), R, nthreads)
    return lib().orc_sq_loss(T.c(), _mats(U), R)


def rmse(T: Tensor, U, nthreads=1):
    return float(np.sqrt(sq_loss(T, U, nthreads) / T.nnz))


def frob(dims, U, lam):
    R = U[0].shape[1]
    d = (C.c_uint64 * len(dims))(*dims)
    return lib().orc_frob(len(dims), d, _mats(U), R, lam)


def als_mode(T_sorted: Tensor, m: int, U, lam: float, w=None, trunc=False, nthreads=1):
    R = U[0].shape[1]
    if nthreads > 1 and w is None and not trunc:
        return lib().orc_als_mode_omp(T_sorted.c(), m, _mats(U), R, lam, nthreads)
    wp = None if w is None else np.ascontiguousarray(w, dtype=np.float64).ctypes.data_as(_f64p)
    return lib().orc_als_mode(T_sorted.c(), m, _mats(U), R, lam, wp, int(trunc))


def ccd_compat_mode(T_sorted: Tensor, m: int, U, lam: float, w=None, trunc=False):
    R = U[0].shape[1]
    wp = None if w is None else np.ascontiguousarray(w, dtype=np.float64).ctypes.data_as(_f64p)
    lib().orc_ccd_compat_mode(T_sorted.c(), m, _mats(U), R, lam, wp, int(trunc))


def residual(T: Tensor, U):
    r = np.zeros(T.nnz, dtype=np.float64)
    lib().orc_residual(T.c(), _mats(U), U[0].shape[1], r.ctypes.data_as(_f64p))
    return r


def ccdpp_outer(T: Tensor, U, lam: float, inner: int, resid, nthreads=1):
    R = U[0].shape[1]
    if nthreads > 1:
        lib().orc_ccdpp_outer_omp(T.c(), _mats(U), R, lam, inner,
                                  resid.ctypes.data_as(_f64p), nthreads)
    else:
        lib().orc_ccdpp_outer(T.c(), _mats(U), R, lam, inner, resid.ctypes.data_as(_f64p))


def sgd_epoch(T_sorted: Tensor, U, lr, lam, scale=1.0, trunc=False):
    lib().orc_sgd_epoch(T_sorted.c(), _mats(U), U[0].shape[1], lr, lam, scale, int(trunc))


def sgd_epoch_hogwild(T: Tensor, U, lr, lam, scale=1.0, nthreads=1):
    lib().orc_sgd_epoch_hogwild(T.c(), _mats(U), U[0].shape[1], lr, lam, scale, nthreads)


def grad(T: Tensor, U, lam):
    G = [np.zeros_like(u) for u in U]
    lib().orc_grad(T.c(), _mats(U), U[0].shape[1], lam, _mats(G))
    return G


def objective(T: Tensor, U, lam):
    return lib().orc_objective(T.c(), _mats(U), U[0].shape[1], lam)


# ---------------------------------------------------------------------------
# The reference's own host code (oracle/_ref/libref_host.so)
# ---------------------------------------------------------------------------

class _RefSptensor(C.Structure):
    _fields_ = [("nmodes", C.c_uint64), ("nnz", C.c_uint64), ("dims", _u64p),
                ("ind", C.POINTER(_u64p)), ("vals", _f64p)]


class _RefCiss(C.Structure):
    _fields_ = [("nmodes", C.c_uint64), ("nnz", C.c_uint64), ("size", C.c_uint64),
                ("dlength", C.c_uint64), ("dims", _u64p), ("directory", _u64p),
                ("dcounter", _u64p), ("entries", _f64p)]


_ref = None


def ref_host_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_host.so"))


def ref_host():
    global _ref
    if _ref is None:
        L = C.CDLL(os.path.join(REF_DIR, "libref_host.so"))
        L.tt_read.argtypes = [C.c_char_p]
        L.tt_read.restype = C.POINTER(_RefSptensor)
        L.tt_free.argtypes = [C.POINTER(_RefSptensor)]
        L.ciss_alloc.argtypes = [C.POINTER(_RefSptensor), C.c_uint64]
        L.ciss_alloc.restype = C.POINTER(_RefCiss)
        L.tt_write_binary.argtypes = [C.POINTER(_RefSptensor), C.c_char_p]
        L.tt_write_binary.restype = None
        _ref = L
    return _ref


def ref_tt_read(path):
    """sgpu/sptensor.c:64 tt_read, run from the reference's own code."""
    p = ref_host().tt_read(path.encode())
    if not p:
        raise OSError(path)
    t = p.contents
    nm, nnz = t.nmodes, t.nnz
    ind = np.stack([np.ctypeslib.as_array(t.ind[m], (nnz,)).copy() for m in range(nm)])
    vals = np.ctypeslib.as_array(t.vals, (nnz,)).copy()
    dims = [t.dims[m] for m in range(nm)]
    ref_host().tt_free(p)
    return Tensor(ind, vals, dims)


def ref_tns_to_bin(tns_path, bin_path):
    """sgpu/sptensor.c:64 tt_read of a .tns file, then sgpu/io.c:347
    tt_write_binary of the result, both run from the reference's own code."""
    p = ref_host().tt_read(tns_path.encode())
    if not p:
        raise OSError(tns_path)
    ref_host().tt_write_binary(p, bin_path.encode())
    ref_host().tt_free(p)


def ref_ciss_alloc(T: Tensor, mode1: int):
    """sgpu/ciss.c:68 ciss_alloc (mode 1-based), run from the reference's own
    code.  The reference leaks the result; the copy returned here is what
    the tests compare."""
    st = _RefSptensor()
    st.nmodes = T.nmodes
    st.nnz = T.nnz
    dims = (C.c_uint64 * T.nmodes)(*T.dims)
    st.dims = dims
    ptrs = (_u64p * T.nmodes)(*[T.ind[m].ctypes.data_as(_u64p) for m in range(T.nmodes)])
    st.ind = ptrs
    st.vals = T.vals.ctypes.data_as(_f64p)
    c = ref_host().ciss_alloc(C.byref(st), mode1).contents
    return dict(
        nnz=c.nnz, dlength=c.dlength, size_rows=c.size,
        directory=np.ctypeslib.as_array(c.directory, (c.dlength,)).copy(),
        dcounter=np.ctypeslib.as_array(c.dcounter, (c.dlength + 1,)).copy(),
        entries=np.ctypeslib.as_array(c.entries, (c.size * 3,)).copy(),
    )


def write_tns(path, T: Tensor, fmt="%.17g"):
    """Write a 1-based .tns text file ("i j k v" per line)."""
    with open(path, "w") as f:
        cols = [T.ind[m] for m in range(T.nmodes)]
        for n in range(T.nnz):
            f.write(" ".join(str(int(c[n])) for c in cols) + " " + (fmt % T.vals[n]) + "\n")


# ---------------------------------------------------------------------------
# Masked CP loss of any order in FP64 (numpy): the checker of the adjoint
# kernel at order 4 (the C restatement, orc_grad / orc_objective, is order 3).
# f = 1/2 sum_Omega (x - sum_r prod_m U_m(i_m, r))^2 + lam sum_m ||U_m||^2
# ---------------------------------------------------------------------------
def cp_objective(ind, vals, U, lam):
    P = np.ones((ind.shape[1], U[0].shape[1]))
    for m, u in enumerate(U):
        P *= u[ind[m].astype(np.int64) - 1]
    e = vals - P.sum(1)
    return 0.5 * float(e @ e) + lam * sum(float((u * u).sum()) for u in U)


def cp_grad(ind, vals, U, lam):
    idx = [ind[m].astype(np.int64) - 1 for m in range(len(U))]
    rows = [u[i] for u, i in zip(U, idx)]
    P = np.ones_like(rows[0])
    for r in rows:
        P = P * r
    e = vals - P.sum(1)
    G = []
    for m, u in enumerate(U):
        others = np.ones_like(rows[0])
        for n, r in enumerate(rows):
            if n != m:
                others = others * r
        g = 2.0 * lam * u
        np.add.at(g, idx[m], -e[:, None] * others)
        G.append(g)
    return G


# ---------------------------------------------------------------------------
# tc_converge bookkeeping (sgpu/completion.c:296-362), called after every
# epoch from the first (sgpu/als.cu:803-806): the convergence RMSE is the
# validation RMSE when a validation tensor is given (:318-324), else the
# training RMSE; an improvement by more than the tolerance (TOLERANCE 1e-4,
# sgpu/base.h:32) resets the bad-epoch count and saves the model as the best
# (:330-338); otherwise the count grows and reaching MAX_BADEPOCHS (3,
# base.h:36) converges (:339-345).  best_rmse starts at BEST_RMSE (1e7,
# base.h:35).
# ---------------------------------------------------------------------------
class Converge:
    def __init__(self, tolerance=1e-4, max_bad=3):
        self.tolerance = tolerance
        self.max_bad = max_bad
        self.best_rmse = 10000000.0
        self.nbad = 0
        self.best_epoch = 0

    def step(self, epoch, rmse):
        """Returns (improved, converged)."""
        if rmse - self.best_rmse < -self.tolerance:
            self.nbad = 0
            self.best_rmse = rmse
            self.best_epoch = epoch
            return True, False
        self.nbad += 1
        return False, self.nbad == self.max_bad
