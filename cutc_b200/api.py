"""ctypes bindings of libctc.so (include/ctc.h) and a host-side mirror of the
reference's single-GPU driver interface.

The reference entry points and their counterparts here:

    tt_read(path)                       sgpu/sptensor.c:64      -> tt_read
    ciss_alloc(t, mode)                 sgpu/ciss.c:68          -> ciss_alloc
    cissbasic_alloc(..., tile_len)      ga/ciss.c:69            -> ciss_alloc(tile_len=)
    tc_als / tc_sgd / tc_ccd            sgpu/als.cuh:20, sgd.cuh:18, ccd.cuh:20
    tc_main_ciss(a, b, c, val, te, alg) sgpu/completion.c:422   -> tc_main_ciss
    tc_rmse(test, mats)                 sgpu/completion.c:123   -> rmse

Every call goes through the CUDA library; there is no CPU fallback.  The
library must have been built (python -m cutc_b200.build).
"""
from __future__ import annotations

import ctypes as C
import weakref
import os
from dataclasses import dataclass, field

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libctc.so")

ALS, SGD, CCD, CCDPP = 0, 1, 2, 3
PREC_F32, PREC_F64, PREC_MIXED = 0, 1, 2
LR_BOLD_DRIVER, LR_EXP_DECAY, LR_CONSTANT = 0, 1, 2
SGD_HOGWILD, SGD_SEQUENTIAL = 0, 1
ALG_NAMES = {"als": ALS, "sgd": SGD, "ccd": CCD, "ccdpp": CCDPP}

_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)


class CtcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ctc error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("alg", C.c_int), ("rank", C.c_int), ("lambda_", C.c_double), ("lr", C.c_double),
                ("lr_scale", C.c_double), ("lr_schedule", C.c_int), ("lr_decay", C.c_double),
                ("iters", C.c_int), ("inner", C.c_int), ("tile_len", C.c_int),
                ("threads_per_block", C.c_int), ("precision", C.c_int), ("compat", C.c_int),
                ("early_stop", C.c_int), ("tolerance", C.c_double), ("max_bad_epochs", C.c_int),
                ("mode_start", C.c_int), ("sgd_order", C.c_int), ("sgd_atomic", C.c_int),
                ("eval_every", C.c_int), ("use_graph", C.c_int), ("seed", C.c_uint64),
                ("sgd_groups", C.c_int), ("sgd_conflicts", C.c_int), ("threads_per_row", C.c_int),
                ("smem_budget", C.c_int)]


class EpochStats(C.Structure):
    _fields_ = [("epoch", C.c_int), ("loss", C.c_double), ("frob", C.c_double),
                ("rmse_tr", C.c_double), ("rmse_vl", C.c_double), ("rmse_te", C.c_double),
                ("ms_epoch", C.c_double), ("lr", C.c_double)]


class Result(C.Structure):
    _fields_ = [("epochs_run", C.c_int), ("best_epoch", C.c_int), ("best_rmse", C.c_double),
                ("final_rmse_tr", C.c_double), ("final_rmse_vl", C.c_double),
                ("final_rmse_te", C.c_double), ("total_ms", C.c_double),
                ("nonspd_rows", C.c_uint64)]


class FoParams(C.Structure):
    _fields_ = [("rank", C.c_int), ("precision", C.c_int), ("lambda_", C.c_double), ("lr", C.c_double),
                ("beta1", C.c_double), ("beta2", C.c_double), ("eps", C.c_double), ("batch", C.c_uint64),
                ("epochs", C.c_int), ("seed", C.c_uint64), ("eval_every", C.c_int)]


class TuneTrial(C.Structure):
    _fields_ = [("tile_len", C.c_int), ("threads_per_row", C.c_int), ("smem_budget", C.c_int),
                ("ms_epoch", C.c_double), ("cached", C.c_int), ("sgd_atomic", C.c_int),
                ("threads_per_block", C.c_int)]


TUNE_FORCE, TUNE_NO_WRITE = 1, 2
EPOCH_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(EpochStats))
BATCH_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                       C.c_double)

_lib = None


def lib():
    """Load libctc.so (fails loudly when the CUDA library is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cutc_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sig = {
            "ctc_last_error": (C.c_char_p, []),
            "ctc_version": (C.c_char_p, []),
            "ctc_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
            "ctc_ctx_destroy": (C.c_int, [P]),
            "ctc_ctx_kernel_launches": (C.c_int, [P, _u64p]),
            "ctc_ctx_stream": (P, [P]),
            "ctc_tensor_load_tns": (C.c_int, [C.c_char_p, C.POINTER(P)]),
            "ctc_tensor_save_bin": (C.c_int, [P, C.c_char_p]),
            "ctc_tensor_save_splatt": (C.c_int, [P, C.c_char_p]),
            "ctc_tensor_write_tns": (C.c_int, [P, C.c_char_p, C.c_int]),
            "ctc_tensor_split": (C.c_int, [P, C.c_uint64, C.POINTER(P), C.POINTER(P), C.POINTER(P)]),
            "ctc_tensor_from_coo": (C.c_int, [C.c_int, C.c_uint64, _u64p, C.POINTER(_u64p), _f64p, C.POINTER(P)]),
            "ctc_tensor_info": (C.c_int, [P, C.POINTER(C.c_int), _u64p, _u64p]),
            "ctc_tensor_export": (C.c_int, [P, C.POINTER(_u64p), _f64p]),
            "ctc_tensor_sort": (C.c_int, [P, C.c_int]),
            "ctc_tensor_free": (C.c_int, [P]),
            "ctc_ciss_build": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(P)]),
            "ctc_ciss_build_ga": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(P)]),
            "ctc_ciss_build_gpu": (C.c_int, [P, P, C.c_int, C.c_int, C.c_int, C.POINTER(P)]),
            "ctc_dataset_dims": (C.c_int, [P, _u64p]),
            "ctc_dataset_set_model": (C.c_int, [P, P]),
            "ctc_dataset_epochs": (C.c_int, [P, C.c_int]),
            "ctc_dataset_set_lr": (C.c_int, [P, C.c_double]),
            "ctc_dataset_evaluate": (C.c_int, [P, C.POINTER(EpochStats)]),
            "ctc_dataset_get_model": (C.c_int, [P, P]),
            "ctc_dataset_probe_wait": (C.c_int, [P, C.c_uint64]),
            "ctc_ctx_set_profiling": (C.c_int, [P, C.c_int]),
            "ctc_ctx_kernel_time": (C.c_int, [P, C.c_char_p, _u64p, _f64p]),
            "ctc_ctx_reset_kernel_times": (C.c_int, [P]),
            "ctc_ciss_sizes": (C.c_int, [P, _u64p, _u64p, _u64p, C.POINTER(C.c_int)]),
            "ctc_ciss_export": (C.c_int, [P, _u64p, _u64p, _f64p, C.POINTER(C.c_uint8)]),
            "ctc_ciss_free": (C.c_int, [P]),
            "ctc_plan_tiles": (C.c_int, [_u64p, C.c_uint64, C.c_uint32, C.c_int, C.POINTER(C.c_int32), C.c_uint64,
                                         _u64p, C.POINTER(C.c_uint32), C.c_uint64, _u64p]),
            "ctc_model_create": (C.c_int, [C.c_int, _u64p, C.c_int, C.POINTER(P)]),
            "ctc_model_init_uniform": (C.c_int, [P, C.c_uint64, C.c_double]),
            "ctc_model_set": (C.c_int, [P, C.c_int, _f64p]),
            "ctc_model_get": (C.c_int, [P, C.c_int, _f64p]),
            "ctc_model_copy": (C.c_int, [P, P]),
            "ctc_model_info": (C.c_int, [P, C.POINTER(C.c_int), _u64p, C.POINTER(C.c_int)]),
            "ctc_model_free": (C.c_int, [P]),
            "ctc_model_write_text": (C.c_int, [P, C.c_int, C.c_char_p]),
            "ctc_model_save": (C.c_int, [P, C.c_char_p]),
            "ctc_model_load": (C.c_int, [C.c_char_p, C.POINTER(P)]),
            "ctc_params_default": (C.c_int, [C.c_int, C.POINTER(Params)]),
            "ctc_params_check": (C.c_int, [C.POINTER(Params)]),
            "ctc_run": (C.c_int, [P, C.POINTER(P), P, P, P, P, C.POINTER(Params), EPOCH_CB, P,
                                  C.POINTER(Result)]),
            "ctc_dataset_create": (C.c_int, [P, C.POINTER(P), P, P, C.POINTER(Params), C.POINTER(P)]),
            "ctc_dataset_free": (C.c_int, [P]),
            "ctc_dataset_run": (C.c_int, [P, P, P, C.POINTER(Params), EPOCH_CB, P, C.POINTER(Result)]),
            "ctc_rmse": (C.c_int, [P, P, P, _f64p]),
            "ctc_grad": (C.c_int, [P, P, P, C.c_double, C.POINTER(_f64p), _f64p]),
            "ctc_sse_noalloc": (C.c_int, [P, C.c_uint64, P, P, P, C.c_int, P, P]),
            "ctc_batch_create": (C.c_int, [P, C.c_int, C.POINTER(P), C.POINTER(P), C.POINTER(Params),
                                           C.POINTER(P)]),
            "ctc_batch_free": (C.c_int, [P]),
            "ctc_autotune": (C.c_int, [P, C.POINTER(P), C.POINTER(Params), C.c_char_p, C.c_int, C.POINTER(Params),
                                       C.POINTER(TuneTrial), C.c_int, C.POINTER(C.c_int)]),
            "ctc_tune_lookup": (C.c_int, [C.c_char_p, P, C.POINTER(Params), C.c_int, C.POINTER(Params)]),
            "ctc_tune_key": (C.c_int, [P, C.POINTER(Params), C.c_int, C.c_char_p, C.c_int]),
            "ctc_fo_params_default": (C.c_int, [C.POINTER(FoParams)]),
            "ctc_fo_create": (C.c_int, [P, P, P, C.POINTER(FoParams), C.POINTER(P)]),
            "ctc_fo_free": (C.c_int, [P]),
            "ctc_fo_dims": (C.c_int, [P, C.POINTER(C.c_int), _u64p]),
            "ctc_fo_run": (C.c_int, [P, P, C.POINTER(FoParams), EPOCH_CB, P, C.POINTER(Result)]),
            "ctc_fo_grad": (C.c_int, [P, P, C.POINTER(_f64p), _f64p]),
            "ctc_batch_info": (C.c_int, [P, C.POINTER(C.c_int), _u64p, _u64p]),
            "ctc_batch_run": (C.c_int, [P, C.POINTER(P), C.POINTER(Params), BATCH_CB, P, C.POINTER(Result)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise CtcError(rc, lib().ctc_last_error().decode(errors="replace"))


def exported_symbols():
    """Names declared in include/ctc.h that the loaded library resolves."""
    L = lib()
    return [n for n in _declared_names() if hasattr(L, n)]


def _declared_names():
    import re
    hdr = os.path.join(os.path.dirname(_PKG), "include", "ctc.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"\b(ctc_[a-z0-9_]+)\s*\(", txt)))


# ---------------------------------------------------------------------------
class Context:
    """One CUDA device + stream (ctc_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().ctc_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device
        self._deps = weakref.WeakSet()  # datasets, batches, first-order states on this context

    def _track(self, obj):
        self._deps.add(obj)

    def launches(self) -> int:
        n = C.c_uint64()
        _check(lib().ctc_ctx_kernel_launches(self.h, C.byref(n)))
        return n.value

    def stream(self):
        return lib().ctc_ctx_stream(self.h)

    def set_profiling(self, on: bool):
        _check(lib().ctc_ctx_set_profiling(self.h, int(on)))

    def kernel_time(self, name: str):
        """(launch count, total device ms) of kernels whose name contains `name`."""
        n = C.c_uint64()
        ms = C.c_double()
        _check(lib().ctc_ctx_kernel_time(self.h, name.encode(), C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def reset_kernel_times(self):
        _check(lib().ctc_ctx_reset_kernel_times(self.h))

    def close(self):
        """Frees every object still living on this context, then the context."""
        if self.h:
            for d in list(self._deps):
                try:
                    d.free()
                except Exception:
                    pass
            lib().ctc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tensor:
    """Host COO tensor (ctc_tensor): indices kept as read (1-based)."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def from_coo(cls, ind, vals, dims=None):
        ind = np.ascontiguousarray(np.asarray(ind, dtype=np.uint64))
        vals = np.ascontiguousarray(np.asarray(vals, dtype=np.float64))
        nm, nnz = ind.shape
        ptrs = (_u64p * nm)(*[ind[m].ctypes.data_as(_u64p) for m in range(nm)])
        d = None if dims is None else (C.c_uint64 * nm)(*[int(x) for x in dims])
        h = C.c_void_p()
        _check(lib().ctc_tensor_from_coo(nm, nnz, d, ptrs, vals.ctypes.data_as(_f64p), C.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path: str):
        h = C.c_void_p()
        _check(lib().ctc_tensor_load_tns(path.encode(), C.byref(h)))
        return cls(h)

    def save_bin(self, path: str):
        _check(lib().ctc_tensor_save_bin(self.h, path.encode()))

    def save_splatt(self, path: str):
        """SPLATT binary coordinate file (the reference's .bin form)."""
        _check(lib().ctc_tensor_save_splatt(self.h, path.encode()))

    def write_tns(self, path: str, digits: int = -1):
        """Text .tns: indices as stored, values "%.<digits>f" (digits >= 0)
        or "%.17g" (digits < 0)."""
        _check(lib().ctc_tensor_write_tns(self.h, path.encode(), digits))

    def split(self, seed: int):
        """(train, test, validation) by tvtensor.py's seeded 80/10/10 rule
        (ctc_tensor_split)."""
        hs = [C.c_void_p(), C.c_void_p(), C.c_void_p()]
        _check(lib().ctc_tensor_split(self.h, seed, C.byref(hs[0]), C.byref(hs[1]), C.byref(hs[2])))
        return tuple(Tensor(h) for h in hs)

    def info(self):
        nm = C.c_int()
        nnz = C.c_uint64()
        dims = (C.c_uint64 * 4)()
        _check(lib().ctc_tensor_info(self.h, C.byref(nm), C.byref(nnz), dims))
        return nm.value, nnz.value, [dims[m] for m in range(nm.value)]

    @property
    def nnz(self):
        return self.info()[1]

    @property
    def dims(self):
        return self.info()[2]

    def export(self):
        nm, nnz, _ = self.info()
        ind = np.zeros((nm, nnz), dtype=np.uint64)
        vals = np.zeros(nnz, dtype=np.float64)
        ptrs = (_u64p * nm)(*[ind[m].ctypes.data_as(_u64p) for m in range(nm)])
        _check(lib().ctc_tensor_export(self.h, ptrs, vals.ctypes.data_as(_f64p)))
        return ind, vals

    def sort(self, mode: int):
        _check(lib().ctc_tensor_sort(self.h, mode))
        return self

    def free(self):
        if self.h:
            lib().ctc_tensor_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def plan_tiles(ind, tile_len: int, from_runs: bool = False):
    """Work tiles of a copy sorted for one mode (ind: that mode's 1-based
    indices): (tiles n x 4 int32 {first, length, heavy or -1, piece},
    heavy rows h x 4 uint32 {row, first tile, tiles, 0})."""
    ind = np.ascontiguousarray(np.asarray(ind, dtype=np.uint64))
    nt, nh = C.c_uint64(), C.c_uint64()
    _check(lib().ctc_plan_tiles(ind.ctypes.data_as(_u64p), ind.size, tile_len, int(from_runs), None, 0,
                                C.byref(nt), None, 0, C.byref(nh)))
    tiles = np.zeros((nt.value, 4), dtype=np.int32)
    heavy = np.zeros((nh.value, 4), dtype=np.uint32)
    _check(lib().ctc_plan_tiles(ind.ctypes.data_as(_u64p), ind.size, tile_len, int(from_runs),
                                tiles.ctypes.data_as(C.POINTER(C.c_int32)), nt.value, C.byref(nt),
                                heavy.ctypes.data_as(C.POINTER(C.c_uint32)), nh.value, C.byref(nh)))
    return tiles, heavy


def ciss_alloc(t: Tensor, mode: int, tile_len: int = 32, ga: bool = False):
    """CISS of `t` (sorted for `mode`, 1-based) as numpy arrays: sgpu/ciss.c:68
    (ga=False) or the GA builder's counters, ga/ciss.c:69 (ga=True)."""
    h = C.c_void_p()
    build = lib().ctc_ciss_build_ga if ga else lib().ctc_ciss_build
    _check(build(t.h, mode, tile_len, C.byref(h)))
    return _ciss_export(h)


CISS_GA, CISS_SORT = 1, 2


def ciss_alloc_gpu(ctx: Context, t: Tensor, mode: int, tile_len: int = 32, ga: bool = False,
                   sort: bool = False):
    """The same CISS built on the device (ctc_ciss_build_gpu); sort=True
    first sorts the nonzeros for `mode` on the device (stable by the mode
    index, then the next mode's)."""
    h = C.c_void_p()
    flags = (CISS_GA if ga else 0) | (CISS_SORT if sort else 0)
    _check(lib().ctc_ciss_build_gpu(ctx.h, t.h, mode, tile_len, flags, C.byref(h)))
    return _ciss_export(h)


def _ciss_export(h):
    try:
        nnz, dl, sz = C.c_uint64(), C.c_uint64(), C.c_uint64()
        tl = C.c_int()
        _check(lib().ctc_ciss_sizes(h, C.byref(nnz), C.byref(dl), C.byref(sz), C.byref(tl)))
        directory = np.zeros(dl.value, dtype=np.uint64)
        dcounter = np.zeros(dl.value + 1, dtype=np.uint64)
        entries = np.zeros(sz.value * 3, dtype=np.float64)
        written = np.zeros(sz.value * 3, dtype=np.uint8)
        _check(lib().ctc_ciss_export(h, directory.ctypes.data_as(_u64p), dcounter.ctypes.data_as(_u64p),
                                     entries.ctypes.data_as(_f64p),
                                     written.ctypes.data_as(C.POINTER(C.c_uint8))))
        return dict(nnz=nnz.value, dlength=dl.value, size_rows=sz.value, tile_len=tl.value,
                    directory=directory, dcounter=dcounter, entries=entries,
                    written=written.astype(bool))
    finally:
        lib().ctc_ciss_free(h)


class Model:
    """Factor matrices (ctc_model), row-major float64 on the host side."""

    def __init__(self, dims, rank: int):
        d = (C.c_uint64 * len(dims))(*[int(x) for x in dims])
        h = C.c_void_p()
        _check(lib().ctc_model_create(len(dims), d, rank, C.byref(h)))
        self.h = h
        self.dims = [int(x) for x in dims]
        self.rank = rank

    def init_uniform(self, seed: int, scale: float):
        _check(lib().ctc_model_init_uniform(self.h, seed, scale))
        return self

    def set(self, mode: int, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.dims[mode], self.rank)
        _check(lib().ctc_model_set(self.h, mode, U.ctypes.data_as(_f64p)))

    def get(self, mode: int):
        U = np.zeros((self.dims[mode], self.rank), dtype=np.float64)
        _check(lib().ctc_model_get(self.h, mode, U.ctypes.data_as(_f64p)))
        return U

    def factors(self):
        return [self.get(m) for m in range(len(self.dims))]

    def write_text(self, mode: int, path: str):
        """Factor `mode` in the reference's mat_write text form."""
        _check(lib().ctc_model_write_text(self.h, mode, path.encode()))

    def save(self, path: str):
        """Exact binary checkpoint of all factors."""
        _check(lib().ctc_model_save(self.h, path.encode()))

    @classmethod
    def load(cls, path: str) -> "Model":
        h = C.c_void_p()
        _check(lib().ctc_model_load(path.encode(), C.byref(h)))
        nm, r = C.c_int(), C.c_int()
        d = (C.c_uint64 * 4)()
        _check(lib().ctc_model_info(h, C.byref(nm), d, C.byref(r)))
        m = cls.__new__(cls)
        m.h = h
        m.dims = [d[k] for k in range(nm.value)]
        m.rank = r.value
        return m

    def set_factors(self, Us):
        for m, U in enumerate(Us):
            self.set(m, U)
        return self

    def free(self):
        if self.h:
            lib().ctc_model_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def params(alg, **kw) -> Params:
    """Reference-default parameters for `alg` (sgpu/base.h:19-64), overridden by kw."""
    if isinstance(alg, str):
        alg = ALG_NAMES[alg]
    p = Params()
    _check(lib().ctc_params_default(alg, C.byref(p)))
    for k, v in kw.items():
        if k == "lambda":
            k = "lambda_"
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


@dataclass
class RunOutput:
    result: dict
    epochs: list = field(default_factory=list)


def _stats_dict(s):
    return dict(epoch=s.epoch, loss=s.loss, frob=s.frob, rmse_tr=s.rmse_tr, rmse_vl=s.rmse_vl,
                rmse_te=s.rmse_te, ms_epoch=s.ms_epoch, lr=s.lr)


def _result_dict(r):
    return {k: getattr(r, k) for k, _ in Result._fields_}


def _train_ptrs(train):
    train = list(train) + [None] * (3 - len(train))
    return (C.c_void_p * 3)(*[t.h if t is not None else None for t in train[:3]])


def run(ctx: Context, train, val, test, model: Model, p: Params, best: Model | None = None,
        callback=None) -> RunOutput:
    """ctc_run: stage, iterate, evaluate, return (reference tc_als/tc_sgd/tc_ccd)."""
    out = RunOutput(result={})

    def _cb(_user, sp):
        d = _stats_dict(sp.contents)
        out.epochs.append(d)
        if callback is not None:
            return int(bool(callback(d)))
        return 0

    cb = EPOCH_CB(_cb)
    res = Result()
    _check(lib().ctc_run(ctx.h, _train_ptrs(train), val.h if val else None, test.h if test else None,
                         model.h, best.h if best else None, C.byref(p), cb, None, C.byref(res)))
    out.result = _result_dict(res)
    return out


class Dataset:
    """Device-resident staged tensors (ctc_dataset) for repeated runs."""

    def __init__(self, ctx: Context, train, val, test, p: Params):
        h = C.c_void_p()
        _check(lib().ctc_dataset_create(ctx.h, _train_ptrs(train), val.h if val else None,
                                        test.h if test else None, C.byref(p), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._track(self)

    def run(self, model: Model, p: Params, best: Model | None = None, callback=None) -> RunOutput:
        out = RunOutput(result={})

        def _cb(_user, sp):
            d = _stats_dict(sp.contents)
            out.epochs.append(d)
            return int(bool(callback(d))) if callback else 0

        cb = EPOCH_CB(_cb)
        res = Result()
        _check(lib().ctc_dataset_run(self.h, model.h, best.h if best else None, C.byref(p), cb, None,
                                     C.byref(res)))
        out.result = _result_dict(res)
        return out

    def dims(self):
        d = (C.c_uint64 * 3)()
        _check(lib().ctc_dataset_dims(self.h, d))
        return [d[m] for m in range(3)]

    def set_model(self, model: Model):
        _check(lib().ctc_dataset_set_model(self.h, model.h))

    def epochs(self, n: int = 1):
        """Enqueue n update epochs on the context stream (asynchronous)."""
        _check(lib().ctc_dataset_epochs(self.h, n))

    def set_lr(self, lr: float):
        _check(lib().ctc_dataset_set_lr(self.h, lr))

    def evaluate(self) -> dict:
        s = EpochStats()
        _check(lib().ctc_dataset_evaluate(self.h, C.byref(s)))
        return _stats_dict(s)

    def get_model(self, model: Model):
        _check(lib().ctc_dataset_get_model(self.h, model.h))
        return model

    def probe_wait(self, limit_ns: int):
        """Enqueue the bounded-wait self-test (ctc_dataset_probe_wait): its
        wait expires after limit_ns and the next evaluate raises CTC_E_TIMEOUT."""
        _check(lib().ctc_dataset_probe_wait(self.h, limit_ns))

    def free(self):
        if self.h:
            lib().ctc_dataset_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def rmse(ctx: Context, t: Tensor, model: Model) -> float:
    v = C.c_double()
    _check(lib().ctc_rmse(ctx.h, t.h, model.h, C.byref(v)))
    return v.value


def grad(ctx: Context, t: Tensor, model: Model, lam: float):
    """Adjoint of the masked CP loss: (grads per mode, objective)."""
    G = [np.zeros((d, model.rank), dtype=np.float64) for d in model.dims]
    ptrs = (_f64p * len(G))(*[g.ctypes.data_as(_f64p) for g in G])
    obj = C.c_double()
    _check(lib().ctc_grad(ctx.h, t.h, model.h, lam, ptrs, C.byref(obj)))
    return G, obj.value


# ---------------------------------------------------------------------------
# mirror of the reference driver names
# ---------------------------------------------------------------------------
def tt_read(path: str) -> Tensor:
    """sgpu/sptensor.c:64."""
    return Tensor.load(path)


def _progress_printer(d):
    # sgpu/completion.c:111-113 plus the test RMSE and the epoch time
    print("epoch:%d   loss: %0.5e   RMSE-tr: %0.5e   RMSE-vl: %0.5e   RMSE-te: %0.5e   ms: %.3f"
          % (d["epoch"], d["loss"], d["rmse_tr"], d["rmse_vl"], d["rmse_te"], d["ms_epoch"]))
    return 0


def _tc(alg, traina, trainb, trainc, validation, test, mats: Model, best_mats: Model | None,
        ctx=None, verbose=True, **kw):
    ctx = ctx or Context(0)
    p = params(alg, rank=mats.rank, **kw)
    return run(ctx, [traina, trainb, trainc], validation, test, mats, p, best=best_mats,
               callback=_progress_printer if verbose else None)


def tc_als(traina, trainb, trainc, validation, test, mats, best_mats=None, regularization_index=10.0,
           **kw):
    """sgpu/als.cuh:20 tc_als."""
    return _tc(ALS, traina, trainb, trainc, validation, test, mats, best_mats,
               **{"lambda": regularization_index, **kw})


def tc_sgd(traina, trainb, trainc, validation, test, mats, best_mats=None, regularization_index=1e-3,
           learning_rate=1e-3, **kw):
    """sgpu/sgd.cuh:18 tc_sgd."""
    return _tc(SGD, traina, trainb, trainc, validation, test, mats, best_mats,
               **{"lambda": regularization_index, "lr": learning_rate, **kw})


def tc_ccd(traina, trainb, trainc, validation, test, mats, best_mats=None, regularization_index=100.0,
           **kw):
    """sgpu/ccd.cuh:20 tc_ccd (the reference's all-column CCD+)."""
    return _tc(CCD, traina, trainb, trainc, validation, test, mats, best_mats,
               **{"lambda": regularization_index, **kw})


def tc_main_ciss(traina, trainb, trainc, validation, test, algorithm_index: int, rank=16, seed=0,
                 **kw):
    """sgpu/completion.c:422: allocate factors (seeded here), pick lambda by
    algorithm, run.  Returns (model, best_model, RunOutput)."""
    dims = [max(a, b) for a, b in zip(traina.dims, validation.dims if validation else traina.dims)]
    mats = Model(dims, rank).init_uniform(seed, 1.0 / np.sqrt(rank))
    best = Model(dims, rank)
    fn = {ALS: tc_als, SGD: tc_sgd, CCD: tc_ccd}.get(algorithm_index)
    if fn is None:
        out = _tc(CCDPP, traina, trainb, trainc, validation, test, mats, best, **kw)
    else:
        out = fn(traina, trainb, trainc, validation, test, mats, best, **kw)
    return mats, best, out


@dataclass
class BatchOutput:
    """Per-instance RMSE history of a batch run: epochs[k] = (epoch, ms_epoch,
    rmse_tr[ninst], rmse_te[ninst])."""
    result: dict
    epochs: list = field(default_factory=list)


class Batch:
    """Many independent completion problems trained together (ctc_batch):
    one block-diagonal stacked tensor, one launch per kernel and epoch."""

    def __init__(self, ctx: Context, train, test, p: Params):
        n = len(train)
        if test is not None and len(test) != n:
            raise ValueError("train and test lists differ in length")
        tr = (C.c_void_p * n)(*[t.h for t in train])
        te = (C.c_void_p * n)(*[t.h for t in test]) if test is not None else None
        h = C.c_void_p()
        _check(lib().ctc_batch_create(ctx.h, n, tr, te, C.byref(p), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._track(self)
        self.ninst = n

    def info(self):
        n = C.c_int()
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().ctc_batch_info(self.h, C.byref(n), C.byref(a), C.byref(b)))
        return n.value, a.value, b.value

    def run(self, models, p: Params, callback=None) -> BatchOutput:
        if len(models) != self.ninst:
            raise ValueError("one model per instance")
        out = BatchOutput(result={})

        def _cb(_user, epoch, n, rtr, rte, ms):
            tr = np.array(rtr[:n], dtype=np.float64)
            te = np.array(rte[:n], dtype=np.float64)
            out.epochs.append((epoch, ms, tr, te))
            return int(bool(callback(epoch, ms, tr, te))) if callback else 0

        cb = BATCH_CB(_cb)
        res = Result()
        hs = (C.c_void_p * self.ninst)(*[m.h for m in models])
        _check(lib().ctc_batch_run(self.h, hs, C.byref(p), cb, None, C.byref(res)))
        out.result = _result_dict(res)
        return out

    def free(self):
        if self.h:
            lib().ctc_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def autotune(ctx: Context, train, p: Params, cache_path: str | None = None, force: bool = False,
             write: bool = True):
    """ctc_autotune: tuned copy of `p` for the shape of train[0] and the
    list of timed trials (dicts)."""
    out = Params()
    trials = (TuneTrial * 64)()
    n = C.c_int()
    flags = (TUNE_FORCE if force else 0) | (0 if write else TUNE_NO_WRITE)
    _check(lib().ctc_autotune(ctx.h, _train_ptrs(train), C.byref(p), cache_path.encode() if cache_path else None,
                              flags, C.byref(out), trials, 64, C.byref(n)))
    return out, [{k: getattr(trials[i], k) for k, _ in TuneTrial._fields_} for i in range(min(n.value, 64))]


def tune_lookup(cache_path: str, train: Tensor, p: Params, sm_count: int = 148):
    """The cached tuned parameters for this shape, or None."""
    out = Params()
    rc = lib().ctc_tune_lookup(cache_path.encode(), train.h, C.byref(p), sm_count, C.byref(out))
    if rc == -9:
        return None
    _check(rc)
    return out


def tune_key(train: Tensor, p: Params, sm_count: int = 148) -> str:
    buf = C.create_string_buffer(512)
    _check(lib().ctc_tune_key(train.h, C.byref(p), sm_count, buf, 512))
    return buf.value.decode()


def fo_params(**kw) -> FoParams:
    """First-order (Adam) parameters: library defaults overridden by kw
    ('lambda' is accepted for lambda_)."""
    p = FoParams()
    _check(lib().ctc_fo_params_default(C.byref(p)))
    for k, v in kw.items():
        if k == "lambda":
            k = "lambda_"
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class FirstOrder:
    """Adjoint-driven full-gradient / minibatch Adam training (ctc_fo) of an
    order-3 or order-4 tensor."""

    def __init__(self, ctx: Context, train: Tensor, test: Tensor | None, p: FoParams):
        h = C.c_void_p()
        _check(lib().ctc_fo_create(ctx.h, train.h, test.h if test else None, C.byref(p), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._track(self)

    def dims(self):
        order = C.c_int()
        d = (C.c_uint64 * 4)()
        _check(lib().ctc_fo_dims(self.h, C.byref(order), d))
        return [d[m] for m in range(order.value)]

    def run(self, model: Model, p: FoParams, callback=None) -> RunOutput:
        out = RunOutput(result={})

        def _cb(_user, sp):
            d = _stats_dict(sp.contents)
            out.epochs.append(d)
            return int(bool(callback(d))) if callback else 0

        cb = EPOCH_CB(_cb)
        res = Result()
        _check(lib().ctc_fo_run(self.h, model.h, C.byref(p), cb, None, C.byref(res)))
        out.result = _result_dict(res)
        return out

    def grad(self, model: Model):
        """(grads per mode, objective) from the training step's adjoint pass
        (ctc_fo_grad: FP32 or BF16 gathers, FP32 accumulation)."""
        G = [np.zeros((d, model.rank), dtype=np.float64) for d in model.dims]
        ptrs = (_f64p * len(G))(*[g.ctypes.data_as(_f64p) for g in G])
        obj = C.c_double()
        _check(lib().ctc_fo_grad(self.h, model.h, ptrs, C.byref(obj)))
        return G, obj.value

    def free(self):
        if self.h:
            lib().ctc_fo_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
