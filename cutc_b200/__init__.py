"""cutc_b200 -- B200-native (sm_100a) sparse tensor completion engine.

A drop-in for the single-GPU driver of cuTC (abovekumo/cuTC): .tns tensor
load, CISS tiling, ALS / CCD / CCD++ / SGD with per-epoch train/val/test
RMSE, behind the C ABI in include/ctc.h (libctc.so).  This package holds the
CUDA/C++ sources (csrc/), the in-tree build (build.py) and the Python
bindings (api.py).
"""
from .api import (ALS, CCD, CCDPP, SGD, PREC_F32, PREC_F64, PREC_MIXED, LR_BOLD_DRIVER,
                  LR_CONSTANT, LR_EXP_DECAY, SGD_HOGWILD, SGD_SEQUENTIAL, Batch, Context, CtcError,
                  Dataset, FirstOrder, Model, Params, Tensor, autotune, ciss_alloc, ciss_alloc_gpu, fo_params, grad, lib, params,
                  plan_tiles,
                  rmse, run, tc_als,
                  tune_key, tune_lookup,
                  tc_ccd, tc_main_ciss, tc_sgd, tt_read)

__all__ = ["ALS", "CCD", "CCDPP", "SGD", "PREC_F32", "PREC_F64", "PREC_MIXED", "LR_BOLD_DRIVER",
           "LR_CONSTANT", "LR_EXP_DECAY", "SGD_HOGWILD", "SGD_SEQUENTIAL", "Batch", "Context", "CtcError",
           "Dataset", "FirstOrder", "Model", "Params", "Tensor", "autotune", "ciss_alloc", "ciss_alloc_gpu", "fo_params", "grad", "lib", "params", "plan_tiles", "rmse",
           "run", "tc_als", "tc_ccd", "tc_main_ciss", "tc_sgd", "tt_read", "tune_key", "tune_lookup"]
