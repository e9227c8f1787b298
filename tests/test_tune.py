"""Autotuner cache (host only): shape keys and lookups of tuned entries."""
from __future__ import annotations

import numpy as np

import cutc_b200 as ctc
from cutc_b200 import synth


def _tensor(nnz, dims, seed=0):
    ind, vals = synth.random_small(nnz, dims, seed=seed)
    return ctc.Tensor.from_coo(ind, vals, dims=dims)


def test_key_buckets_shapes():
    p = ctc.params(ctc.SGD, rank=16)
    k1 = ctc.tune_key(_tensor(1000, (50, 40, 30)), p)
    k2 = ctc.tune_key(_tensor(1010, (50, 40, 30), seed=1), p)
    k3 = ctc.tune_key(_tensor(2000, (50, 40, 30)), p)
    assert k1 == k2            # same half-power-of-two bucket
    assert k1 != k3            # twice the nonzeros: another shape
    assert "alg=1" in k1 and "rank=16" in k1 and "sms=148" in k1
    assert ctc.tune_key(_tensor(1000, (50, 40, 30)), p, sm_count=132) != k1
    assert ctc.tune_key(_tensor(1000, (50, 40, 30)), ctc.params(ctc.ALS, rank=16)) != k1


def test_lookup_hit_miss_and_last_entry_wins(tmp_path):
    t = _tensor(3000, (60, 50, 40))
    p = ctc.params(ctc.CCDPP, rank=32)
    path = str(tmp_path / "tune.txt")
    assert ctc.tune_lookup(str(tmp_path / "missing.txt"), t, p) is None
    key = ctc.tune_key(t, p)
    with open(path, "w") as f:
        f.write("garbage line\n")
        f.write("alg=9,other 1 2 3\n")
        f.write(f"{key} tile_len=128 threads_per_row=0 smem_budget=-1 sgd_atomic=1 threads_per_block=0 ms=1.5\n")
        f.write(f"{key} tile_len=512 threads_per_row=0 smem_budget=0 sgd_atomic=2 threads_per_block=128 ms=1.2\n")
        # lines without the reduction mode or the block size (older caches) are not entries
        f.write(f"{key} tile_len=256 threads_per_row=0 smem_budget=0 ms=1.0\n")
        f.write(f"{key} tile_len=256 threads_per_row=0 smem_budget=0 sgd_atomic=2 ms=1.0\n")
    q = ctc.tune_lookup(path, t, p)
    assert q is not None
    assert (q.tile_len, q.threads_per_row, q.smem_budget, q.sgd_atomic, q.threads_per_block) == (512, 0, 0, 2, 128)
    # everything else is the caller's
    assert q.rank == 32 and q.alg == ctc.CCDPP and abs(q.lambda_ - p.lambda_) == 0
    assert ctc.tune_lookup(path, t, ctc.params(ctc.CCDPP, rank=16)) is None


def test_block_size_is_validated_on_the_host():
    """threads_per_block: 0 or a power of two up to 512; the reference GA's
    4-16 thread blocks are below a warp and rejected as unsupported; 1024
    only for the block-merged hot-row form with at most two 16-byte slices
    per lane.  The checks run before any device is touched."""
    import ctypes as C
    L = ctc.lib()
    for ok in (0, 32, 64, 128, 256, 512):
        assert L.ctc_params_check(C.byref(ctc.params(ctc.SGD, rank=16, threads_per_block=ok))) == 0
    for bad, code in ((100, -1), (2048, -1), (-32, -1), (16, -5), (4, -5), (1024, -5)):
        p = ctc.params(ctc.SGD, rank=16, threads_per_block=bad)
        assert L.ctc_params_check(C.byref(p)) == code, bad
        assert b"threads_per_block" in L.ctc_last_error()
    # rank 32: 8 lanes a nonzero hold one slice each, 4 lanes two, 2 lanes four
    for tpr, code in ((8, 0), (4, 0), (0, 0), (2, -5)):
        p = ctc.params(ctc.SGD, rank=32, threads_per_block=1024, sgd_atomic=3, threads_per_row=tpr)
        assert L.ctc_params_check(C.byref(p)) == code, tpr
    p = ctc.params(ctc.SGD, rank=32, threads_per_block=1024, sgd_atomic=1)
    assert L.ctc_params_check(C.byref(p)) == -5
