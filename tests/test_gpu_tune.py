"""Autotuner on the device: every candidate is timed, the winner comes from
the candidate set and is cached, a second call is a cache hit, and runs
with the tuned parameters give the same model quality."""
from __future__ import annotations

import pytest

import cutc_b200 as ctc
from tests.helpers import Problem

pytestmark = pytest.mark.gpu


def test_tune_sgd_searches_caches_and_hits(ctx, tmp_path):
    P = Problem(40000, (400, 300, 200), 16, seed=61)
    p = ctc.params(ctc.SGD, rank=16, lr=0.01, lr_scale=1.0, **{"lambda": 0.01})
    path = str(tmp_path / "tune.txt")
    q, trials = ctc.autotune(ctx, P.c_sorted(), p, cache_path=path)
    # tile length x lanes per nonzero x reduction mode (vector atomics, bulk
    # rows, block-merged hot rows) at 256 threads per block, then 128 and
    # 512 threads for each tile length's fastest candidate, and 1024 where
    # that candidate is the hot-row form with at most two slices per lane
    big = [t for t in trials if t["threads_per_block"] == 1024]
    assert 36 + 8 <= len(trials) == 36 + 8 + len(big) <= 36 + 12
    assert all(t["cached"] == 0 and t["ms_epoch"] > 0 for t in trials)
    assert all(t["sgd_atomic"] == 3 and t["threads_per_row"] in (0, 2, 4) for t in big)
    assert {t["sgd_atomic"] for t in trials} == {1, 2, 3}
    assert {0, 128, 512} <= {t["threads_per_block"] for t in trials} <= {0, 128, 512, 1024}
    assert q.tile_len in (128, 256, 512, 1024) and q.threads_per_row in (4, 2, 1) and q.sgd_atomic in (1, 2, 3)
    assert q.threads_per_block in (0, 128, 512, 1024)
    best = min(trials, key=lambda t: t["ms_epoch"])
    keys = ("tile_len", "threads_per_row", "sgd_atomic", "threads_per_block")
    assert tuple(getattr(q, k) for k in keys) == tuple(best[k] for k in keys)
    q2, trials2 = ctc.autotune(ctx, P.c_sorted(), p, cache_path=path)
    assert len(trials2) == 1 and trials2[0]["cached"] == 1
    assert tuple(getattr(q2, k) for k in keys) == tuple(getattr(q, k) for k in keys)
    assert ctc.tune_lookup(path, P.c_sorted()[0], p) is not None


def test_tune_ccdpp_keeps_results(ctx, tmp_path):
    P = Problem(30000, (300, 200, 100), 16, seed=62)
    p = ctc.params(ctc.CCDPP, rank=16, inner=2, iters=2, early_stop=0, eval_every=1, **{"lambda": 0.1})
    q, trials = ctc.autotune(ctx, P.c_sorted(), p, cache_path=None)
    assert len(trials) == 6
    assert q.tile_len in (128, 256, 512) and q.smem_budget in (0, -1)
    m0, m1 = P.c_model(), P.c_model()
    o0 = ctc.run(ctx, P.c_sorted(), None, P.c_test(), m0, p)
    o1 = ctc.run(ctx, P.c_sorted(), None, P.c_test(), m1, q)
    a, b = o0.epochs[-1]["rmse_te"], o1.epochs[-1]["rmse_te"]
    assert abs(a - b) / a < 1e-5


def test_tune_als(ctx):
    P = Problem(30000, (300, 200, 100), 16, seed=63, heavy_row=3000)
    p = ctc.params(ctc.ALS, rank=16, **{"lambda": 0.05})
    q, trials = ctc.autotune(ctx, P.c_sorted(), p, write=False)
    assert len(trials) == 4 and q.tile_len in (256, 512, 1024, 2048)
