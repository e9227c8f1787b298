"""Batches of independent problems (ctc_batch_*): every instance trained in
one stacked launch must follow the same trajectory as the instance trained
alone through ctc_run, and as the FP64 CPU oracle."""
from __future__ import annotations

import numpy as np
import pytest

import cutc_b200 as ctc
from oracle import pyoracle as po
from tests.helpers import Problem, max_factor_rel

pytestmark = pytest.mark.gpu


def instances(n, R, seed=0, heavy=False, nnz_range=(800, 12000), dim_range=(20, 160)):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n):
        nnz = int(rng.integers(*nnz_range))
        dims = tuple(int(x) for x in rng.integers(*dim_range, 3))
        out.append(Problem(nnz, dims, R, seed=seed * 100 + b, heavy_row=(1500 if heavy and b == 1 else 0)))
    return out


def run_batch(ctx, probs, alg, iters, **kw):
    kw.setdefault("eval_every", 1)
    kw.setdefault("early_stop", 0)
    p = ctc.params(alg, rank=probs[0].R, iters=iters, **kw)
    train = [ctc.Tensor.from_coo(*P.train, dims=P.dims) for P in probs]
    test = [P.c_test() for P in probs]
    B = ctc.Batch(ctx, train, test, p)
    models = [P.c_model() for P in probs]
    out = B.run(models, p)
    B.free()
    return [m.factors() for m in models], out


def run_alone(ctx, P, alg, iters, **kw):
    kw.setdefault("eval_every", 1)
    kw.setdefault("early_stop", 0)
    p = ctc.params(alg, rank=P.R, iters=iters, **kw)
    m = P.c_model()
    out = ctc.run(ctx, P.c_sorted(), None, P.c_test(), m, p)
    return m.factors(), out


def test_batch_als_f64_matches_single_runs_and_oracle(ctx):
    probs = instances(5, 16, seed=1, heavy=True)
    lam = {"lambda": 0.05}
    Gb, ob = run_batch(ctx, probs, ctc.ALS, 2, precision=ctc.PREC_F64, **lam)
    assert len(ob.epochs) == 3
    for b, P in enumerate(probs):
        Ga, oa = run_alone(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F64, **lam)
        assert max_factor_rel(Gb[b], Ga) < 1e-9, b
        for e in range(3):
            assert abs(ob.epochs[e][2][b] - oa.epochs[e]["rmse_tr"]) <= 1e-9 * oa.epochs[e]["rmse_tr"], (b, e)
            assert abs(ob.epochs[e][3][b] - oa.epochs[e]["rmse_te"]) <= 1e-9 * oa.epochs[e]["rmse_te"], (b, e)
        # and the FP64 oracle (ALS, modes in order)
        U = P.factors()
        for _ in range(2):
            for m in range(3):
                po.als_mode(P.o_sorted(m), m, U, 0.05)
        assert max_factor_rel(Gb[b], U) < 1e-9, b


def test_batch_als_f32_per_instance_rmse(ctx):
    """FP32: per-iteration test RMSE of every instance within 1e-5 of the
    FP64 oracle, factors after one iteration within 1e-4 (later iterations
    compound FP32 Gram rounding), and the same RMSE as the instance alone."""
    probs = instances(7, 32, seed=2, nnz_range=(6000, 20000), dim_range=(20, 60))
    lam = {"lambda": 0.05}
    G1, _ = run_batch(ctx, probs, ctc.ALS, 1, precision=ctc.PREC_F32, **lam)
    Gb, ob = run_batch(ctx, probs, ctc.ALS, 3, precision=ctc.PREC_F32, **lam)
    for b, P in enumerate(probs):
        U = P.factors()
        te = []
        for it in range(3):
            for m in range(3):
                po.als_mode(P.o_sorted(m), m, U, 0.05)
            if it == 0:
                assert max_factor_rel(G1[b], U) < 1e-4, b
            te.append(po.rmse(P.o_test(), U))
        for it in range(3):
            assert abs(ob.epochs[it + 1][3][b] - te[it]) / te[it] < 1e-5, (b, it)
        Ga, oa = run_alone(ctx, P, ctc.ALS, 3, precision=ctc.PREC_F32, **lam)
        te_b, te_a = ob.epochs[-1][3][b], oa.epochs[-1]["rmse_te"]
        assert abs(te_b - te_a) / te_a < 1e-5, b


def test_batch_sgd_sequential_matches_single_runs(ctx):
    """The stacked tensor in mode-1 order is instance-major, so the
    deterministic SGD order visits each instance's nonzeros exactly as a run
    of that instance alone does."""
    probs = instances(4, 16, seed=3)
    kw = dict(precision=ctc.PREC_F64, sgd_order=ctc.SGD_SEQUENTIAL, lr=0.01, lr_scale=1.0,
              lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95, **{"lambda": 0.01})
    Gb, ob = run_batch(ctx, probs, ctc.SGD, 3, **kw)
    for b, P in enumerate(probs):
        Ga, oa = run_alone(ctx, P, ctc.SGD, 3, **kw)
        assert max_factor_rel(Gb[b], Ga) < 1e-9, b


def test_batch_sgd_hogwild_learns_every_instance(ctx):
    probs = instances(6, 16, seed=4)
    Gb, ob = run_batch(ctx, probs, ctc.SGD, 8, precision=ctc.PREC_F32, lr=0.02, lr_scale=1.0,
                       lr_schedule=ctc.LR_CONSTANT, **{"lambda": 0.01})
    first, last = ob.epochs[0][3], ob.epochs[-1][3]
    assert np.all(np.isfinite(last))
    assert np.all(last < first), (first, last)


def test_batch_rejects_ccdpp(ctx):
    probs = instances(2, 16, seed=5)
    p = ctc.params(ctc.CCDPP, rank=16, iters=1)
    train = [ctc.Tensor.from_coo(*P.train, dims=P.dims) for P in probs]
    with pytest.raises(ctc.CtcError):
        ctc.Batch(ctx, train, None, p)
