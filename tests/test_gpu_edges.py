"""The update rules at the edges of the input space, in FP64 on the GPU
against the FP64 oracle: factors within 1e-9 of the largest factor entry,
per-iteration RMSE within 1e-9 (relative, absolute below 1; the values
lie between 1 and 5).

- a mode with a single row, in each of the three positions;
- a single nonzero;
- 32k, 32k + 1 and 32k + 31 nonzeros: full, just started and nearly full
  32-entry groups, the warp and tile edges of the reference layout
  (sgpu/base.h:62, DEFAULT_T_TILE_LENGTH 32);
- modes whose rows are mostly empty: ALS and CCD++ set a row without
  nonzeros to 0 (sgpu/als.cu:699, 730, 757 clear each factor before its
  row solves; the rank-one update gives 0 / (lambda + 0)), CCD and SGD
  leave it as it was;
- the mode-1 tensor alone, so that the other two copies are sorted, split
  into row runs and planned on the device at these sizes too.

An empty training or test tensor is rejected on the host, before any
launch, with CTC_E_ARG (the reference would divide by its zero nonzero
count in the RMSE, sgpu/completion.c:129)."""
import numpy as np
import pytest

import cutc_b200 as ctc
from oracle import pyoracle as po
from tests.helpers import Problem, max_factor_rel

R = 8
ITERS = 2
# CCD (the reference rule, all R columns of a row from one residual) needs
# the larger lambda to stay bounded on these few nonzeros
LAM = {"als": 0.5, "ccd": 5.0, "ccdpp": 0.1, "sgd": 0.01}
INNER = 2
LR, DECAY = 0.01, 0.95

CASES = {
    "one-row-mode-1": (25, (1, 9, 8)),
    "one-row-mode-2": (25, (9, 1, 8)),
    "one-row-mode-3": (25, (9, 8, 1)),
    "one-nonzero": (1, (3, 4, 5)),
    "nnz-64": (64, (12, 10, 8)),
    "nnz-65": (65, (12, 10, 8)),
    "nnz-95": (95, (12, 10, 8)),
    "mostly-empty-rows": (40, (500, 400, 300)),
}


def make_problem(case):
    nnz, dims = CASES[case]
    P = Problem(nnz, dims, R, seed=200 + sorted(CASES).index(case), test_frac=0.0)
    P.test = (P.train[0][:, :5], P.train[1][:5])
    return P


def oracle_run(P, alg):
    U = P.factors()
    hist = [(po.rmse(P.o_train(), U), po.rmse(P.o_test(), U))]
    T0 = P.o_sorted(0)
    resid = po.residual(T0, U) if alg == "ccdpp" else None
    lr = LR
    for _ in range(ITERS):
        if alg == "als":
            for m in range(3):
                po.als_mode(P.o_sorted(m), m, U, LAM[alg])
        elif alg == "ccd":
            for m in range(3):
                po.ccd_compat_mode(P.o_sorted(m), m, U, LAM[alg], None, False)
        elif alg == "ccdpp":
            po.ccdpp_outer(T0, U, LAM[alg], INNER, resid)
        else:
            po.sgd_epoch(T0, U, lr, LAM[alg])
            lr *= DECAY
        hist.append((po.rmse(P.o_train(), U), po.rmse(P.o_test(), U)))
    return U, hist


def engine_params(alg, precision=ctc.PREC_F64):
    kw = dict(rank=R, iters=ITERS, precision=precision, early_stop=0, eval_every=1)
    kw["lambda"] = LAM[alg]
    if alg == "ccdpp":
        kw["inner"] = INNER
    if alg == "sgd":
        kw.update(sgd_order=ctc.SGD_SEQUENTIAL, lr=LR, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY,
                  lr_decay=DECAY)
    return ctc.params(alg, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("copies", ["three", "one"])
@pytest.mark.parametrize("alg", ["als", "ccd", "ccdpp", "sgd"])
@pytest.mark.parametrize("case", list(CASES))
def test_edge_shapes_match_oracle(ctx, case, alg, copies):
    if alg == "sgd" and copies == "one":
        pytest.skip("SGD reads the mode-1 copy only")
    P = make_problem(case)
    U, hist = oracle_run(P, alg)
    train = P.c_sorted() if copies == "three" else P.c_sorted()[:1]
    model = P.c_model()
    out = ctc.run(ctx, train, None, P.c_test(), model, engine_params(alg))
    G = model.factors()
    assert max_factor_rel(G, U) < 1e-9
    for e, (tr, te) in enumerate(hist):
        if alg != "sgd":
            assert abs(out.epochs[e]["rmse_tr"] - tr) < 1e-9 * max(tr, 1.0), e
        assert abs(out.epochs[e]["rmse_te"] - te) < 1e-9 * max(te, 1.0), e


# FP32 against the FP64 oracle on the same edges.  RMSE within 5e-5
# absolute: 1e-5 of the largest value (5); on these few nonzeros a late
# RMSE is a small difference of values near 5, so a relative bound would
# measure the cancellation, not the kernels.  Factors within 1e-4 of the
# largest entry, CCD++ within 1e-3: its rank-one updates on 95 nonzeros
# amplify rounding (a float32 numpy restatement of the same two outer
# iterations lands 1.3e-4 from FP64; ALS restated the same way, 7.5e-6).
F32_FACTORS = {"als": 1e-4, "ccd": 1e-4, "ccdpp": 1e-3, "sgd": 1e-4}


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["als", "ccd", "ccdpp", "sgd"])
@pytest.mark.parametrize("case", list(CASES))
def test_edge_shapes_fp32(ctx, case, alg):
    """FP32 at the same edges.  For CCD++ the mixed-precision form (the
    residual packed into the key word) runs too: these dimensions leave
    all 32 residual bits beside the key, so it must equal the FP32 run bit
    for bit."""
    P = make_problem(case)
    U, hist = oracle_run(P, alg)
    model = P.c_model()
    out = ctc.run(ctx, P.c_sorted(), None, P.c_test(), model, engine_params(alg, ctc.PREC_F32))
    G = model.factors()
    assert max_factor_rel(G, U) < F32_FACTORS[alg]
    for e, (tr, te) in enumerate(hist):
        if alg != "sgd":
            assert abs(out.epochs[e]["rmse_tr"] - tr) < 5e-5, e
        assert abs(out.epochs[e]["rmse_te"] - te) < 5e-5, e
    if alg == "ccdpp":
        mm = P.c_model()
        om = ctc.run(ctx, P.c_sorted(), None, P.c_test(), mm, engine_params(alg, ctc.PREC_MIXED))
        for a, b in zip(mm.factors(), G):
            assert np.array_equal(a, b)
        assert [x["rmse_te"] for x in om.epochs] == [x["rmse_te"] for x in out.epochs]


@pytest.mark.gpu
@pytest.mark.parametrize("atomic", [1, 2, 3])
@pytest.mark.parametrize("case", list(CASES))
def test_edge_shapes_hogwild_learn(ctx, case, atomic):
    """Hogwild SGD in FP32 (vector atomics, bulk row reductions, block-merged
    hot rows: fewer rows than hot-row slots here) on the same edges, five
    epochs at lr 0.05: the factors stay finite and the test RMSE falls, as
    the sequential oracle's does on every case (a bulk reduction still in
    flight when the next nonzero of the same row reads it is Hogwild's own
    staleness, so these tiny, all-hot tensors are not held to the
    sequential trajectory; the 0.5 % pins run on realistic tensors)."""
    P = make_problem(case)
    kw = dict(rank=R, iters=5, precision=ctc.PREC_F32, early_stop=0, eval_every=1, tile_len=128,
              sgd_atomic=atomic, lr=0.05, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY, lr_decay=DECAY)
    kw["lambda"] = LAM["sgd"]
    model = P.c_model()
    out = ctc.run(ctx, P.c_sorted()[:1], None, P.c_test(), model, ctc.params("sgd", **kw))
    assert all(np.isfinite(g).all() for g in model.factors())
    te = [e["rmse_te"] for e in out.epochs]
    assert te[-1] < te[0], te


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["als", "ccd", "sgd"])
def test_edge_shapes_in_one_batch(ctx, alg):
    """All the edge tensors above as the instances of one batch
    (ctc_batch_*: stacked block-diagonally, one launch per mode update for
    all of them; CCD++ does not batch): each instance matches its own FP64
    oracle run, factors and per-iteration RMSE within 1e-9."""
    probs = [make_problem(c) for c in CASES]
    p = engine_params(alg)
    B = ctc.Batch(ctx, [ctc.Tensor.from_coo(*P.train, dims=P.dims) for P in probs],
                  [P.c_test() for P in probs], p)
    models = [P.c_model() for P in probs]
    try:
        out = B.run(models, p)
    finally:
        B.free()
    for b, P in enumerate(probs):
        U, hist = oracle_run(P, alg)
        assert max_factor_rel(models[b].factors(), U) < 1e-9, list(CASES)[b]
        for e, (tr, te) in enumerate(hist):
            if alg != "sgd":
                assert abs(out.epochs[e][2][b] - tr) < 1e-9 * max(tr, 1.0), (list(CASES)[b], e)
            assert abs(out.epochs[e][3][b] - te) < 1e-9 * max(te, 1.0), (list(CASES)[b], e)


def test_mostly_empty_rows_keep_the_reference_values():
    """The oracle side of the empty-row rule the GPU test above checks
    (no GPU needed): after ALS and CCD++ the rows without nonzeros are 0,
    after CCD and SGD they keep their initial values."""
    P = make_problem("mostly-empty-rows")
    for alg in ("als", "ccd", "ccdpp", "sgd"):
        U, _ = oracle_run(P, alg)
        for m in range(3):
            hit = np.zeros(P.dims[m], dtype=bool)
            hit[P.train[0][m].astype(np.int64) - 1] = True
            empty = ~hit
            assert empty.sum() > 0
            if alg in ("als", "ccdpp"):
                assert np.all(U[m][empty] == 0.0), (alg, m)
            else:
                assert np.array_equal(U[m][empty], P.U0[m][empty]), (alg, m)


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["als", "ccd", "ccdpp", "sgd"])
def test_empty_tensors_are_rejected(ctx, alg):
    P = make_problem("nnz-64")
    empty = ctc.Tensor.from_coo(np.zeros((3, 0), dtype=np.uint64), np.zeros(0), dims=P.dims)
    p = engine_params(alg)
    with pytest.raises(ctc.CtcError) as e:
        ctc.run(ctx, [empty], None, P.c_test(), P.c_model(), p)
    assert e.value.code == -1 and "empty" in str(e.value)
    with pytest.raises(ctc.CtcError) as e:
        ctc.run(ctx, P.c_sorted(), None, empty, P.c_model(), p)
    assert e.value.code == -1 and "empty" in str(e.value)
    with pytest.raises(ctc.CtcError) as e:
        ctc.rmse(ctx, empty, P.c_model())
    assert e.value.code == -1 and "empty" in str(e.value)
