"""Parity pins of the forms the bench measures, against the FP64 CPU oracle
on the same seeded inputs and initial factors (engine called through the C
ABI):

  - Hogwild SGD as benchmarked (per-row step damping on, vector atomics and
    bulk row reductions) on a 2M-nonzero sample of the 100M Zipf(1.1)
    workload's distribution, with the workload's SGD schedule: final test
    RMSE within 0.5 % of the deterministic sequential FP64 oracle;
  - plain FP32 ALS on the small uniform workload exactly as configured
    (2,000 x 1,500 x 200, 200,000 nonzeros, R 16, lambda 0.05, 10
    iterations): per-iteration RMSE within 1e-5, factors within 1e-4;
  - the early-stop loop with a validation tensor (tc_converge,
    sgpu/completion.c:296-362): stop epoch, best epoch and best factors
    equal the oracle's;
  - the FP32 and BF16 adjoint passes the first-order training uses, against
    the FP64 gradient (ctc_grad), at order 3 and 4;
  - mixed-precision CCD++ (packed residual slots): bit-identical to plain
    FP32 when the residual keeps all 32 bits, within 0.5 % of it per outer
    iteration on the Zipf sample, where it keeps 19.
"""
import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import synth
from oracle import pyoracle as po
from tests.helpers import max_factor_rel, rel

pytestmark = pytest.mark.gpu


class Data:
    """A generated workload as train (mode-1 sorted) / test / validation."""

    def __init__(self, w, seed, R, val_frac=0.0, factor_seed=0):
        g = synth.generate(w, seed=seed, device="cpu")
        self.dims = tuple(int(d) for d in g["dims"])
        self.R = R
        self.train = synth.sort_for_mode(*g["train"], 0)
        ti, tv = g["test"]
        if val_frac > 0:
            rng = np.random.default_rng(seed + 7)
            isv = rng.random(tv.shape[0]) < val_frac
            self.val = (ti[:, isv], tv[isv])
            self.test = (ti[:, ~isv], tv[~isv])
        else:
            self.val = None
            self.test = (ti, tv)
        rng = np.random.default_rng(factor_seed)
        self.U0 = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in self.dims]

    def o(self, part):
        return po.Tensor(*part, dims=self.dims)

    def c(self, part):
        return ctc.Tensor.from_coo(*part, dims=self.dims)

    def model(self):
        m = ctc.Model(self.dims, self.R)
        m.set_factors(self.U0)
        return m


# ------------------------------------------------------------------ SGD
@pytest.fixture(scope="module")
def zipf2m():
    # the 100M workload's distribution (500k x 20k x 2k, Zipf(1.1) in every
    # mode, CP rank 16 + N(0, 0.25^2) clipped to [1, 5]) at 2M nonzeros
    w = synth.scaled(synth.WORKLOADS["zipf-100m"], 2_000_000)
    return Data(w, seed=11, R=32)


@pytest.fixture(scope="module")
def zipf2m_oracle(zipf2m):
    D = zipf2m
    U = [u.copy() for u in D.U0]
    T = D.o(D.train)
    lr = 1e-3
    for _ in range(20):
        po.sgd_epoch(T, U, lr, 0.01, 1.0, False)
        lr *= 0.95
    return po.rmse(D.o(D.test), U, nthreads=8), po.rmse(T, U, nthreads=8)


@pytest.mark.parametrize("atomic,block,tile,tpr,groups",
                         [(1, 0, 0, 0, 0), (2, 0, 0, 0, 0), (3, 0, 0, 0, 0), (3, 1024, 0, 8, 0), (3, 1024, 128, 8, 384)])
def test_sgd_hogwild_damped_on_zipf_matches_sequential_oracle(ctx, zipf2m, zipf2m_oracle, atomic, block, tile,
                                                             tpr, groups):
    """The benchmarked Hogwild form: per-row damping at its default bound
    (rows whose expected in-flight updates exceed 128 take proportionally
    smaller steps; on this sample the hottest rows of modes 2 and 3 are
    damped), lr 1e-3 x 0.95 per epoch, lambda 0.01, 20 epochs; each
    reduction mode at the library's launch shape, the hot-row form in
    1024-thread blocks, and the shape the autotuner picks on the 100M tensor
    (1024-thread blocks, 128-nonzero tiles, 8 lanes a nonzero) at that
    tensor's concurrency: there one block per SM keeps 148 x 128 = 18,944 of
    703,000 tiles (2.7 %) in flight, while on this 2M sample the same launch
    would run all 15,600 tiles at once (1.2 % off the oracle, at any block
    size), so the groups in flight are capped at 384 (2.5 %)."""
    D = zipf2m
    p = ctc.params("sgd", rank=32, iters=20, lr=1e-3, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY,
                   lr_decay=0.95, sgd_order=ctc.SGD_HOGWILD, sgd_atomic=atomic, early_stop=0, eval_every=0,
                   threads_per_block=block, tile_len=tile, threads_per_row=tpr, sgd_groups=groups,
                   **{"lambda": 0.01})
    m = D.model()
    out = ctc.run(ctx, [D.c(D.train)], None, D.c(D.test), m, p)
    te, tr = zipf2m_oracle
    got = out.epochs[-1]["rmse_te"]
    assert abs(got - te) / te < 0.005, (got, te)
    assert abs(out.epochs[-1]["rmse_tr"] - tr) / tr < 0.005


# ------------------------------------------------------------------ ALS, small uniform workload
def test_als_small_uniform_workload_exactly(ctx):
    """2,000 x 1,500 x 200, 200,000 uniform distinct cells (rank-8 CP values
    in [1, 5] + N(0, 0.1^2)), 90/10 split, R 16, lambda 0.05, 10 iterations,
    FP32, factors U(0,1)/sqrt(16)."""
    w = synth.WORKLOADS["small-als"]
    D = Data(w, seed=1, R=16)
    assert D.train[1].shape[0] + D.test[1].shape[0] == 200_000
    U = [u.copy() for u in D.U0]
    sorted_o = [D.o(synth.sort_for_mode(*D.train, m)) for m in range(3)]
    hist = [(po.rmse(D.o(D.train), U), po.rmse(D.o(D.test), U))]
    for _ in range(10):
        for m in range(3):
            po.als_mode(sorted_o[m], m, U, 0.05, None, False, nthreads=8)
        hist.append((po.rmse(D.o(D.train), U), po.rmse(D.o(D.test), U)))
    p = ctc.params("als", rank=16, iters=10, precision=ctc.PREC_F32, early_stop=0, eval_every=1,
                   **{"lambda": 0.05})
    m = D.model()
    out = ctc.run(ctx, [D.c(D.train)], None, D.c(D.test), m, p)
    assert len(out.epochs) == 11
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-5, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-5, e
    assert max_factor_rel(m.factors(), U) < 1e-4


# ------------------------------------------------------------------ early stop
@pytest.mark.parametrize("alg", ["als", "ccdpp"])
def test_early_stop_with_validation_matches_tc_converge(ctx, alg):
    """A small sparse tensor at rank 32 with a tiny lambda overfits: the
    validation RMSE falls, then rises.  With early_stop = 1 the run must
    stop at the epoch where tc_converge's bad-epoch count reaches 3, report
    the oracle's best epoch, and hand back that epoch's factors as the
    best model."""
    from tests.helpers import Problem
    P = Problem(4000, (60, 50, 40), 32, seed=23, test_frac=0.3)
    ti, tv = P.test
    half = tv.shape[0] // 2
    val = (ti[:, :half], tv[:half])
    test = (ti[:, half:], tv[half:])
    lam = 1e-3
    U = P.factors()
    conv = po.Converge(1e-4, 3)
    snaps = {}
    stop = None
    T0 = P.o_sorted(0)
    r = po.residual(T0, U) if alg == "ccdpp" else None
    for e in range(1, 61):
        if alg == "als":
            for m in range(3):
                po.als_mode(P.o_sorted(m), m, U, lam)
        else:
            po.ccdpp_outer(T0, U, lam, 1, r)
        vr = po.rmse(po.Tensor(*val, dims=P.dims), U)
        improved, converged = conv.step(e, vr)
        if improved:
            snaps[e] = [u.copy() for u in U]
        if converged:
            stop = e
            break
    assert stop is not None and conv.best_epoch < stop, "the problem must overfit"
    p = ctc.params(alg, rank=32, iters=60, precision=ctc.PREC_F64, early_stop=1, inner=1, **{"lambda": lam})
    m = P.c_model()
    best = P.c_model()
    out = ctc.run(ctx, P.c_sorted(), ctc.Tensor.from_coo(*val, dims=P.dims), ctc.Tensor.from_coo(*test, dims=P.dims),
                  m, p, best=best)
    assert out.result["epochs_run"] == stop
    assert out.result["best_epoch"] == conv.best_epoch
    assert abs(out.result["best_rmse"] - conv.best_rmse) / conv.best_rmse < 1e-9
    assert len(out.epochs) == stop + 1
    assert max_factor_rel(best.factors(), snaps[conv.best_epoch]) < 1e-9
    assert max_factor_rel(m.factors(), U) < 1e-9


# ------------------------------------------------------------------ adjoint in FP32 / BF16
def _order4(nnz, dims, R, seed):
    rng = np.random.default_rng(seed)
    cells = rng.choice(int(np.prod(dims)), size=nnz, replace=False)
    ind = []
    for d in reversed(dims):
        ind.append(cells % d)
        cells = cells // d
    ind = np.stack(ind[::-1]).astype(np.uint64) + 1
    vals = rng.uniform(1, 5, nnz)
    U = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]
    return ind, vals, U


@pytest.mark.parametrize("order,R", [(3, 16), (3, 64), (4, 32)])
@pytest.mark.parametrize("prec", [ctc.PREC_F32, ctc.PREC_MIXED])
def test_adjoint_fp32_bf16_against_fp64_gradient(ctx, order, R, prec):
    """The gradient the first-order step consumes (ctc_fo_grad: the
    minibatch adjoint kernel over all training nonzeros) against the FP64
    gradient (ctc_grad).  Modes small enough to keep their gradient rows in
    shared memory and modes reduced in global memory are both present.
    Bounds, relative to each mode's largest gradient entry: FP32 1e-5; BF16
    gathers (factors rounded to 8 significant bits, relative error 2^-9 per
    element, three or four per product) 2e-2, and the mean error 10x below."""
    dims = (3000, 200, 40) if order == 3 else (2000, 150, 60, 12)
    ind, vals, U = _order4(30000, dims, R, seed=order * 100 + R)
    lam = 0.01
    t = ctc.Tensor.from_coo(ind, vals, dims=dims)
    m = ctc.Model(dims, R)
    m.set_factors(U)
    G64, obj64 = ctc.grad(ctx, t, m, lam)
    p = ctc.fo_params(rank=R, precision=prec, batch=0, epochs=1, **{"lambda": lam})
    F = ctc.FirstOrder(ctx, t, None, p)
    G, obj = F.grad(m)
    F.free()
    bound = 1e-5 if prec == ctc.PREC_F32 else 2e-2
    for g, g64 in zip(G, G64):
        scale = np.max(np.abs(g64))
        assert np.max(np.abs(g - g64)) / scale < bound
        if prec == ctc.PREC_MIXED:
            assert np.mean(np.abs(g - g64)) / scale < bound / 10
    assert abs(obj - obj64) / obj64 < (1e-6 if prec == ctc.PREC_F32 else 1e-2)
    assert rel(G[0], G64[0]) < bound


# ------------------------------------------------------------------ CCD++ mixed precision (packed slots)
def test_ccdpp_packed_with_full_residual_bits_equals_plain(ctx):
    """Small dimensions leave 32 bits beside the key, so the packed slots
    hold the FP32 residual unrounded: the mixed-precision run must equal
    the plain FP32 run bit for bit (same arithmetic, other layout)."""
    from tests.helpers import Problem
    P = Problem(40000, (900, 700, 40), 16, seed=44, heavy_row=3000)
    outs = {}
    for prec in (ctc.PREC_F32, ctc.PREC_MIXED):
        p = ctc.params("ccdpp", rank=16, iters=2, inner=2, precision=prec, early_stop=0, eval_every=1,
                       tile_len=128, **{"lambda": 0.1})
        m = P.c_model()
        out = ctc.run(ctx, P.c_sorted(), None, P.c_test(), m, p)
        outs[prec] = (m.factors(), [e["rmse_tr"] for e in out.epochs], [e["rmse_te"] for e in out.epochs])
    for a, b in zip(outs[ctc.PREC_F32][0], outs[ctc.PREC_MIXED][0]):
        assert np.array_equal(a, b)
    assert outs[ctc.PREC_F32][1:] == outs[ctc.PREC_MIXED][1:]


def test_ccdpp_packed_on_zipf_tracks_plain(ctx, zipf2m):
    """The 100M workload's dimensions need 45 key bits, leaving 19 for the
    residual (FP32 sign and exponent, 10 mantissa bits).  Per outer
    iteration the test RMSE stays within 0.5 % of plain FP32, and the
    training RMSE read from the packed residuals agrees with the record
    squared-error kernel on the final factors."""
    D = zipf2m
    runs = {}
    for prec in (ctc.PREC_F32, ctc.PREC_MIXED):
        p = ctc.params("ccdpp", rank=32, iters=4, inner=3, precision=prec, early_stop=0, eval_every=1,
                       **{"lambda": 0.1})
        m = D.model()
        out = ctc.run(ctx, [D.c(D.train)], None, D.c(D.test), m, p)
        runs[prec] = (out, m)
    for e in range(5):
        a = runs[ctc.PREC_F32][0].epochs[e]["rmse_te"]
        b = runs[ctc.PREC_MIXED][0].epochs[e]["rmse_te"]
        assert abs(a - b) / a < 0.005, (e, a, b)
    out, m = runs[ctc.PREC_MIXED]
    tr = ctc.rmse(ctx, D.c(D.train), m)
    assert abs(out.epochs[-1]["rmse_tr"] - tr) / tr < 1e-3, (out.epochs[-1]["rmse_tr"], tr)


# ------------------------------------------------------------------ CCD++ and ALS on the Zipf sample
def test_ccdpp_on_zipf_matches_oracle(ctx, zipf2m):
    """CCD++ with the benchmarked schedule (lambda 0.1, 3 inner sweeps) on
    the Zipf sample, whose hottest rows hold hundreds of thousands of
    nonzeros (long-row groups, partial sums across warps).  FP64: factors
    and per-iteration RMSE within 1e-9 of the FP64 oracle (the same
    algorithm).  FP32: per-iteration RMSE within 1e-5; factors within 1e-2
    of the largest entry, not 1e-4: on this sample the FP32 sums
    r.h over a hot row cancel to a small numerator, which the weakly
    regularised updates of rarely observed rows (lambda + sum h^2 near 0.1)
    then amplify over the 192 column updates (measured: 3.9e-3, on the
    2,000-row mode)."""
    D = zipf2m
    U = [u.copy() for u in D.U0]
    T = D.o(D.train)
    r = po.residual(T, U)
    hist = [(po.rmse(T, U, nthreads=8), po.rmse(D.o(D.test), U, nthreads=8))]
    for _ in range(2):
        po.ccdpp_outer(T, U, 0.1, 3, r, nthreads=8)
        hist.append((po.rmse(T, U, nthreads=8), po.rmse(D.o(D.test), U, nthreads=8)))
    for prec, tol_r, tol_f in ((ctc.PREC_F64, 1e-9, 1e-9), (ctc.PREC_F32, 1e-5, 1e-2)):
        p = ctc.params("ccdpp", rank=32, iters=2, inner=3, precision=prec, early_stop=0, eval_every=1,
                       **{"lambda": 0.1})
        m = D.model()
        out = ctc.run(ctx, [D.c(D.train)], None, D.c(D.test), m, p)
        for e, (tr, te) in enumerate(hist):
            assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < tol_r, (prec, e)
            assert abs(out.epochs[e]["rmse_te"] - te) / te < tol_r, (prec, e)
        assert max_factor_rel(m.factors(), U) < tol_f, prec


@pytest.mark.parametrize("prec", [ctc.PREC_F32, ctc.PREC_MIXED])
def test_als_on_zipf_matches_oracle(ctx, zipf2m, prec):
    """ALS (lambda 0.1, rank 32) on the Zipf sample, one iteration: FP32
    within 1e-5 (RMSE) and 1e-4 (factors) of the FP64 oracle; the mixed
    form, whose long rows take their Gram from BF16 tensor-core MMAs, within
    0.5 % (RMSE) and 3e-2 (factors)."""
    D = zipf2m
    U = [u.copy() for u in D.U0]
    sorted_o = [D.o(synth.sort_for_mode(*D.train, m)) for m in range(3)]
    for m in range(3):
        po.als_mode(sorted_o[m], m, U, 0.1, None, False, nthreads=8)
    tr, te = po.rmse(D.o(D.train), U, nthreads=8), po.rmse(D.o(D.test), U, nthreads=8)
    p = ctc.params("als", rank=32, iters=1, precision=prec, early_stop=0, eval_every=1, **{"lambda": 0.1})
    m = D.model()
    out = ctc.run(ctx, [D.c(D.train)], None, D.c(D.test), m, p)
    tol_r, tol_f = (1e-5, 1e-4) if prec == ctc.PREC_F32 else (5e-3, 3e-2)
    assert abs(out.epochs[1]["rmse_tr"] - tr) / tr < tol_r
    assert abs(out.epochs[1]["rmse_te"] - te) / te < tol_r
    assert max_factor_rel(m.factors(), U) < tol_f
