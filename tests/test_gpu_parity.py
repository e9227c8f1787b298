"""Parity of the CUDA engine (called through the C ABI) with the FP64 CPU
oracle on the same seeded tensors and initial factors.

Tolerances (relative to the largest magnitude of the compared quantity):
  FP64 runs          factors and RMSE within 1e-9
  FP32 runs          per-iteration RMSE within 1e-5, factors within 1e-4 (ALS,
                     CCD++); SGD trajectory within 1e-3
  Hogwild SGD        final test RMSE within 0.5 % of the sequential oracle
"""
import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import synth
from oracle import pyoracle as po
from tests.helpers import Problem, max_factor_rel, rel

pytestmark = pytest.mark.gpu


def engine_run(ctx, P, alg, iters, **kw):
    kw.setdefault("early_stop", 0)
    kw.setdefault("eval_every", 1)
    kw.setdefault("rank", P.R)
    p = ctc.params(alg, iters=iters, **kw)
    model = P.c_model()
    out = ctc.run(ctx, P.c_sorted(), None, P.c_test(), model, p)
    return model.factors(), out


def oracle_rmse(P, U):
    return po.rmse(P.o_train(), U), po.rmse(P.o_test(), U)


# ------------------------------------------------------------------ RMSE
def test_rmse_kernel(ctx):
    P = Problem(20000, (300, 200, 100), 16, seed=1)
    m = P.c_model()
    got = ctc.rmse(ctx, P.c_test(), m)
    want = po.rmse(P.o_test(), P.factors())
    assert abs(got - want) / want < 1e-5


@pytest.mark.parametrize("R", [8, 16, 32, 64])
def test_rmse_ranks(ctx, R):
    P = Problem(5000, (80, 70, 60), R, seed=R)
    assert abs(ctc.rmse(ctx, P.c_test(), P.c_model()) - po.rmse(P.o_test(), P.factors())) < 1e-5 * 5


# ------------------------------------------------------------------ ALS
def oracle_als(P, iters, lam, w=None, trunc=False):
    U = P.factors()
    hist = [oracle_rmse(P, U)]
    for _ in range(iters):
        for m in range(3):
            po.als_mode(P.o_sorted(m), m, U, lam, None if w is None else w[m], trunc)
        hist.append(oracle_rmse(P, U))
    return U, hist


@pytest.mark.parametrize("R", [8, 16, 32])
def test_als_f64(ctx, R):
    P = Problem(12000, (150, 120, 40), R, seed=3)
    U, hist = oracle_als(P, 3, 0.05)
    G, out = engine_run(ctx, P, ctc.ALS, 3, precision=ctc.PREC_F64, **{"lambda": 0.05})
    assert max_factor_rel(G, U) < 1e-9
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-9
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-9


@pytest.mark.parametrize("R", [8, 16, 32, 64])
def test_als_short_rows_dual_solve(ctx, R):
    """Mode 1 has 3000 rows for 9000 nonzeros, so most of its rows hold at
    most R / 2 nonzeros and take the k x k dual solve (u = H^T (H H^T +
    lambda I)^-1 x); modes 2 and 3 have long rows and take the R x R
    solves.  Both match the FP64 oracle to 1e-9 in FP64 and to the FP32
    bars in FP32."""
    P = Problem(10000, (3000, 40, 30), R, seed=41)
    U, hist = oracle_als(P, 2, 0.1)
    G, out = engine_run(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F64, **{"lambda": 0.1})
    assert max_factor_rel(G, U) < 1e-9
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-9
    U1, hist1 = oracle_als(P, 1, 0.1)
    G1, out1 = engine_run(ctx, P, ctc.ALS, 1, precision=ctc.PREC_F32, **{"lambda": 0.1})
    assert max_factor_rel(G1, U1) < 1e-4
    assert abs(out1.epochs[1]["rmse_te"] - hist1[1][1]) / hist1[1][1] < 1e-5


def test_als_f32_config(ctx):
    """Plain FP32 ALS at R=16, lambda=0.05 (the small uniform workload's
    settings), 10 iterations."""
    P = Problem(40000, (400, 300, 40), 16, seed=4)
    U, hist = oracle_als(P, 10, 0.05)
    G, out = engine_run(ctx, P, ctc.ALS, 10, precision=ctc.PREC_F32, **{"lambda": 0.05})
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-5, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-5, e
    assert max_factor_rel(G, U) < 1e-4


def test_als_heavy_rows(ctx):
    """Rows longer than a tile go through the piece + fixup path."""
    P = Problem(6000, (60, 50, 40), 16, seed=5, heavy_row=1800)
    U, hist = oracle_als(P, 2, 0.1)
    G, out = engine_run(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F64, tile_len=64, **{"lambda": 0.1})
    assert max_factor_rel(G, U) < 1e-9


@pytest.mark.parametrize("R,tile_len", [(64, 256), (32, 256), (32, 96), (32, 48)])
def test_als_mixed_tensor_core(ctx, R, tile_len):
    """Ranks 64 and 32, mixed precision: pieces of long rows get their Gram
    from tcgen05 MMAs on BF16 factor copies (FP32 accumulation in tensor
    memory), every row its FP64 solve.  At rank 32 one 128-byte operand row
    carries two nonzeros; tile lengths 96 and 48 give chunks of more and of
    fewer than 64 nonzeros.  Final test RMSE within 0.5 % of plain FP32,
    first-iteration factors within BF16-level error of the FP64 oracle."""
    P = Problem(60000, (200, 150, 100), R, seed=30, heavy_row=20000)
    lam = {"lambda": 0.05}
    # every mode has rows longer than a tile, so the tensor-core Gram runs
    # once per mode and iteration
    _, o32 = engine_run(ctx, P, ctc.ALS, 5, precision=ctc.PREC_F32, tile_len=tile_len, **lam)
    ctx.set_profiling(True)
    ctx.reset_kernel_times()
    Gm, om = engine_run(ctx, P, ctc.ALS, 5, precision=ctc.PREC_MIXED, tile_len=tile_len, **lam)
    n_tc, ms_tc = ctx.kernel_time("k_als_gram_tc")
    ctx.set_profiling(False)
    assert n_tc == 3 * 5, n_tc
    te32, tem = o32.epochs[-1]["rmse_te"], om.epochs[-1]["rmse_te"]
    assert abs(tem - te32) / te32 < 0.005, (tem, te32)
    U, _ = oracle_als(P, 1, 0.05)
    G1, _ = engine_run(ctx, P, ctc.ALS, 1, precision=ctc.PREC_MIXED, tile_len=tile_len, **lam)
    assert max_factor_rel(G1, U) < 3e-2


def test_als_compat_matches_reference_semantics(ctx):
    """compat=1: values stored through an integer and the reference warp
    kernel's per-lane multiplicities (nnz % 32 == 0 for every copy)."""
    P = Problem(4096 + 455, (70, 60, 50), 16, seed=6, test_frac=0.0)
    n = P.train[0].shape[1] // 32 * 32
    P.train = (P.train[0][:, :n], P.train[1][:n])
    from cutc_b200 import synth
    P.sorted = [synth.sort_for_mode(*P.train, m) for m in range(3)]
    P.test = (P.train[0][:, :64], P.train[1][:64])
    w = [po.compat_weights(P.o_sorted(m), m, 0) for m in range(3)]
    U, hist = oracle_als(P, 2, 10.0, w=w, trunc=True)
    G, out = engine_run(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F64, compat=1, **{"lambda": 10.0})
    assert max_factor_rel(G, U) < 1e-9


# ------------------------------------------------------------------ CCD
def test_ccd_compat(ctx):
    P = Problem(8192 + 500, (90, 80, 30), 16, seed=7, test_frac=0.0)
    n = P.train[0].shape[1] // 32 * 32
    P.train = (P.train[0][:, :n], P.train[1][:n])
    from cutc_b200 import synth
    P.sorted = [synth.sort_for_mode(*P.train, m) for m in range(3)]
    P.test = (P.train[0][:, :64], P.train[1][:64])
    w = [po.compat_weights(P.o_sorted(m), m, 1) for m in range(3)]
    U = P.factors()
    for _ in range(2):
        for m in range(3):
            po.ccd_compat_mode(P.o_sorted(m), m, U, 100.0, w[m], True)
    G, out = engine_run(ctx, P, ctc.CCD, 2, precision=ctc.PREC_F64, compat=1, **{"lambda": 100.0})
    assert max_factor_rel(G, U) < 1e-9


def test_ccd_plain_f64(ctx):
    P = Problem(9000, (90, 80, 30), 16, seed=8, heavy_row=700)
    U = P.factors()
    for _ in range(2):
        for m in range(3):
            po.ccd_compat_mode(P.o_sorted(m), m, U, 1.0, None, False)
    G, out = engine_run(ctx, P, ctc.CCD, 2, precision=ctc.PREC_F64, tile_len=64, **{"lambda": 1.0})
    assert max_factor_rel(G, U) < 1e-9


# ------------------------------------------------------------------ CCD++
def oracle_ccdpp(P, iters, lam, inner):
    U = P.factors()
    T = P.o_sorted(0)
    r = po.residual(T, U)
    hist = [oracle_rmse(P, U)]
    for _ in range(iters):
        po.ccdpp_outer(T, U, lam, inner, r)
        hist.append(oracle_rmse(P, U))
    return U, hist, r


@pytest.mark.parametrize("R", [8, 32])
def test_ccdpp_f64(ctx, R):
    P = Problem(15000, (200, 150, 60), R, seed=9, heavy_row=900)
    U, hist, _ = oracle_ccdpp(P, 2, 0.1, 3)
    G, out = engine_run(ctx, P, ctc.CCDPP, 2, precision=ctc.PREC_F64, inner=3, tile_len=128,
                        **{"lambda": 0.1})
    assert max_factor_rel(G, U) < 1e-9
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-9
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-9


def test_ccdpp_f32(ctx):
    P = Problem(50000, (500, 300, 60), 32, seed=10)
    U, hist, _ = oracle_ccdpp(P, 3, 0.1, 3)
    G, out = engine_run(ctx, P, ctc.CCDPP, 3, precision=ctc.PREC_F32, inner=3, **{"lambda": 0.1})
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-5, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-5, e
    assert max_factor_rel(G, U) < 1e-4


@pytest.mark.parametrize("tile_len", [128, 256, 512])
def test_ccdpp_column_staging_paths_agree(ctx, tile_len):
    """The factor columns a pass gathers come from shared memory (staged by a
    bulk async copy) when they fit the block budget, else from global
    memory.  All staged, one staged and none staged give bit-identical
    factors (same values, same summation order), and match the oracle."""
    P = Problem(40000, (9000, 700, 40), 16, seed=44, heavy_row=3000)
    U, hist, _ = oracle_ccdpp(P, 2, 0.1, 2)
    runs = {}
    # budgets: default (all fit), one column fits (mode 2: 40 values), none
    for budget in (0, 1024, -1):
        G, out = engine_run(ctx, P, ctc.CCDPP, 2, precision=ctc.PREC_F32, inner=2, tile_len=tile_len,
                            smem_budget=budget, **{"lambda": 0.1})
        runs[budget] = (G, out)
    for budget in (1024, -1):
        for m in range(3):
            assert np.array_equal(runs[budget][0][m], runs[0][0][m]), (budget, m)
    G, out = runs[0]
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-5, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-5, e
    assert max_factor_rel(G, U) < 1e-4


def test_ccdpp_one_block_per_sm_sweeps_agree(ctx):
    """Later sweeps that stage one column of 32 KB or more and gather the
    other through L1 run as one 1024-thread block per SM: here the mode-1
    passes, which stage the 12,000-row column (48 KB) and gather the
    40,000-row one (FP32: 48 KB; FP64: 96 KB).  (The columns' first passes
    do not stage half packs: the two gathered modes' packs exceed a block's
    shared memory.)  In FP32 and FP64 the factors equal those of the run
    that stages nothing, bit for bit; the FP64 run matches the FP64 oracle
    to 1e-9 in RMSE and 1e-7 in the factors (this small, overfitted problem,
    whose 40,000-row mode has about 3 nonzeros a row against lambda 0.1,
    ends at a train RMSE near 0.06 and amplifies rounding: FP32 shows at
    1e-3 relative, FP64 factors at 5.5e-9)."""
    P = Problem(150000, (300, 12000, 40000), 16, seed=45)
    U, hist, _ = oracle_ccdpp(P, 2, 0.1, 2)
    for prec in (ctc.PREC_F32, ctc.PREC_F64):
        runs = {}
        for budget in (0, -1):
            runs[budget] = engine_run(ctx, P, ctc.CCDPP, 2, precision=prec, inner=2, tile_len=256,
                                      smem_budget=budget, **{"lambda": 0.1})
        for m in range(3):
            assert np.array_equal(runs[0][0][m], runs[-1][0][m]), (prec, m)
    G, out = runs[0]
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-9, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-9, e
    assert max_factor_rel(G, U) < 1e-7


# ------------------------------------------------------------------ SGD
def oracle_sgd(P, iters, lr, lam, scale=1.0, decay=1.0, trunc=False):
    U = P.factors()
    T = P.o_sorted(0)
    hist = [oracle_rmse(P, U)]
    for _ in range(iters):
        po.sgd_epoch(T, U, lr, lam, scale, trunc)
        lr *= decay
        hist.append(oracle_rmse(P, U))
    return U, hist


@pytest.mark.parametrize("R", [16, 32])
def test_sgd_sequential_f64(ctx, R):
    P = Problem(6000, (100, 80, 50), R, seed=11)
    U, hist = oracle_sgd(P, 3, 0.01, 0.01, decay=0.95)
    G, out = engine_run(ctx, P, ctc.SGD, 3, precision=ctc.PREC_F64, sgd_order=ctc.SGD_SEQUENTIAL,
                        lr=0.01, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95,
                        **{"lambda": 0.01})
    assert max_factor_rel(G, U) < 1e-9
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-9


def test_sgd_sequential_f32_trajectory(ctx):
    P = Problem(20000, (200, 150, 60), 32, seed=12)
    U, hist = oracle_sgd(P, 8, 0.01, 0.01, decay=0.95)
    G, out = engine_run(ctx, P, ctc.SGD, 8, precision=ctc.PREC_F32, sgd_order=ctc.SGD_SEQUENTIAL,
                        lr=0.01, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95,
                        **{"lambda": 0.01})
    for e, (tr, te) in enumerate(hist):
        assert abs(out.epochs[e]["rmse_tr"] - tr) / tr < 1e-3, e
        assert abs(out.epochs[e]["rmse_te"] - te) / te < 1e-3, e


@pytest.mark.parametrize("atomic,R", [(1, 32), (2, 32), (2, 8), (2, 64), (3, 8), (3, 32), (3, 64)])
def test_sgd_hogwild_final_rmse(ctx, atomic, R):
    """Hogwild with vector atomic adds (1), bulk row reductions from shared
    memory (2, the default) or block-merged hot rows (3): final test RMSE
    within 0.5 % of the deterministic sequential order."""
    P = Problem(200000, (2000, 1500, 200), R, seed=13)
    U, hist = oracle_sgd(P, 10, 0.01, 0.01, decay=0.95)
    G, out = engine_run(ctx, P, ctc.SGD, 10, precision=ctc.PREC_F32, sgd_order=ctc.SGD_HOGWILD,
                        sgd_atomic=atomic, lr=0.01, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY,
                        lr_decay=0.95, **{"lambda": 0.01})
    assert abs(out.epochs[-1]["rmse_te"] - hist[-1][1]) / hist[-1][1] < 0.005


@pytest.mark.parametrize("block,atomic,tpr", [(32, 2, 0), (128, 2, 0), (512, 2, 0), (1024, 3, 8), (1024, 3, 4)])
def test_sgd_hogwild_block_size(ctx, block, atomic, tpr):
    """ctc_params.threads_per_block (the reference GA's block-size gene)
    sets the Hogwild launch; every block size stays within 0.5 % of the
    sequential order (1024-thread blocks: the block-merged hot-row form,
    one or two 16-byte slices per lane)."""
    P = Problem(200000, (2000, 1500, 200), 32, seed=13)
    U, hist = oracle_sgd(P, 10, 0.01, 0.01, decay=0.95)
    G, out = engine_run(ctx, P, ctc.SGD, 10, precision=ctc.PREC_F32, sgd_order=ctc.SGD_HOGWILD,
                        sgd_atomic=atomic, threads_per_block=block, threads_per_row=tpr, lr=0.01, lr_scale=1.0,
                        lr_schedule=ctc.LR_EXP_DECAY, lr_decay=0.95, **{"lambda": 0.01})
    assert abs(out.epochs[-1]["rmse_te"] - hist[-1][1]) / hist[-1][1] < 0.005


def test_sgd_hogwild_plain_stores_stay_finite(ctx):
    """The store-based Hogwild variant (sgd_atomic=0) loses updates under
    contention -- it is kept as an option, not as a parity mode; it must
    still not increase the training error or produce non-finite values."""
    P = Problem(200000, (2000, 1500, 200), 32, seed=13)
    G, out = engine_run(ctx, P, ctc.SGD, 5, precision=ctc.PREC_F32, sgd_order=ctc.SGD_HOGWILD,
                        sgd_atomic=0, lr=0.01, lr_scale=1.0, lr_schedule=ctc.LR_EXP_DECAY,
                        lr_decay=0.95, **{"lambda": 0.01})
    assert out.epochs[-1]["rmse_tr"] <= out.epochs[0]["rmse_tr"]
    assert np.isfinite(out.epochs[-1]["rmse_te"])


def test_sgd_reference_defaults_bold_driver(ctx):
    """Reference constants: lr 1e-3, step scale 1e-5, lambda 1e-3, bold driver."""
    P = Problem(8000, (100, 90, 40), 16, seed=14)
    U = P.factors()
    T = P.o_sorted(0)
    lr, prev = 1e-3, None
    hist = []
    for e in range(4):
        if e > 0:
            po.sgd_epoch(T, U, lr, 1e-3, 1e-5, False)
        loss = po.sq_loss(T, U)
        obj = loss + po.frob(P.dims, U, 1e-3)
        hist.append(np.sqrt(loss / T.nnz))
        if e > 1:
            lr *= 1.05 if obj < prev else 0.5
        if e > 0:
            prev = obj
        else:
            prev = obj
    G, out = engine_run(ctx, P, ctc.SGD, 3, precision=ctc.PREC_F64, sgd_order=ctc.SGD_SEQUENTIAL)
    assert max_factor_rel(G, U) < 1e-9
    for e in range(4):
        assert abs(out.epochs[e]["rmse_tr"] - hist[e]) / hist[e] < 1e-9


# ------------------------------------------------------------------ adjoint
def test_grad_matches_oracle_and_finite_differences(ctx):
    P = Problem(3000, (40, 30, 20), 8, seed=15)
    lam = 0.05
    m = P.c_model()
    G, obj = ctc.grad(ctx, P.c_test() if False else ctc.Tensor.from_coo(*P.train, dims=P.dims), m, lam)
    U = P.factors()
    T = P.o_train()
    Go = po.grad(T, U, lam)
    assert max_factor_rel(G, Go) < 1e-9
    assert abs(obj - po.objective(T, U, lam)) / po.objective(T, U, lam) < 1e-10
    # central finite differences of the FP64 objective on a few coordinates
    rng = np.random.default_rng(0)
    h = 1e-5
    for _ in range(12):
        mode = int(rng.integers(3))
        r = int(rng.integers(P.dims[mode]))
        f = int(rng.integers(P.R))
        Up = [u.copy() for u in U]
        Um = [u.copy() for u in U]
        Up[mode][r, f] += h
        Um[mode][r, f] -= h
        fd = (po.objective(T, Up, lam) - po.objective(T, Um, lam)) / (2 * h)
        assert abs(fd - G[mode][r, f]) <= 1e-6 * max(1.0, abs(fd))


# ------------------------------------------------------------------ edge cases
def test_single_row_and_tiny(ctx):
    P = Problem(25, (1, 9, 8), 8, seed=16, test_frac=0.0)
    P.test = (P.train[0][:, :5], P.train[1][:5])
    U, hist = oracle_als(P, 2, 0.5)
    G, out = engine_run(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F64, **{"lambda": 0.5})
    assert max_factor_rel(G, U) < 1e-9


def test_rejects_bad_input(ctx):
    ind = np.array([[0, 1], [1, 1], [1, 2]], dtype=np.uint64)
    t = ctc.Tensor.from_coo(ind, [1.0, 2.0], dims=[2, 2, 2])
    m = ctc.Model([2, 2, 2], 8)
    with pytest.raises(ctc.CtcError) as e:
        ctc.run(ctx, [t], None, None, m, ctc.params("als", rank=8, iters=1))
    assert e.value.code == -1
    with pytest.raises(ctc.CtcError):
        ctc.run(ctx, [t], None, None, m, ctc.params("als", rank=12, iters=1))


@pytest.mark.parametrize("alg", ["als", "ccd", "ccdpp", "sgd"])
def test_rejects_out_of_range_indices_on_every_staging_path(ctx, alg):
    """Indices are range-checked in the staging pass that reads them (the
    record upload of every copy and of the test tensor): a bad index is an
    argument error before any kernel runs."""
    P = Problem(3000, (40, 30, 20), 8, seed=17)
    p = ctc.params(alg, rank=8, iters=1, lr=1e-3, lr_scale=1.0)
    ncopies = 1 if alg == "sgd" else 3

    def copies(bad_copy=None, mode=0, at=0, value=0):
        out = []
        for m in range(ncopies):
            ind, vals = P.sorted[m]
            ind = ind.copy()
            if m == bad_copy:
                ind[mode, at] = value
            out.append(ctc.Tensor.from_coo(ind, vals, dims=P.dims))
        return out

    ctc.run(ctx, copies(), None, P.c_test(), P.c_model(), p)  # well formed
    n = P.sorted[0][0].shape[1]
    cases = [copies(0, 1, n // 2, P.dims[1] + 1)]          # past mode 2's rows, middle of copy 1
    if ncopies == 3:
        cases.append(copies(2, 2, n - 1, P.dims[2] + 1))  # the last (largest) row of copy 3
        cases.append(copies(1, 0, 0, 0))                  # a 0 index (indices are 1-based)
    for train in cases:
        with pytest.raises(ctc.CtcError) as e:
            ctc.run(ctx, train, None, P.c_test(), P.c_model(), p)
        assert e.value.code == -1 and "1-based" in str(e.value)
    tind, tvals = P.test
    tind = tind.copy()
    tind[1, 0] = 0
    with pytest.raises(ctc.CtcError) as e:
        ctc.run(ctx, copies(), None, ctc.Tensor.from_coo(tind, tvals, dims=P.dims), P.c_model(), p)
    assert e.value.code == -1 and "test tensor" in str(e.value)


@pytest.mark.parametrize("alg,prec", [("ccdpp", ctc.PREC_F32), ("ccdpp", ctc.PREC_F64), ("als", ctc.PREC_F32),
                                      ("ccd", ctc.PREC_F64)])
def test_device_sorted_copies_match_host_sorted_copies(ctx, alg, prec):
    """train[0] alone: copies 2 and 3 are sorted on the device (stable by
    (mode, next mode), the order ctc_tensor_sort gives; CCD++ slots by the
    full key, the larger other mode first).  The training is the same, bit
    for bit, as with the three copies sorted on the host from train[0] and
    passed in."""
    P = Problem(60000, (300, 200, 100), 16, seed=19, heavy_row=3000)
    c0 = P.sorted[0]
    host = [c0] + [synth.sort_for_mode(*c0, m) for m in (1, 2)]
    p = ctc.params(alg, rank=16, iters=2, precision=prec, early_stop=0, eval_every=1, inner=2, **{"lambda": 0.1})
    m3, m1 = P.c_model(), P.c_model()
    o3 = ctc.run(ctx, [ctc.Tensor.from_coo(*h, dims=P.dims) for h in host], None, P.c_test(), m3, p)
    o1 = ctc.run(ctx, [ctc.Tensor.from_coo(*c0, dims=P.dims)], None, P.c_test(), m1, p)
    for a, b in zip(m3.factors(), m1.factors()):
        assert np.array_equal(a, b)
    assert [e["rmse_te"] for e in o3.epochs] == [e["rmse_te"] for e in o1.epochs]


def test_rejects_unsorted_copy(ctx):
    P = Problem(3000, (40, 30, 20), 8, seed=18)
    tr = P.sorted
    ind, vals = tr[1]
    ind, vals = ind[:, ::-1].copy(), vals[::-1].copy()  # mode-2 order reversed
    train = [ctc.Tensor.from_coo(*tr[0], dims=P.dims), ctc.Tensor.from_coo(ind, vals, dims=P.dims),
             ctc.Tensor.from_coo(*tr[2], dims=P.dims)]
    for alg in ("ccdpp", "als"):
        with pytest.raises(ctc.CtcError) as e:
            ctc.run(ctx, train, None, None, P.c_model(), ctc.params(alg, rank=8, iters=1))
        assert e.value.code == -1 and "not sorted" in str(e.value)


def test_checkpoint_resume_is_exact(ctx, tmp_path):
    """Two ALS iterations straight equal one iteration, a checkpoint
    (ctc_model_save / ctc_model_load) and one more iteration, bit for bit."""
    P = Problem(20000, (200, 150, 100), 16, seed=71)
    lam = {"lambda": 0.05}
    G2, _ = engine_run(ctx, P, ctc.ALS, 2, precision=ctc.PREC_F32, **lam)
    m = P.c_model()
    ctc.run(ctx, P.c_sorted(), None, P.c_test(), m, ctc.params(ctc.ALS, rank=16, iters=1, early_stop=0, **lam))
    path = str(tmp_path / "ck.ctcm")
    m.save(path)
    m2 = ctc.Model.load(path)
    ctc.run(ctx, P.c_sorted(), None, P.c_test(), m2, ctc.params(ctc.ALS, rank=16, iters=1, early_stop=0, **lam))
    for a, b in zip(m2.factors(), G2):
        assert np.array_equal(a, b)
