"""First-order path: the order-3/4 adjoint kernel against the FP64 numpy
restatement, central finite differences, torch.autograd.gradcheck and the
reference SGD's update direction; Adam training (full gradient and
minibatch, FP32 and BF16 gathers)."""
from __future__ import annotations

import numpy as np
import pytest

import cutc_b200 as ctc
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def order4(nnz, dims, R, seed=0, cp_rank=4, noise=0.05):
    rng = np.random.default_rng(seed)
    keys = set()
    cols = []
    while len(cols) < nnz:
        c = tuple(int(rng.integers(1, d + 1)) for d in dims)
        if c not in keys:
            keys.add(c)
            cols.append(c)
    ind = np.array(cols, dtype=np.uint64).T
    F = [rng.standard_normal((d, cp_rank)) for d in dims]
    v = np.ones((nnz, cp_rank))
    for m in range(len(dims)):
        v *= F[m][ind[m].astype(np.int64) - 1]
    v = v.sum(1)
    v = 1.0 + 4.0 * (v - v.min()) / (v.max() - v.min()) + noise * rng.standard_normal(nnz)
    U = [rng.uniform(0, 1, (d, R)) / np.sqrt(R) for d in dims]
    return ind, v, U


def model_of(dims, U):
    m = ctc.Model(dims, U[0].shape[1])
    m.set_factors(U)
    return m


@pytest.mark.parametrize("R", [8, 16, 64])
def test_adjoint_order4_matches_numpy_and_fd(ctx, R):
    dims = (30, 25, 20, 6)
    ind, v, U = order4(10000, dims, R, seed=R)
    t = ctc.Tensor.from_coo(ind, v, dims=dims)
    lam = 0.05
    G, obj = ctc.grad(ctx, t, model_of(dims, U), lam)
    Gr = po.cp_grad(ind, v, U, lam)
    assert abs(obj - po.cp_objective(ind, v, U, lam)) / obj < 1e-12
    for g, gr in zip(G, Gr):
        assert np.max(np.abs(g - gr)) / np.max(np.abs(gr)) < 1e-10
    # central finite differences (FP64) on random coordinates of every mode
    rng = np.random.default_rng(7)
    h = 1e-6
    for m in range(4):
        for _ in range(4):
            r, c = int(rng.integers(dims[m])), int(rng.integers(R))
            Up = [u.copy() for u in U]
            Um = [u.copy() for u in U]
            Up[m][r, c] += h
            Um[m][r, c] -= h
            _, fp = ctc.grad(ctx, t, model_of(dims, Up), lam)
            _, fm = ctc.grad(ctx, t, model_of(dims, Um), lam)
            fd = (fp - fm) / (2 * h)
            assert abs(fd - G[m][r, c]) <= 1e-5 * max(1.0, abs(fd)), (m, r, c, fd, G[m][r, c])


def test_autograd_gradcheck(ctx):
    torch = pytest.importorskip("torch")
    from cutc_b200.autograd import masked_cp_loss
    dims = (6, 5, 4, 3)
    ind, v, U = order4(150, dims, 8, seed=3)
    t = ctc.Tensor.from_coo(ind, v, dims=dims)
    factors = [torch.tensor(u, dtype=torch.float64, requires_grad=True) for u in U]
    assert torch.autograd.gradcheck(lambda *f: masked_cp_loss(t, ctx, 0.1, *f), factors, eps=1e-6, atol=1e-6)


def test_adjoint_is_the_reference_sgd_direction(ctx):
    """One nonzero, one sequential SGD epoch of the reference rule
    (sgpu/sgd.cu:92-99: every row from the same pre-update snapshot): the
    step is -lr * scale * grad of 1/2 e^2 + (lambda/2) ||U||^2 on the rows
    the nonzero touches."""
    dims = (5, 4, 3)
    R = 16
    rng = np.random.default_rng(11)
    ind = np.array([[3], [2], [1]], dtype=np.uint64)
    v = np.array([4.2])
    U = [rng.uniform(0, 1, (d, R)) for d in dims]
    lr, lam, scale = 0.01, 0.3, 1.0
    Us = [u.copy() for u in U]
    po.sgd_epoch(po.Tensor(ind, v, dims=dims), Us, lr, lam, scale, False)
    t = ctc.Tensor.from_coo(ind, v, dims=dims)
    G, _ = ctc.grad(ctx, t, model_of(dims, U), lam / 2)
    for m in range(3):
        r = int(ind[m, 0]) - 1
        step = Us[m][r] - U[m][r]
        assert np.max(np.abs(step + lr * scale * G[m][r])) < 1e-12, m


def test_fo_full_gradient_decreases_loss(ctx):
    dims = (60, 50, 40, 8)
    ind, v, U = order4(20000, dims, 16, seed=21)
    n = ind.shape[1]
    te = np.arange(n) % 10 == 0
    tr = ctc.Tensor.from_coo(ind[:, ~te], v[~te], dims=dims)
    ts = ctc.Tensor.from_coo(ind[:, te], v[te], dims=dims)
    p = ctc.fo_params(rank=16, lr=0.01, batch=0, epochs=30, eval_every=1, **{"lambda": 1e-3})
    F = ctc.FirstOrder(ctx, tr, ts, p)
    m = model_of(dims, U)
    out = F.run(m, p)
    loss = [e["loss"] + e["frob"] for e in out.epochs]
    assert len(loss) == 31
    # one Adam step per epoch on the exact gradient: a steady descent
    assert loss[-1] < 0.75 * loss[0]
    assert all(b < a for a, b in zip(loss[:10], loss[1:11]))


def test_fo_minibatch_mixed_matches_fp32(ctx):
    dims = (200, 150, 100, 12)
    ind, v, U = order4(60000, dims, 16, seed=31)
    n = ind.shape[1]
    te = np.arange(n) % 10 == 0
    tr = ctc.Tensor.from_coo(ind[:, ~te], v[~te], dims=dims)
    ts = ctc.Tensor.from_coo(ind[:, te], v[te], dims=dims)
    res = {}
    for prec in (ctc.PREC_F32, ctc.PREC_MIXED):
        p = ctc.fo_params(rank=16, precision=prec, lr=0.01, batch=4096, epochs=8, eval_every=0,
                          **{"lambda": 1e-4})
        F = ctc.FirstOrder(ctx, tr, ts, p)
        m = model_of(dims, U)
        out = F.run(m, p)
        res[prec] = out.epochs[-1]["rmse_te"]
        assert out.epochs[-1]["rmse_te"] < out.epochs[0]["rmse_te"] * 0.5
        F.free()
    assert abs(res[ctc.PREC_MIXED] - res[ctc.PREC_F32]) / res[ctc.PREC_F32] < 0.005, res


def test_fo_order3(ctx):
    from tests.helpers import Problem
    P = Problem(20000, (100, 80, 60), 16, seed=41)
    p = ctc.fo_params(rank=16, lr=0.02, batch=2048, epochs=6, **{"lambda": 1e-3})
    F = ctc.FirstOrder(ctx, ctc.Tensor.from_coo(*P.train, dims=P.dims), P.c_test(), p)
    out = F.run(P.c_model(), p)
    assert out.epochs[-1]["rmse_te"] < out.epochs[0]["rmse_te"]
