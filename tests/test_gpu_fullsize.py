"""Properties at the full size of the 100M-nonzero workload (500,000 x
20,000 x 2,000 Zipf(1.1), 90M training nonzeros, R = 32), where the FP64
oracle would take too long.  Each compares two computations that must
agree exactly or to FP32 rounding:

  * the device CISS builder against the host builder (bit for bit), for
    a sorted copy and for the unsorted tensor sorted on the device;
  * CCD++ staged from the mode-1 tensor alone against the three host-sorted
    copies (bit for bit: the slots are ordered by the full key either way);
  * the training RMSE a CCD++ run reports from its residuals against the
    squared-error kernel over the records (ctc_rmse);
  * one ALS iteration in FP32 against FP64 (test RMSE)."""
from __future__ import annotations

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import synth

pytestmark = pytest.mark.gpu


def _sorted_copies(ind, vals, dims):
    """Stable sorts by (mode m, mode m+1) on the GPU (the order of the
    reference's traina/b/c files)."""
    import torch
    ti = torch.from_numpy(ind.astype(np.int64)).cuda()
    out = []
    for m in range(3):
        key = ti[m] * (dims[(m + 1) % 3] + 1) + ti[(m + 1) % 3]
        _, order = torch.sort(key, stable=True)
        o = order.cpu().numpy()
        out.append((np.ascontiguousarray(ind[:, o]), np.ascontiguousarray(vals[o])))
        del key, order
    del ti
    torch.cuda.empty_cache()
    return out


@pytest.fixture(scope="module")
def big():
    w = synth.WORKLOADS["zipf-100m"]
    data = synth.generate(w, seed=0, device="cuda")
    ind, vals = data["train"]
    copies = _sorted_copies(ind, vals, w.dims)
    out = dict(w=w, n=int(vals.size),
               tr=[ctc.Tensor.from_coo(i, v, dims=w.dims) for i, v in copies],
               te=ctc.Tensor.from_coo(*data["test"], dims=w.dims),
               unsorted=ctc.Tensor.from_coo(ind, vals, dims=w.dims))
    del data, copies
    yield out


def _same_ciss(a, b):
    assert a["nnz"] == b["nnz"] and a["dlength"] == b["dlength"] and a["size_rows"] == b["size_rows"]
    assert np.array_equal(a["directory"], b["directory"]) and np.array_equal(a["dcounter"], b["dcounter"])
    assert np.array_equal(a["written"], b["written"])
    w = a["written"]
    assert np.array_equal(a["entries"].view(np.uint64)[w], b["entries"].view(np.uint64)[w])


def test_fullsize_ciss_device_equals_host(ctx, big):
    host = ctc.ciss_alloc(big["tr"][0], 1, 32)
    _same_ciss(host, ctc.ciss_alloc_gpu(ctx, big["tr"][0], 1, 32))
    # the unsorted tensor, sorted on the device: the host-sorted copy's CISS
    _same_ciss(host, ctc.ciss_alloc_gpu(ctx, big["unsorted"], 1, 32, sort=True))


def test_fullsize_ccdpp_one_tensor_equals_three_copies(ctx, big):
    w = big["w"]
    p = ctc.params("ccdpp", rank=w.rank, inner=3, iters=1, early_stop=0, eval_every=1, **{"lambda": 0.1})
    m3 = ctc.Model(w.dims, w.rank).init_uniform(1, 1.0 / np.sqrt(w.rank))
    m1 = ctc.Model(w.dims, w.rank).init_uniform(1, 1.0 / np.sqrt(w.rank))
    o3 = ctc.run(ctx, big["tr"], None, big["te"], m3, p)
    o1 = ctc.run(ctx, [big["tr"][0]], None, big["te"], m1, p)
    for a, b in zip(m3.factors(), m1.factors()):
        assert np.array_equal(a, b)
    assert [e["rmse_te"] for e in o3.epochs] == [e["rmse_te"] for e in o1.epochs]
    # the run's training RMSE (from the CCD++ residuals) against the
    # squared-error kernel over the records with the same factors
    tr_run = o1.epochs[-1]["rmse_tr"]
    tr_sse = ctc.rmse(ctx, big["tr"][0], m1)
    assert abs(tr_run - tr_sse) / tr_sse < 1e-5, (tr_run, tr_sse)
    assert o1.epochs[-1]["rmse_te"] < 0.5 * o1.epochs[0]["rmse_te"]


def test_fullsize_als_f32_tracks_f64(ctx, big):
    w = big["w"]
    te = []
    for prec in (ctc.PREC_F64, ctc.PREC_F32):
        p = ctc.params("als", rank=w.rank, iters=1, early_stop=0, eval_every=1, precision=prec,
                       **{"lambda": 0.1})
        m = ctc.Model(w.dims, w.rank).init_uniform(1, 1.0 / np.sqrt(w.rank))
        te.append(ctc.run(ctx, [big["tr"][0]], None, big["te"], m, p).epochs[-1]["rmse_te"])
    assert abs(te[1] - te[0]) / te[0] < 1e-5, te
