"""ctc_sse_noalloc: the squared-error sum for callers that cannot allocate
device memory (their GPU memory is owned by another allocator, or they
cannot take an allocation's synchronisation).  Called through the C ABI on
nonzeros and factors that the test places on the device, and checked
against the allocating entry point ctc_rmse on the same tensor, within the
RMSE tolerance of the other GPU tests, on two calls in a row.  This file is
collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import api
from tests.helpers import Problem

pytestmark = pytest.mark.gpu


def _device_inputs(P, model):
    import torch
    ind, vals = P.test
    rec = np.empty((ind.shape[1], 4), dtype=np.uint32)
    rec[:, :3] = (ind - 1).T.astype(np.uint32)
    rec[:, 3] = vals.astype(np.float32).view(np.uint32)
    d_rec = torch.from_numpy(rec.view(np.int32)).cuda()
    d_U = [torch.from_numpy(u.astype(np.float32)).cuda().contiguous() for u in model.factors()]
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    return d_rec, d_U, d_out


@pytest.mark.parametrize("R", [16, 32])
def test_noalloc_sse_matches_rmse_entry_point(ctx, R):
    import torch
    P = Problem(60000, (400, 300, 50), R, seed=21, test_frac=0.5)
    model = P.c_model()
    want = ctc.rmse(ctx, P.c_test(), model)
    d_rec, d_U, d_out = _device_inputs(P, model)
    n = d_rec.shape[0]
    for call in range(2):
        d_out.zero_()
        rc = api.lib().ctc_sse_noalloc(C.c_void_p(d_rec.data_ptr()), n, C.c_void_p(d_U[0].data_ptr()),
                                       C.c_void_p(d_U[1].data_ptr()), C.c_void_p(d_U[2].data_ptr()), R,
                                       C.c_void_p(d_out.data_ptr()), None)
        assert rc == 0, api.lib().ctc_last_error()
        torch.cuda.synchronize()
        got = float(np.sqrt(d_out.item() / n))
        assert abs(got - want) / want < 1e-5, (call, got, want)
