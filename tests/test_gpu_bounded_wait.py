"""The bounded-wait error path, exercised without a fault: a self-test
kernel waits on a barrier that nothing arrives at, with the bounded wait
the tensor-core Gram and the CCD++ pass use.  The wait gives up after a
short limit, the kernel records the error flag and returns, and the host
reports CTC_E_TIMEOUT once; the context and the dataset stay usable."""
import pytest

import cutc_b200 as ctc
from tests.helpers import Problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alg", ["ccdpp", "als"])
def test_bounded_wait_expires_reports_once_and_clears(ctx, alg):
    P = Problem(5000, (60, 50, 40), 16, seed=3)
    p = ctc.params(alg, rank=16, iters=1, early_stop=0, **{"lambda": 0.1})
    ds = ctc.Dataset(ctx, P.c_sorted(), None, P.c_test(), p)
    ds.set_model(P.c_model())
    base = ds.evaluate()
    ds.probe_wait(50_000_000)  # 50 ms
    with pytest.raises(ctc.CtcError) as e:
        ds.evaluate()
    assert e.value.code == -7 and "self-test" in str(e.value)
    # reported once: the next evaluation succeeds with the same model
    again = ds.evaluate()
    assert again["rmse_te"] == base["rmse_te"]
    # the dataset still trains
    ds.epochs(1)
    assert ds.evaluate()["rmse_tr"] < base["rmse_tr"]
    # staging a model clears a pending flag too
    ds.probe_wait(50_000_000)
    ds.set_model(P.c_model())
    assert ds.evaluate()["rmse_te"] == base["rmse_te"]
    ds.free()


def test_probe_wait_rejects_bad_limit(ctx):
    P = Problem(2000, (30, 20, 10), 8, seed=4)
    p = ctc.params("als", rank=8, iters=1, early_stop=0)
    ds = ctc.Dataset(ctx, P.c_sorted(), None, None, p)
    with pytest.raises(ctc.CtcError):
        ds.probe_wait(1000)  # no model staged yet
    ds.set_model(P.c_model())
    for bad in (0, 3_000_000_000):
        with pytest.raises(ctc.CtcError) as e:
            ds.probe_wait(bad)
        assert e.value.code == -1
    ds.free()
