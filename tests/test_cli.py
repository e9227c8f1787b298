"""The `tc` command line (cutc_b200/tc), the reference driver's surface
(sgpu/tc.c:17-60: `tc traina trainb trainc validation test`, progress line
of sgpu/completion.c:111-113 plus RMSE-te and the epoch's device time), on
five .tns files prepared the reference's way (a seeded tvtensor split and
the stensor mode-2 / mode-3 copies).  The argument checks run on the CPU;
a run needs the GPU."""
import os
import re
import subprocess

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import prep, synth
from oracle import pyoracle as po

TC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cutc_b200", "tc")
LINE = re.compile(r"^epoch:(\d+)   loss: (\S+)   RMSE-tr: (\S+)   RMSE-vl: (\S+)   RMSE-te: (\S+)   ms: (\S+)$")


def five_files(tmp_path, nnz=30000, dims=(300, 200, 60), seed=3):
    ind, vals = synth.random_small(nnz, dims, seed=seed)
    src = str(tmp_path / "data.tns")
    ctc.Tensor.from_coo(ind, vals, dims=dims).write_tns(src, 2)
    paths = prep.tvtensor(src, str(tmp_path), "data", seed)
    paths.update(prep.stensor(paths["_tr"], str(tmp_path), "data"))
    return [paths[k] for k in ("_tr", "_tr2", "_tr3", "_v", "_te")]


def run_tc(args, timeout=600):
    return subprocess.run([TC, *args], capture_output=True, text=True, timeout=timeout)


def test_cli_usage_and_argument_errors(tmp_path):
    assert os.path.exists(TC), "build the CLI with python -m cutc_b200.build"
    r = run_tc([])
    assert r.returncode == 2 and "usage: tc traina.tns" in r.stderr
    files = five_files(tmp_path, nnz=2000)
    r = run_tc([*files, "--alg", "nope"])
    assert r.returncode == 2
    r = run_tc([*files, "--precision", "f16"])
    assert r.returncode == 2
    r = run_tc([files[0], files[1], files[2], str(tmp_path / "missing.tns"), files[4]])
    assert r.returncode == 1 and "missing.tns" in r.stderr
    # parameters are checked before a device is touched
    r = run_tc([*files, "--rank", "12"])
    assert r.returncode == 1 and "rank 12" in r.stderr
    r = run_tc([*files, "--threads-per-block", "16"])
    assert r.returncode == 1 and "threads_per_block" in r.stderr


@pytest.mark.gpu
def test_cli_als_run_prints_the_reference_progress_line(tmp_path):
    """ALS, FP64, rank 16, 3 iterations: one progress line per epoch (0 =
    the starting point), in the reference's format with RMSE-te added; the
    printed training and validation RMSEs equal the FP64 oracle's on the
    same seeded initial factors (ctc_model_init_uniform, seed 5) to the 6
    printed digits; the factor files have one line per row."""
    files = five_files(tmp_path)
    prefix = str(tmp_path / "fac")
    r = run_tc([*files, "--alg", "als", "--rank", "16", "--lambda", "0.05", "--iters", "3", "--no-early-stop",
                "--precision", "f64", "--seed", "5", "--write-factors", prefix])
    assert r.returncode == 0, r.stderr
    lines = [LINE.match(x) for x in r.stdout.splitlines() if x.startswith("epoch:")]
    assert len(lines) == 4 and all(lines)
    assert [int(m.group(1)) for m in lines] == [0, 1, 2, 3]
    assert "best epoch" in r.stdout
    # oracle: the same tensors and initial factors
    t = [ctc.Tensor.load(f) for f in files]
    dims = [max(x.dims[m] for x in t) for m in range(3)]
    model = ctc.Model(dims, 16).init_uniform(5, 1.0 / np.sqrt(16))
    U = model.factors()
    T = [po.Tensor(*x.export(), dims=dims) for x in t]
    for e, m in enumerate(lines):
        if e > 0:
            for mode in range(3):
                po.als_mode(T[mode], mode, U, 0.05)
        tr, vl = po.rmse(T[0], U), po.rmse(T[3], U)
        assert abs(float(m.group(3)) - tr) / tr < 1e-5, (e, m.group(3), tr)
        assert abs(float(m.group(4)) - vl) / vl < 1e-5, (e, m.group(4), vl)
    for mode in range(3):
        rows = open(f"{prefix}{mode + 1}.txt").read().splitlines()
        assert len(rows) == dims[mode] and len(rows[0].split()) == 16


@pytest.mark.gpu
@pytest.mark.parametrize("alg", ["sgd", "ccdpp", "ccd"])
def test_cli_other_algorithms_run(tmp_path, alg):
    files = five_files(tmp_path, nnz=20000)
    r = run_tc([*files, "--alg", alg, "--iters", "2", "--no-early-stop"])
    assert r.returncode == 0, r.stderr
    lines = [LINE.match(x) for x in r.stdout.splitlines() if x.startswith("epoch:")]
    assert len(lines) == 3 and all(lines)
    assert all(np.isfinite(float(m.group(3))) for m in lines)
