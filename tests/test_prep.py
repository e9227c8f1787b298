"""Seeded data preparation against the reference's own scripts: the bytes
tvtensor.py and stensor.py wrote (with random.seed fixed, fixtures made by
tests/golden/prep/make_prep_golden.py) equal what cutc_b200.prep writes through
the C ABI (ctc_tensor_split, ctc_tensor_sort, ctc_tensor_write_tns).  Also
the SPLATT binary form of the reference's .bin path: its header layout,
narrow and wide words, and round trips."""
import os
import struct

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import prep

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "prep", "prep.npz")


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


@pytest.mark.parametrize("which", [0, 1])
def test_tvtensor_and_stensor_bytes_match_reference_scripts(golden, tmp_path, which):
    seed = int(golden["seeds"][which])
    src = tmp_path / "in.tns"
    src.write_bytes(golden["input"].tobytes())
    paths = prep.tvtensor(str(src), str(tmp_path), "x", seed)
    paths.update(prep.stensor(paths["_tr"], str(tmp_path), "x"))
    for suffix in ("_tr", "_v", "_te", "_tr2", "_tr3"):
        got = open(paths[suffix], "rb").read()
        want = golden[f"{seed}{suffix}"].tobytes()
        assert got == want, suffix


def test_split_is_a_partition_in_ij_order(golden, tmp_path):
    src = tmp_path / "in.tns"
    src.write_bytes(golden["input"].tobytes())
    t = ctc.Tensor.load(str(src))
    ind, vals = t.export()
    parts = t.split(3)
    sizes = [p.nnz for p in parts]
    assert sum(sizes) == t.nnz
    # about 80 / 10 / 10
    assert 0.75 < sizes[0] / t.nnz < 0.85
    for p in parts:
        pi, _ = p.export()
        key = pi[0].astype(object) * (1 << 20) + pi[1].astype(object)
        assert all(a <= b for a, b in zip(key[:-1], key[1:]))
    # another seed gives another split
    assert [p.nnz for p in t.split(4)] != sizes or not np.array_equal(parts[1].export()[1], t.split(4)[1].export()[1])


def test_write_tns_round_trip_and_formats(tmp_path):
    rng = np.random.default_rng(1)
    ind = rng.integers(1, 1000, (3, 5000)).astype(np.uint64)
    vals = rng.standard_normal(5000) * 1e3
    t = ctc.Tensor.from_coo(ind, vals)
    p17 = str(tmp_path / "a.tns")
    t.write_tns(p17)
    i2, v2 = ctc.Tensor.load(p17).export()
    assert np.array_equal(i2, ind) and np.array_equal(v2, vals)
    p1 = str(tmp_path / "b.tns")
    t.write_tns(p1, 1)
    lines = open(p1).read().splitlines()
    assert lines[0] == "%d %d %d %.1f" % (ind[0, 0], ind[1, 0], ind[2, 0], vals[0])
    assert len(lines) == 5000


def test_splatt_bin_reads_the_reference_writer_layout(tmp_path):
    """The layout tt_write_binary_file writes (sgpu/io.c:347-431): magic 0,
    idx_width 8, val_width 4 (float values), u64 nmodes, dims, nnz, index
    arrays -- which the reference's own reader rejects."""
    rng = np.random.default_rng(2)
    n = 1000
    ind = rng.integers(1, 500, (3, n)).astype(np.uint64)
    vals = rng.uniform(1, 5, n)
    dims = [600, 510, 505]
    raw = struct.pack("<iQQ", 0, 8, 4) + struct.pack("<QQQQQ", 3, *dims, n)
    raw += ind.tobytes() + vals.astype(np.float32).tobytes()
    p = tmp_path / "ref.bin"
    p.write_bytes(raw)
    t = ctc.Tensor.load(str(p))
    i2, v2 = t.export()
    assert t.dims == dims
    assert np.array_equal(i2, ind)
    assert np.array_equal(v2, vals.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("wide_idx,wide_val", [(False, False), (True, False), (False, True), (True, True)])
def test_splatt_bin_round_trip(tmp_path, wide_idx, wide_val):
    rng = np.random.default_rng(3)
    n = 3000
    ind = rng.integers(1, 800, (3, n)).astype(np.uint64)
    if wide_idx:
        ind[0, 5] = (1 << 33) + 7
    vals = rng.integers(1, 6, n).astype(np.float64)
    if wide_val:
        vals[7] = 1.0 / 3.0
    t = ctc.Tensor.from_coo(ind, vals)
    p = str(tmp_path / "t.bin")
    t.save_splatt(p)
    head = open(p, "rb").read(20)
    magic, iw, vw = struct.unpack("<iQQ", head)
    assert (magic, iw, vw) == (0, 8 if wide_idx else 4, 8 if wide_val else 4)
    t2 = ctc.Tensor.load(p)
    i2, v2 = t2.export()
    assert np.array_equal(i2, ind) and np.array_equal(v2, vals)
    assert t2.dims == t.dims


def test_splatt_bin_rejects_truncated_and_oversized(tmp_path):
    ind = np.ones((3, 10), dtype=np.uint64)
    t = ctc.Tensor.from_coo(ind, np.ones(10))
    p = str(tmp_path / "t.bin")
    t.save_splatt(p)
    raw = open(p, "rb").read()
    cut = tmp_path / "cut.bin"
    cut.write_bytes(raw[:-3])
    with pytest.raises(ctc.CtcError) as e:
        ctc.Tensor.load(str(cut))
    assert e.value.code == -2
    # a header claiming 2^40 nonzeros is rejected before anything is sized
    big = bytearray(raw)
    off = 20 + 4 * 4  # magic, widths, nmodes and three dims (4-byte words)
    big[off:off + 4] = struct.pack("<I", 0xFFFFFFF0)
    (tmp_path / "big.bin").write_bytes(bytes(big))
    with pytest.raises(ctc.CtcError) as e:
        ctc.Tensor.load(str(tmp_path / "big.bin"))
    assert e.value.code == -2


def test_ctcb_rejects_oversized_nnz_header(tmp_path):
    ind = np.ones((3, 10), dtype=np.uint64)
    t = ctc.Tensor.from_coo(ind, np.ones(10))
    p = str(tmp_path / "t.ctcb")
    t.save_bin(p)
    raw = bytearray(open(p, "rb").read())
    raw[12:20] = struct.pack("<Q", 1 << 40)
    (tmp_path / "big.ctcb").write_bytes(bytes(raw))
    with pytest.raises(ctc.CtcError) as e:
        ctc.Tensor.load(str(tmp_path / "big.ctcb"))
    assert e.value.code == -2 and "not a valid CTCB" in str(e.value)


def test_splatt_bin_written_by_the_reference_reads_as_its_tns(tmp_path):
    """A .bin file written by the reference's own tt_write_binary (built
    from its sources into oracle/_ref) loads with the indices and dims of
    the .tns it came from, and its values as the float the reference
    stores (its header writer always picks 4-byte values)."""
    from oracle import pyoracle as po
    if not po.ref_host_available():
        pytest.skip("reference host library not built")
    rng = np.random.default_rng(4)
    n = 2000
    ind = np.stack([rng.integers(1, d + 1, n) for d in (300, 200, 50)]).astype(np.uint64)
    vals = np.round(rng.uniform(1, 5, n), 3)
    src = str(tmp_path / "t.tns")
    po.write_tns(src, po.Tensor(ind, vals, dims=[300, 200, 50]))
    out = str(tmp_path / "t.bin")
    po.ref_tns_to_bin(src, out)
    magic, iw, vw = struct.unpack("<iQQ", open(out, "rb").read(20))
    assert (magic, iw, vw) == (0, 8, 4)
    tb = ctc.Tensor.load(out)
    tt = ctc.Tensor.load(src)
    ib, vb = tb.export()
    it, vt = tt.export()
    assert np.array_equal(ib, it)
    assert tb.dims == tt.dims
    assert np.array_equal(vb, vt.astype(np.float32).astype(np.float64))
