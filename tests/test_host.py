"""Host-side behaviour of libctc and of the oracle, CPU only: exports, error
codes, tensor I/O round trips, sorting, seeded model init, and the oracle's
own consistency (gradient vs finite differences, monotone ALS / CCD++)."""
import os
import re

import numpy as np
import pytest

import cutc_b200 as ctc
from cutc_b200 import api, synth
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    declared = api._declared_names()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(api.lib(), n)]
    assert not missing, missing


def test_declared_entry_points_cite_reference_or_say_none():
    txt = open(os.path.join(ROOT, "include", "ctc.h")).read()
    assert "sgpu/" in txt and "ga/ciss.c" in txt


def test_error_codes_without_crash(tmp_path):
    with pytest.raises(ctc.CtcError) as e:
        ctc.tt_read(str(tmp_path / "missing.tns"))
    assert e.value.code == -2
    t = ctc.Tensor.from_coo(np.ones((3, 4), dtype=np.uint64), np.ones(4))
    with pytest.raises(ctc.CtcError) as e:
        ctc.ciss_alloc(t, 1, 0)
    assert e.value.code == -1
    with pytest.raises(ctc.CtcError):
        ctc.ciss_alloc(t, 4, 32)


def test_context_without_gpu_is_an_error_not_a_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ctc.CtcError) as e:
        ctc.Context(0)
    assert e.value.code == -8


def test_coo_roundtrip_and_dims():
    ind, vals = synth.random_small(500, (30, 20, 10), seed=1)
    t = ctc.Tensor.from_coo(ind, vals)
    nm, nnz, dims = t.info()
    assert (nm, nnz) == (3, 500)
    assert dims == [int(ind[m].max()) for m in range(3)]
    i2, v2 = t.export()
    assert np.array_equal(i2, ind) and np.array_equal(v2, vals)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_sort_is_stable_lexsort(mode):
    ind, vals = synth.random_small(3000, (9, 8, 7), seed=2, distinct=False)
    t = ctc.Tensor.from_coo(ind, vals).sort(mode)
    i2, v2 = t.export()
    si, sv = synth.sort_for_mode(ind, vals, mode)
    assert np.array_equal(i2, si) and np.array_equal(v2, sv)


def test_binary_roundtrip(tmp_path):
    ind, vals = synth.random_small(777, (50, 40, 30), seed=3)
    t = ctc.Tensor.from_coo(ind, vals, dims=[60, 40, 30])
    p = str(tmp_path / "x.ctcb")
    t.save_bin(p)
    t2 = ctc.tt_read(p)
    assert t2.dims == [60, 40, 30]
    i2, v2 = t2.export()
    assert np.array_equal(i2, ind) and np.array_equal(v2, vals)
    (tmp_path / "bad.ctcb").write_bytes(b"CTCX0000")
    with pytest.raises(ctc.CtcError):
        ctc.tt_read(str(tmp_path / "bad.ctcb"))


def test_binary_large_roundtrip_and_truncation(tmp_path):
    """A file read by byte ranges on the host threads: exact round trip; a
    truncated file is rejected."""
    rng = np.random.default_rng(9)
    n = 600_000
    ind = np.stack([rng.integers(1, d + 1, n) for d in (900, 800, 700)]).astype(np.uint64)
    vals = rng.standard_normal(n)
    p = str(tmp_path / "big.ctcb")
    ctc.Tensor.from_coo(ind, vals).save_bin(p)
    i2, v2 = ctc.tt_read(p).export()
    assert np.array_equal(i2, ind) and np.array_equal(v2.view(np.uint64), vals.view(np.uint64))
    q = tmp_path / "cut.ctcb"
    q.write_bytes(open(p, "rb").read()[:-8])
    with pytest.raises(ctc.CtcError):
        ctc.tt_read(str(q))


def test_tns_reader_large_parallel_matches_oracle(tmp_path):
    """A file big enough for the parallel chunked parse (> 1 MiB)."""
    ind, vals = synth.random_small(60000, (500, 400, 300), seed=4)
    p = str(tmp_path / "big.tns")
    po.write_tns(p, po.Tensor(ind, vals))
    a = ctc.tt_read(p)
    b = po.tns_read(p)
    ia, va = a.export()
    assert np.array_equal(ia, b.ind) and np.array_equal(va.view(np.uint64), b.vals.view(np.uint64))
    assert a.dims == b.dims


_TOKEN_LINES = [
    "1 2 3 4.5", "# a comment", "", "  7\t8 9 1e5", "+3 4 5 +2.5", "10 11 12 0x1p3", "2 3 4 -0.0",
    "5 6 7 .25\r", "18446744073709551615 1 1 3", "4 5 6 1.7976931348623157e308", "4 5 6 4.9e-324",
    "6 6 6 1e-400", "7 7 7 inf", "7 7 8 -nan", "8 9 10 12abc", "3 4 5 1.5e", "9 9 9 0.1000000000000000055511151231257827",
    "1 1 1 123456789012345678901234567890", "2 2 2 -3.25E-2",
]


def _reference_parse(lines, nmodes):
    """Each data line through libc's strtoul / strtod, chained as the
    reference's reader chains them (sgpu/io.c:58-106)."""
    import ctypes as C
    libc = C.CDLL(None)
    libc.strtoul.restype, libc.strtod.restype = C.c_ulong, C.c_double
    libc.strtoul.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_int]
    libc.strtod.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    ind, vals = [], []
    for line in lines:
        if len(line) + 1 <= 1 or line.startswith("#"):
            continue
        buf = C.create_string_buffer(line.encode())
        ptr = C.c_void_p(C.addressof(buf))
        row = []
        for _ in range(nmodes):
            end = C.c_void_p()
            row.append(libc.strtoul(ptr, C.byref(end), 10))
            ptr = end
        end = C.c_void_p()
        vals.append(libc.strtod(ptr, C.byref(end)))
        ind.append(row)
    return np.array(ind, dtype=np.uint64).T, np.array(vals, dtype=np.float64)


@pytest.mark.parametrize("repeat", [1, 40000])
def test_tns_token_forms_parse_as_strtoul_strtod(tmp_path, repeat):
    """Blanks, tabs, signs, hex floats, CRLF, overflow, subnormals,
    underflow, inf / nan and tokens glued to text: the reader's values equal
    libc's strtoul / strtod bit for bit (repeat = 40000 makes the file large
    enough for the chunked parallel parse)."""
    p = tmp_path / "forms.tns"
    p.write_bytes(("\n".join(_TOKEN_LINES * repeat) + "\n").encode())
    a = ctc.tt_read(str(p))
    ia, va = a.export()
    ib, vb = _reference_parse(_TOKEN_LINES * repeat, 3)
    assert np.array_equal(ia, ib)
    assert np.array_equal(va.view(np.uint64), vb.view(np.uint64))


def test_tns_first_line_token_rule(tmp_path):
    """The mode count comes from strtok on the first data line, so trailing
    whitespace there adds a mode (sgpu/io.c:249-257) -- in both readers."""
    p = tmp_path / "ws.tns"
    p.write_text("1 2 3 4.5 \n2 1 1 1.0\n")
    a, b = ctc.tt_read(str(p)), po.tns_read(str(p))
    assert a.info()[0] == b.nmodes == 4


def test_model_init_is_seeded_and_bounded():
    m1 = ctc.Model([100, 80, 60], 16).init_uniform(42, 0.25)
    m2 = ctc.Model([100, 80, 60], 16).init_uniform(42, 0.25)
    m3 = ctc.Model([100, 80, 60], 16).init_uniform(43, 0.25)
    for a, b, c in zip(m1.factors(), m2.factors(), m3.factors()):
        assert np.array_equal(a, b)
        assert not np.array_equal(a, c)
        assert a.min() >= 0 and a.max() < 0.25
    assert abs(np.mean(m1.get(0)) - 0.125) < 0.01


def test_params_reference_defaults():
    p = ctc.params("als")
    assert (p.rank, p.lambda_, p.iters, p.max_bad_epochs) == (16, 10.0, 1000, 3)
    assert abs(p.tolerance - 1e-4) < 1e-12
    assert ctc.params("sgd").lambda_ == 1e-3 and ctc.params("sgd").lr_scale == 1e-5
    assert ctc.params("ccd").lambda_ == 100.0


def test_value_through_integer():
    vals = np.array([3.7, 2.0, 0.999, -2.5, 1e20, 5.0])
    got = po.value_trunc(vals)
    assert got[0] == 3.0 and got[1] == 2.0 and got[2] == 0.0 and got[5] == 5.0
    assert got[3] == float(2**64 - 2)


# ------------------------------------------------------------------ oracle
def test_oracle_grad_finite_differences():
    ind, vals = synth.random_small(400, (12, 10, 8), seed=5)
    T = po.Tensor(ind, vals, [12, 10, 8])
    rng = np.random.default_rng(0)
    U = [rng.uniform(0, 1, (d, 4)) for d in (12, 10, 8)]
    G = po.grad(T, U, 0.1)
    h = 1e-6
    for mode in range(3):
        for r, f in [(0, 0), (3, 2), (7, 3)]:
            Up = [u.copy() for u in U]
            Um = [u.copy() for u in U]
            Up[mode][r, f] += h
            Um[mode][r, f] -= h
            fd = (po.objective(T, Up, 0.1) - po.objective(T, Um, 0.1)) / (2 * h)
            assert abs(fd - G[mode][r, f]) < 1e-5 * max(1, abs(fd))


def test_oracle_als_and_ccdpp_decrease_objective():
    ind, vals = synth.random_small(3000, (40, 30, 20), seed=6)
    T = po.Tensor(ind, vals, [40, 30, 20])
    rng = np.random.default_rng(1)
    U = [rng.uniform(0, 1, (d, 8)) / np.sqrt(8) for d in (40, 30, 20)]
    lam = 0.1

    def obj(U):  # the ALS objective: sum of squares + lambda ||U||^2
        return po.sq_loss(T, U) + po.frob([40, 30, 20], U, lam)

    prev = obj(U)
    for _ in range(3):
        for m in range(3):
            po.als_mode(T.sorted_for_mode(m), m, U, lam)
            cur = obj(U)
            assert cur <= prev * (1 + 1e-12)
            prev = cur
    U2 = [rng.uniform(0, 1, (d, 8)) / np.sqrt(8) for d in (40, 30, 20)]
    r = po.residual(T, U2)
    prev = obj(U2)
    for _ in range(2):
        po.ccdpp_outer(T, U2, lam, 2, r)
        cur = obj(U2)
        assert cur <= prev * (1 + 1e-12)
        prev = cur
    assert np.allclose(r, po.residual(T, U2), atol=1e-9)


def test_oracle_omp_variants_agree():
    ind, vals = synth.random_small(20000, (300, 200, 100), seed=7)
    T = po.Tensor(ind, vals, [300, 200, 100])
    rng = np.random.default_rng(2)
    U = [rng.uniform(0, 1, (d, 16)) / 4 for d in (300, 200, 100)]
    assert abs(po.sq_loss(T, U) - po.sq_loss(T, U, nthreads=4)) < 1e-8 * po.sq_loss(T, U)
    Ua = [u.copy() for u in U]
    Ub = [u.copy() for u in U]
    Ts = T.sorted_for_mode(1)
    po.als_mode(Ts, 1, Ua, 0.1)
    po.als_mode(Ts, 1, Ub, 0.1, nthreads=4)
    assert max(np.max(np.abs(a - b)) for a, b in zip(Ua, Ub)) < 1e-10
    ra, rb = po.residual(T, U), po.residual(T, U)
    Ua = [u.copy() for u in U]
    Ub = [u.copy() for u in U]
    po.ccdpp_outer(T, Ua, 0.1, 1, ra)
    po.ccdpp_outer(T, Ub, 0.1, 1, rb, nthreads=4)
    assert max(np.max(np.abs(a - b)) for a, b in zip(Ua, Ub)) < 1e-9


def test_compat_weights_rules():
    """Reference lane multiplicities on a hand-made 64-nonzero tensor."""
    # rows: tile 0 = 32 nonzeros of row 1 (one segment -> all dropped);
    # tile 1 = rows 2 (10), 3 (22): row 2 is the tile's first segment -> 0,
    # row 3 ends at lane 31 with head 10 -> lanes 10..31 weight 1, lane 31
    # gets K - (31 - 10) extra where K = continuation bits among lanes 1..31
    rows = np.array([1] * 32 + [2] * 10 + [3] * 22, dtype=np.uint64)
    ind = np.stack([rows, np.arange(64, dtype=np.uint64) % 5 + 1, np.arange(64, dtype=np.uint64) % 7 + 1])
    T = po.Tensor(ind, np.ones(64), [3, 5, 7])
    w = po.compat_weights(T, 0, 0)
    assert np.all(w[:32] == 0)
    assert np.all(w[32:42] == 0)
    K = 9 + 21  # continuation lanes: 1..9 (row 2) and 11..31 (row 3)
    assert np.all(w[42:63] == 1)
    assert w[63] == 1 + (K - (31 - 10))


# ------------------------------------------------------------------ factor files
def _ref_mat_write(U, path):
    """The reference's own mat_write (sgpu/io.c:554-591, built from its
    sources into oracle/_ref) on a row-first ordi_matrix."""
    import ctypes as C

    class OrdiMatrix(C.Structure):
        _fields_ = [("I", C.c_uint64), ("J", C.c_uint64), ("values", C.POINTER(C.c_double)),
                    ("row_col_flag", C.c_int)]

    lib = C.CDLL(os.path.join(po.REF_DIR, "libref_host.so"))
    lib.mat_write.argtypes = [C.POINTER(OrdiMatrix), C.c_char_p]
    U = np.ascontiguousarray(U, dtype=np.float64)
    m = OrdiMatrix(U.shape[0], U.shape[1], U.ctypes.data_as(C.POINTER(C.c_double)), 1)
    lib.mat_write(C.byref(m), path.encode())


@pytest.mark.skipif(not po.ref_host_available(), reason="reference host code not built")
def test_factor_text_matches_reference_mat_write(tmp_path):
    rng = np.random.default_rng(4)
    m = ctc.Model([7, 5, 3], 8)
    U = [rng.standard_normal((d, 8)) * 10.0 ** rng.integers(-5, 5, (d, 8)) for d in (7, 5, 3)]
    U[0][0, 0] = 0.0
    U[0][0, 1] = -0.0
    m.set_factors(U)
    for mode in range(3):
        ours, ref = str(tmp_path / f"ours{mode}.txt"), str(tmp_path / f"ref{mode}.txt")
        m.write_text(mode, ours)
        _ref_mat_write(U[mode], ref)
        assert open(ours, "rb").read() == open(ref, "rb").read()


def test_large_factor_text_matches_reference_mat_write(tmp_path):
    """200k rows: the rows are formatted in parallel blocks and written in
    order; the file is the reference's byte for byte."""
    rng = np.random.default_rng(6)
    U = rng.standard_normal((200_000, 16)) * 10.0 ** rng.integers(-8, 8, (200_000, 16))
    m = ctc.Model([200_000, 3, 2], 16)
    m.set_factors([U, np.zeros((3, 16)), np.zeros((2, 16))])
    ours, ref = str(tmp_path / "ours.txt"), str(tmp_path / "ref.txt")
    m.write_text(0, ours)
    _ref_mat_write(U, ref)
    assert open(ours, "rb").read() == open(ref, "rb").read()


def test_model_checkpoint_round_trip_and_rejects_bad_files(tmp_path):
    rng = np.random.default_rng(5)
    for dims in ([11, 7, 5], [6, 5, 4, 3]):
        m = ctc.Model(dims, 16)
        U = [rng.standard_normal((d, 16)) for d in dims]
        U[0][1, 2] = np.nextafter(1.0, 2.0)
        m.set_factors(U)
        p = str(tmp_path / "m.ctcm")
        m.save(p)
        q = ctc.Model.load(p)
        assert q.dims == dims and q.rank == 16
        for a, b in zip(q.factors(), U):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    bad = tmp_path / "bad.ctcm"
    bad.write_bytes(b"NOPE" + b"\0" * 64)
    with pytest.raises(ctc.CtcError):
        ctc.Model.load(str(bad))
    raw = open(p, "rb").read()
    (tmp_path / "short.ctcm").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(ctc.CtcError):
        ctc.Model.load(str(tmp_path / "short.ctcm"))


# ------------------------------------------------------------------ tile plans
def _zipf_rows(n, nrows, seed):
    rng = np.random.default_rng(seed)
    w = 1.0 / np.arange(1, nrows + 1) ** 1.1
    return np.sort(rng.choice(nrows, size=n, p=w / w.sum()) + 1).astype(np.uint64)


@pytest.mark.parametrize("n,nrows,T", [(1, 5, 256), (5000, 40, 128), (70000, 3000, 256),
                                       ((1 << 20) + 17, 20000, 512), (3 << 20, 500000, 256)])
def test_plan_from_runs_is_the_plan_from_indices(n, nrows, T):
    """The device staging plans from the rows' run lengths; the host staging
    from the index array.  Same tiles, same long rows, chunk cuts included
    (n above 2^20 takes the 64-chunk form)."""
    ind = _zipf_rows(n, nrows, seed=n + T)
    ta, ha = ctc.plan_tiles(ind, T, from_runs=False)
    tb, hb = ctc.plan_tiles(ind, T, from_runs=True)
    assert np.array_equal(ta, tb) and np.array_equal(ha, hb)
    # the tiles cover [0, n) in order; light tiles hold whole rows
    assert ta[0, 0] == 0 and int(ta[-1, 0]) + int(ta[-1, 1]) == n
    assert np.all(ta[1:, 0] == ta[:-1, 0] + ta[:-1, 1]) and np.all((ta[:, 1] >= 1) & (ta[:, 1] <= T))
    light = ta[ta[:, 2] < 0]
    starts, ends = light[:, 0], light[:, 0] + light[:, 1]
    assert np.all((starts == 0) | (ind[np.maximum(starts - 1, 0)] != ind[starts]))
    assert np.all((ends == n) | (ind[np.minimum(ends, n - 1)] != ind[ends - 1]))
    # long rows: pieces of T, numbered in order, one entry per row longer than T
    runs = np.diff(np.flatnonzero(np.r_[True, ind[1:] != ind[:-1], True]))
    assert len(ha) == int(np.sum(runs > T))
    for h, (row, first, np_, _) in enumerate(ha):
        pieces = ta[first:first + np_]
        assert np.all(pieces[:, 2] == h) and np.array_equal(pieces[:, 3], np.arange(np_))
        assert np.all(ind[pieces[:, 0]] == row + 1)
    # the tiles with a long-row index are exactly the long rows' ranges, in
    # order (the staging lists the pieces from the long-row table)
    ranges = [np.arange(f, f + k) for (_, f, k, _) in ha]
    listed = np.concatenate(ranges) if ranges else np.zeros(0, dtype=np.int64)
    assert np.array_equal(np.flatnonzero(ta[:, 2] >= 0), listed)


def test_plan_rejects_unsorted_indices():
    ind = np.array([1, 1, 3, 2, 4], dtype=np.uint64)
    for runs in (False, True):
        with pytest.raises(ctc.CtcError):
            ctc.plan_tiles(ind, 32, from_runs=runs)


def test_sort_through_the_host_worker_pool_is_numpys_stable_sort():
    """ctc_tensor_sort on 300k nonzeros (large enough that its copies run on
    the persistent host workers), three modes in a row: numpy's stable
    (mode, next mode) order, values included."""
    rng = np.random.default_rng(7)
    n, dims = 300_000, (5000, 4000, 300)
    ind = np.stack([rng.integers(1, d + 1, n) for d in dims]).astype(np.uint64)
    vals = rng.random(n)
    for m in range(3):
        t = ctc.Tensor.from_coo(ind, vals, dims=dims)
        api._check(api.lib().ctc_tensor_sort(t.h, m))
        gi, gv = t.export()
        o = np.lexsort((ind[(m + 1) % 3], ind[m]))
        assert np.array_equal(gi, ind[:, o]) and np.array_equal(gv, vals[o]), m


@pytest.mark.parametrize("case", ["tile_1", "rows_of_exactly_T", "one_row", "n_at_chunk_threshold"])
def test_plan_edge_cases_agree(case):
    """Edge cases of the two planners: tile length 1 (every row of more than
    one nonzero becomes pieces), rows exactly one tile long, a single row
    (all pieces), and n = 2^20 (the smallest chunked plan)."""
    rng = np.random.default_rng(11)
    if case == "tile_1":
        ind, T = np.sort(rng.integers(1, 50, 3000)).astype(np.uint64), 1
    elif case == "rows_of_exactly_T":
        T = 64
        ind = np.repeat(np.arange(1, 201, dtype=np.uint64), T)
    elif case == "one_row":
        ind, T = np.full(10000, 7, dtype=np.uint64), 256
    else:
        ind, T = _zipf_rows(1 << 20, 30000, seed=5), 256
    ta, ha = ctc.plan_tiles(ind, T, from_runs=False)
    tb, hb = ctc.plan_tiles(ind, T, from_runs=True)
    assert np.array_equal(ta, tb) and np.array_equal(ha, hb)
    assert int(ta[:, 1].sum()) == ind.size and np.all(ta[:, 1] <= T)
    if case == "rows_of_exactly_T":
        assert len(ha) == 0 and np.all(ta[:, 1] == T)  # a row of exactly T is one light tile
    if case == "one_row":
        assert len(ha) == 1 and ha[0][0] == 6 and ha[0][2] == len(ta)


def _sorted_random(n, dims, seed, mode):
    rng = np.random.default_rng(seed)
    ind = np.stack([rng.integers(1, d + 1, n) for d in dims]).astype(np.uint64)
    vals = rng.uniform(-2, 6, n)
    o = np.lexsort((ind[(mode + 1) % 3], ind[mode]))
    return ind[:, o].copy(), vals[o].copy()


@pytest.mark.skipif(not po.ref_host_available(), reason="reference host library not built")
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_parallel_ciss_equals_the_reference_builder_on_a_large_tensor(mode):
    """1.5M nonzeros: the host builder runs in chunks of tiles in parallel;
    every written slot equals the reference's own ciss_alloc bit for bit."""
    dims = (40000, 3000, 200)
    ind, vals = _sorted_random(1_500_000, dims, 21 + mode, mode)
    got = ctc.ciss_alloc(ctc.Tensor.from_coo(ind, vals, dims=dims), mode + 1, 32)
    ref = po.ref_ciss_alloc(po.Tensor(ind, vals, list(dims)), mode + 1)
    w = got["written"]
    assert got["size_rows"] == ref["size_rows"]
    assert np.array_equal(got["directory"], ref["directory"]) and np.array_equal(got["dcounter"], ref["dcounter"])
    assert np.array_equal(got["entries"].view(np.uint64)[w], ref["entries"].view(np.uint64)[w])


_SERIAL_CISS = """
import sys, numpy as np
sys.path.insert(0, {root!r})
import cutc_b200 as ctc
z = np.load({src!r})
c = ctc.ciss_alloc(ctc.Tensor.from_coo(z["ind"], z["vals"], dims=[int(x) for x in z["dims"]]),
                   {mode}, {T}, ga={ga})
np.savez({dst!r}, **{{k: v for k, v in c.items() if isinstance(v, np.ndarray)}})
"""


@pytest.mark.parametrize("T,ga", [(1, True), (16, True), (63, True), (32, False)])
def test_parallel_ciss_equals_the_serial_loop(tmp_path, T, ga):
    """The chunked builder against the same build on one host thread (the
    reference loop as written), everything compared: written slots,
    unwritten zeros and the written mask, GA counters and odd tile lengths."""
    import subprocess
    import sys
    dims = (30000, 2000, 100)
    ind, vals = _sorted_random(1_200_000, dims, 33, 0)
    src, dst = str(tmp_path / "t.npz"), str(tmp_path / "serial.npz")
    np.savez(src, ind=ind, vals=vals, dims=np.array(dims))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = _SERIAL_CISS.format(root=root, src=src, dst=dst, mode=1, T=T, ga=ga)
    env = dict(os.environ, CTC_HOST_THREADS="1")
    subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
    serial = np.load(dst)
    got = ctc.ciss_alloc(ctc.Tensor.from_coo(ind, vals, dims=dims), 1, T, ga=ga)
    for k in ("directory", "dcounter", "written"):
        assert np.array_equal(got[k], serial[k]), k
    assert np.array_equal(got["entries"].view(np.uint64), serial["entries"].view(np.uint64))


@pytest.mark.parametrize("case", ["duplicates", "zero_and_large", "wide_keys"])
def test_radix_sort_cases_are_numpys_stable_sort(case):
    """Many equal pairs (stability), 0 indices with indices near 2^32, and
    pairs too wide for one 64-bit key (the comparison sort)."""
    rng = np.random.default_rng(12)
    n = 200_000
    if case == "duplicates":
        ind = np.stack([rng.integers(1, 9, n), rng.integers(1, 5, n), rng.integers(1, 1000, n)]).astype(np.uint64)
    elif case == "zero_and_large":
        ind = np.stack([rng.integers(0, 3, n), rng.integers(2**32 - 50, 2**32 + 50, n),
                        rng.integers(0, 7, n)]).astype(np.uint64)
    else:
        ind = np.stack([rng.integers(2**40, 2**40 + 9, n), rng.integers(2**39, 2**39 + 7, n),
                        rng.integers(1, 5, n)]).astype(np.uint64)
    vals = rng.random(n)
    for m in range(3):
        t = ctc.Tensor.from_coo(ind, vals)
        api._check(api.lib().ctc_tensor_sort(t.h, m))
        gi, gv = t.export()
        o = np.lexsort((ind[(m + 1) % 3], ind[m]))
        assert np.array_equal(gi, ind[:, o]) and np.array_equal(gv, vals[o]), (case, m)
