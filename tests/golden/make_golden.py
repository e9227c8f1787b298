"""Generates the golden fixtures in tests/golden/ from the reference's own
host code, built from its sources by oracle/build_ref.sh:

  oracle/_ref/libref_host.so     sgpu tt_read (sptensor.c:64) and
                                 ciss_alloc (ciss.c:68), tile length 32
  oracle/_ref/libref_ga_host.so  ga cissbasic_alloc (ga/ciss.c:69), any
                                 tile length

For every case a seeded tensor is written as .tns text, read back with the
reference tt_read, sorted for each mode and tiled with the reference CISS
builder.  The reference leaves some CISS slots uninitialised; which slots it
writes is determined from the reference alone by running each build twice
in child processes whose glibc malloc fills fresh memory with different
bytes (perturb tunable / mallopt M_PERTURB, thread cache off): the slots that agree are the written ones.

    python tests/golden/make_golden.py      (needs the reference tree)
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")

_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)


class RefSptensor(C.Structure):
    _fields_ = [("nmodes", C.c_uint64), ("nnz", C.c_uint64), ("dims", _u64p),
                ("ind", C.POINTER(_u64p)), ("vals", _f64p)]


class RefCiss(C.Structure):
    _fields_ = [("nmodes", C.c_uint64), ("nnz", C.c_uint64), ("size", C.c_uint64),
                ("dlength", C.c_uint64), ("dims", _u64p), ("directory", _u64p),
                ("dcounter", _u64p), ("entries", _f64p)]


def child(args):
    """Runs in a fresh process: one reference CISS build, raw outputs to npz."""
    src, mode0, tile, perturb, out = args[0], int(args[1]), int(args[2]), int(args[3]), args[4]
    libc = C.CDLL("libc.so.6")
    libc.mallopt(-6, perturb)  # M_PERTURB
    z = np.load(src)
    ind, vals, dims = z["ind"], z["vals"], z["dims"]
    nm, nnz = ind.shape
    # one padding element: the GA builder reads ind[mode][nnz] before its bound test
    cols = [np.concatenate([ind[m], [0]]).astype(np.uint64) for m in range(nm)]
    v = np.ascontiguousarray(vals, dtype=np.float64)
    st = RefSptensor()
    st.nmodes, st.nnz = nm, nnz
    d = (C.c_uint64 * nm)(*[int(x) for x in dims])
    st.dims = d
    ptrs = (_u64p * nm)(*[c.ctypes.data_as(_u64p) for c in cols])
    st.ind = ptrs
    st.vals = v.ctypes.data_as(_f64p)
    if tile == 32:
        L = C.CDLL(os.path.join(REF, "libref_host.so"))
        L.ciss_alloc.restype = C.POINTER(RefCiss)
        L.ciss_alloc.argtypes = [C.POINTER(RefSptensor), C.c_uint64]
        c = L.ciss_alloc(C.byref(st), mode0 + 1).contents
    else:
        L = C.CDLL(os.path.join(REF, "libref_ga_host.so"))
        L.cissbasic_alloc.restype = C.POINTER(RefCiss)
        L.cissbasic_alloc.argtypes = [C.POINTER(RefSptensor), C.c_uint64, C.c_uint64, C.c_uint64, C.c_int]
        ib = int(ind[mode0][0])
        ie = int(ind[mode0][nnz - 1]) + 1
        c = L.cissbasic_alloc(C.byref(st), mode0, ib, ie, tile).contents
    np.savez(out, directory=np.ctypeslib.as_array(c.directory, (c.dlength,)).copy(),
             dcounter=np.ctypeslib.as_array(c.dcounter, (c.dlength + 1,)).copy(),
             entries=np.ctypeslib.as_array(c.entries, (c.size * 3,)).copy(),
             size=c.size, dlength=c.dlength)


def ref_ciss(tmp, ind, vals, dims, mode0, tile):
    src = os.path.join(tmp, "in.npz")
    np.savez(src, ind=ind, vals=vals, dims=np.asarray(dims, dtype=np.uint64))
    outs = []
    for k, pb in enumerate((0x5A, 0xC3)):
        out = os.path.join(tmp, f"out{k}.npz")
        # tcache off so that every fresh chunk goes through the perturbing paths
        env = dict(os.environ, GLIBC_TUNABLES=f"glibc.malloc.tcache_count=0:glibc.malloc.perturb={pb}")
        subprocess.run([sys.executable, __file__, "--child", src, str(mode0), str(tile), str(pb), out],
                       check=True, env=env)
        outs.append(np.load(out))
    a, b = outs
    for key in ("directory", "dcounter"):
        assert np.array_equal(a[key], b[key])
    ea, eb = a["entries"].view(np.uint64), b["entries"].view(np.uint64)
    written = ea == eb
    entries = np.where(written, a["entries"], 0.0)
    return dict(directory=a["directory"], dcounter=a["dcounter"], entries=entries, written=written)


def ref_tt_read(path):
    L = C.CDLL(os.path.join(REF, "libref_host.so"))
    L.tt_read.restype = C.POINTER(RefSptensor)
    L.tt_read.argtypes = [C.c_char_p]
    t = L.tt_read(path.encode()).contents
    nm, nnz = t.nmodes, t.nnz
    ind = np.stack([np.ctypeslib.as_array(t.ind[m], (nnz,)).copy() for m in range(nm)])
    vals = np.ctypeslib.as_array(t.vals, (nnz,)).copy()
    return ind, vals, np.array([t.dims[m] for m in range(nm)], dtype=np.uint64)


def write_tns(path, ind, vals, header=True, blank=True, tabs=False):
    sep = "\t" if tabs else " "
    with open(path, "w") as f:
        if header:
            f.write("# generated test tensor\n")
        for n in range(ind.shape[1]):
            if blank and n == 3:
                f.write("\n")
            f.write(sep.join(str(int(ind[m, n])) for m in range(ind.shape[0])) + sep + "%.17g\n" % vals[n])


def sort_mode(ind, vals, m):
    o = np.lexsort((ind[(m + 1) % 3], ind[m]))
    return ind[:, o], vals[o]


CASES = [
    # name, nnz, dims, seed, extra
    ("survey_example", 5, (4, 3, 3), 0, {"rows": [1, 1, 3, 3, 4]}),
    ("single", 1, (3, 3, 3), 1, {}),
    ("n31", 31, (6, 5, 4), 2, {}),
    ("n32", 32, (6, 5, 4), 3, {}),
    ("n33", 33, (6, 5, 4), 4, {}),
    ("n64", 64, (9, 7, 5), 5, {}),
    ("n100", 100, (12, 9, 7), 6, {}),
    ("n257", 257, (20, 15, 9), 7, {}),
    ("n1000", 1000, (40, 30, 20), 8, {}),
    ("distinct_rows", 40, (60, 5, 5), 9, {"distinct_mode0": True}),
    ("one_row", 70, (1, 9, 8), 10, {}),
    ("zero_based", 50, (6, 5, 4), 11, {"zero_based": True}),
]
TILE_CASES = [1, 2, 16, 31, 63]


def make_case(name, nnz, dims, seed, extra, tmp):
    rng = np.random.default_rng(seed)
    base = 0 if extra.get("zero_based") else 1
    ind = np.stack([rng.integers(0, d, nnz) for d in dims]).astype(np.uint64) + base
    if extra.get("distinct_mode0"):
        ind[0] = rng.permutation(dims[0])[:nnz].astype(np.uint64) + 1
    if "rows" in extra:
        ind[0] = np.asarray(extra["rows"], dtype=np.uint64)
    vals = rng.uniform(-3.0, 7.0, nnz)
    special = [0.5, 2.9999999999, -0.0, 1e20, -2.5, 4.0]
    for q, v in enumerate(special[: nnz // 4]):
        vals[q * 3 % nnz] = v
    path = os.path.join(tmp, name + ".tns")
    write_tns(path, ind, vals, tabs=(seed % 2 == 1))
    rind, rvals, rdims = ref_tt_read(path)
    out = {"tns": open(path).read(), "ind": rind, "vals": rvals, "dims": rdims}
    if not extra.get("zero_based"):
        for m in range(3):
            si, sv = sort_mode(rind, rvals, m)
            c = ref_ciss(tmp, si, sv, rdims, m, 32)
            for k, v in c.items():
                out[f"m{m}_{k}"] = v
        if name == "n100":
            si, sv = sort_mode(rind, rvals, 0)
            for T in TILE_CASES:
                c = ref_ciss(tmp, si, sv, rdims, 0, T)
                for k, v in c.items():
                    out[f"t{T}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **{k: (np.asarray(v) if k != "tns" else np.array(v)) for k, v in out.items()})
    return {"name": name, "nnz": int(rind.shape[1]), "dims": [int(x) for x in rdims]}


def main():
    if not os.path.exists(os.path.join(REF, "libref_host.so")):
        raise SystemExit("oracle/_ref/libref_host.so missing: run oracle/build_ref.sh first")
    index = []
    with tempfile.TemporaryDirectory() as tmp:
        for case in CASES:
            index.append(make_case(*case, tmp))
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump({"cases": index, "tile_cases": TILE_CASES,
                   "source": "reference tt_read + ciss_alloc / cissbasic_alloc"}, f, indent=1)
    print(f"wrote {len(index)} golden cases")


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--child":
        child(sys.argv[2:])
    else:
        main()
