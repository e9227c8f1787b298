"""Argument checks of ctc_sse_noalloc, the squared-error sum for callers
that cannot allocate device memory.  Every check runs on the host before
any CUDA call, so these run without a GPU: the pointers passed here are
never dereferenced."""
import ctypes as C

from cutc_b200 import api


def _call(rec, n, u0, u1, u2, rank, out):
    return api.lib().ctc_sse_noalloc(C.c_void_p(rec), n, C.c_void_p(u0), C.c_void_p(u1), C.c_void_p(u2),
                                     rank, C.c_void_p(out), None)


def test_noalloc_rejects_oversize_and_bad_rank():
    big = (1 << 30) + 1
    rc = _call(16, big, 16, 16, 16, 16, 16)
    assert rc == -1 and b"2^30" in api.lib().ctc_last_error()
    rc = _call(16, 10, 16, 16, 16, 12, 16)
    assert rc == -5


def test_noalloc_rejects_null_and_empty():
    assert _call(0, 10, 16, 16, 16, 16, 16) == -1
    assert _call(16, 0, 16, 16, 16, 16, 16) == -1


def test_noalloc_rejects_misaligned_pointers():
    """rec and the factors are read with 16-byte vector loads: a pointer
    that is 8-byte but not 16-byte aligned is an argument error, not a
    device fault."""
    for args in ((24, 16, 16, 16), (16, 40, 16, 16), (16, 16, 8, 16), (16, 16, 16, 4)):
        rc = _call(args[0], 10, args[1], args[2], args[3], 16, 16)
        assert rc == -1 and b"16-byte aligned" in api.lib().ctc_last_error(), args
    rc = _call(16, 10, 16, 16, 16, 16, 12)
    assert rc == -1 and b"8-byte aligned" in api.lib().ctc_last_error()
