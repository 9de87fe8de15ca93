"""The allocation-free read search (sbwt_search_reads_noalloc).

It exists for callers that may not allocate device memory -- code running
while another framework owns the device allocator, serving loops where a
cudaMalloc would stall or synchronize the device, hosts with a fixed memory
budget -- and keeps its scratch in one fixed device array inside the library.
This file is collected last on purpose, so a run that stops at the first
failure has already run every other test.  It checks, through the C ABI, that
two calls in a row give exactly the results of sbwt_search_reads (integer
output: the tolerance is zero), and that a batch over the stated limit is
refused with a clear error before any device work.
"""
import ctypes as C

import numpy as np
import pytest

import sbwt_b200 as S
from helpers import mixed_reads, synthetic

pytestmark = pytest.mark.gpu

MAX_CHARS = 8 << 20
MAX_READS = 1 << 18


def _noalloc():
    f = S.lib().sbwt_search_reads_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p,
                  C.c_uint64, C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_matches_search_reads_twice():
    import torch
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 41, 20000, median=100, sigma=0.7, len_min=0, len_max=600,
                              sub=0.01, n_rate=0.01)
    assert len(chars) <= MAX_CHARS and len(ends) <= MAX_READS
    d_chars = torch.from_numpy(chars.copy()).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
    n_k = idx.count_kmers(ends)
    ref = torch.empty(n_k, dtype=torch.int64, device="cuda")
    assert idx.search_reads(d_chars, d_ends, out=ref) == n_k
    expected = ref.cpu().numpy().view(np.uint64)
    f = _noalloc()
    for call in range(2):
        out = torch.full((n_k,), -7, dtype=torch.int64, device="cuda")
        n = C.c_uint64(0)
        rc = f(idx._h, d_chars.data_ptr(), len(chars), d_ends.data_ptr(), len(ends),
               out.data_ptr(), n_k, C.byref(n), 0, None)
        S.check(rc)
        assert n.value == n_k
        got = out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, expected), f"call {call} differs"


def test_noalloc_rejects_oversized_batches():
    import torch
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    f = _noalloc()
    n = C.c_uint64(0)
    # real (small) buffers; the sizes are refused on the host before any launch
    buf = torch.zeros(64, dtype=torch.int64, device="cuda")
    p = buf.data_ptr()
    rc = f(idx._h, p, MAX_CHARS + 1, p, 1, p, 64, C.byref(n), 0, None)
    assert rc == S.E_INVALID
    assert b"at most" in S.lib().sbwt_last_error()
    rc = f(idx._h, p, 100, p, MAX_READS + 1, p, 64, C.byref(n), 0, None)
    assert rc == S.E_INVALID
