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


def _reads(n_reads, length, seed):
    rng = np.random.default_rng(seed)
    chars = rng.choice(np.frombuffer(b"ACGT", np.uint8), n_reads * length)
    ends = np.arange(1, n_reads + 1, dtype=np.uint64) * length
    return chars, ends


@pytest.mark.parametrize("shape", [(MAX_READS, MAX_CHARS // MAX_READS),
                                   (MAX_CHARS // 400, 400)])
@pytest.mark.parametrize("kernel", [0, 1, 2, 6])
def test_noalloc_at_its_limits_allocates_nothing(shape, kernel):
    """A batch at the stated limits (every read slot used, or nearly every
    char with the smallest tile, 16 k-mers, so that the tile table is full)
    gives sbwt_search_reads's results on every read search kernel, and the
    call leaves the device's free memory unchanged."""
    import torch
    n_reads, length = shape
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = _reads(n_reads, length, 3 + length)
    # half of the reads from the genomes, so that k-mers are found
    gen = g.chars[: (n_reads // 2) * length]
    chars[: len(gen)] = gen
    assert len(chars) <= MAX_CHARS and len(ends) <= MAX_READS
    d_chars = torch.from_numpy(chars.copy()).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
    n_k = idx.count_kmers(ends)
    S.set_table_kernel(kernel)
    S.set_launch_config(tile=16)
    try:
        ref = torch.empty(n_k, dtype=torch.int64, device="cuda")
        assert idx.search_reads(d_chars, d_ends, out=ref) == n_k
        expected = ref.cpu().numpy().view(np.uint64)
        assert (expected < (1 << 62)).any()
        f = _noalloc()
        out = torch.full((n_k,), -7, dtype=torch.int64, device="cuda")
        n = C.c_uint64(0)
        S.check(f(idx._h, d_chars.data_ptr(), len(chars), d_ends.data_ptr(), len(ends),
                  out.data_ptr(), n_k, C.byref(n), 0, None))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        out.fill_(-7)
        S.check(f(idx._h, d_chars.data_ptr(), len(chars), d_ends.data_ptr(), len(ends),
                  out.data_ptr(), n_k, C.byref(n), 0, None))
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        assert n.value == n_k
        assert np.array_equal(out.cpu().numpy().view(np.uint64), expected)
    finally:
        S.set_table_kernel(S.TABLE_KERNEL_DEFAULT)
        S.set_launch_config()
