"""Result formatting on the GPU (sbwt_format_index_results /
sbwt_format_color_results) against the host writers, which reproduce the
reference's files byte for byte: every format, adversarial values, empty
reads, the golden fixtures' expected ascii files, and device buffers."""
import ctypes as C
import struct

import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
from helpers import FIXTURE_FILES, GOLDEN, TMP, golden_sbwt_path, host_fastx, oracle_index

pytestmark = pytest.mark.gpu
EXT_INDEX = {0: ".txt", 1: ".bin", 2: ".bool"}
EXT_COLOR = {0: ".txt", 1: ".bin", 2: ".csv"}


def host_index_bytes(res, ends, k, fmt, name):
    L = S.lib()
    L.sbwt_write_index_results.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_uint64, C.c_uint32]
    out = TMP / name
    S.check(L.sbwt_write_index_results(str(out).encode(), fmt, 0,
                                       res.ctypes.data if len(res) else None,
                                       ends.ctypes.data if len(ends) else None, len(ends), k))
    return (TMP / (name + EXT_INDEX[fmt])).read_bytes()


def host_color_bytes(ids, offs, C_, fmt, name):
    L = S.lib()
    L.sbwt_write_color_results.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_uint64, C.c_uint64]
    out = TMP / name
    S.check(L.sbwt_write_color_results(str(out).encode(), fmt, 0,
                                       ids.ctypes.data if len(ids) else None, offs.ctypes.data,
                                       len(offs) - 1, C_))
    b = (TMP / (name + EXT_COLOR[fmt])).read_bytes()
    return b[b.index(b"\n") + 1:] if fmt == 2 else b  # csv: drop the title row


def random_index_batch(seed, n_reads, k=31):
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 3 * k, n_reads)
    lens[rng.random(n_reads) < 0.1] = int(rng.integers(0, k))  # reads shorter than k
    ends = np.cumsum(lens).astype(np.uint64)
    nk = int(np.maximum(lens - k + 1, 0).sum())
    res = rng.integers(0, 1 << 40, nk, dtype=np.uint64)
    small = rng.random(nk) < 0.5
    res[small] = rng.integers(0, 1000, int(small.sum()), dtype=np.uint64)
    res[rng.random(nk) < 0.2] = O.NOT_FOUND
    res[rng.random(nk) < 0.1] = O.INVALID
    res[rng.random(nk) < 0.02] = np.uint64(O.INVALID - 1)  # 20-digit value
    return res, ends


@pytest.mark.parametrize("fmt", [0, 1, 2])
@pytest.mark.parametrize("seed", [1, 2])
def test_index_formats_match_host_writer(fmt, seed):
    res, ends = random_index_batch(seed, 3000 + seed)
    got = S.format_index_results(res, ends, 31, fmt)
    assert got == host_index_bytes(res, ends, 31, fmt, f"fi_{seed}_{fmt}")


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_index_ascii_reproduces_reference_fixture(name, tmp_path):
    idx = oracle_index(golden_sbwt_path(), 10)
    text = (GOLDEN / "index_search" / name).read_bytes()
    chars, ends = host_fastx(text, tmp_path / "q.fx")
    reads = O.parse_fastx(text)
    res = np.concatenate(O.index_search_reads(idx, reads) + [np.zeros(0, np.uint64)])
    body = S.format_index_results(res.astype(np.uint64), ends, 30, 0)
    head = b"".join(struct.pack("<Q", len(s)) + s for s in (b"ascii", b"v1.0"))
    exp = (GOLDEN / "index_search" / "expected" / (name.split(".")[0] + ".txt")).read_bytes()
    assert head + body == exp


@pytest.mark.parametrize("fmt", [0, 1, 2])
def test_color_formats_match_host_writer(fmt):
    rng = np.random.default_rng(fmt)
    n_reads, n_colors = 2500, 3000
    counts = rng.integers(0, 40, n_reads)
    counts[rng.random(n_reads) < 0.3] = 0
    offs = np.zeros(n_reads + 1, np.uint64)
    offs[1:] = np.cumsum(counts)
    ids = np.concatenate([np.sort(rng.choice(n_colors, int(c), replace=False))
                          for c in counts]).astype(np.uint32)
    got = S.format_color_results(ids, offs, n_colors, fmt)
    assert got == host_color_bytes(ids, offs, n_colors, fmt, f"fc_{fmt}")


def test_device_buffers_and_capacity():
    import torch
    res, ends = random_index_batch(9, 500)
    exp = S.format_index_results(res, ends, 31, 0)
    d_res = torch.from_numpy(res.view(np.int64)).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64)).cuda()
    d_out = torch.zeros(len(exp), dtype=torch.uint8, device="cuda")
    nb = C.c_uint64()
    L = S.lib()
    st = torch.cuda.current_stream().cuda_stream
    rc = L.sbwt_format_index_results(d_res.data_ptr(), d_ends.data_ptr(), len(ends), 31, 0,
                                     d_out.data_ptr(), len(exp) - 1, C.byref(nb),
                                     S.DEVICE_POINTERS, 0, st)
    assert rc == S.E_CAPACITY and nb.value == len(exp)
    S.check(L.sbwt_format_index_results(d_res.data_ptr(), d_ends.data_ptr(), len(ends), 31, 0,
                                        d_out.data_ptr(), len(exp), C.byref(nb),
                                        S.DEVICE_POINTERS, 0, st))
    assert d_out.cpu().numpy().tobytes() == exp
    assert S.format_index_results(np.zeros(0, np.uint64), np.zeros(0, np.uint64), 31, 0) == b""
