"""Index step on the GPU through the C ABI, bit-exact against the oracle,
the reference's own kernels compiled for the host, and the reference's
golden fixtures."""
import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
import sbwt_tools as T
from helpers import FIXTURE_FILES, GOLDEN, golden_sbwt_path, synthetic, oracle_index, \
    mixed_reads, oracle_results

pytestmark = pytest.mark.gpu

# the library's default choice of read search kernel for indexes with a k-mer table
DEFAULT_TABLE_KERNEL = S.TABLE_KERNEL_DEFAULT
# read search kernels of an index with a k-mer table: general, table, the
# walks kernel as (walks per lane, blocks per SM) = (1, 5), (2, 4), (2, 3),
# (4, 2), the k-mers kernel, automatic, the lean walks kernel with 1 and 2
# walks per lane
KERNEL_MODES = list(range(20))


@pytest.fixture(scope="module")
def golden_index():
    return S.SbwtIndex.open(golden_sbwt_path())


@pytest.mark.parametrize("name", FIXTURE_FILES)
@pytest.mark.parametrize("per_kmer", [False, True])
@pytest.mark.parametrize("table", [True, False])
def test_reads_reproduce_reference_fixture(golden_index, name, per_kmer, table):
    assert (golden_index.set_kmer_table(table) > 0) == table
    reads = O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    chars = b"".join(reads)
    ends = np.cumsum([len(r) for r in reads]).astype(np.uint64)
    res = golden_index.search_reads(chars, ends, per_kmer_walk=per_kmer)
    rows, t = [], 0
    for r in reads:
        m = max(0, len(r) - golden_index.k + 1)
        rows.append(O.as_signed_tokens(res[t:t + m]))
        t += m
    exp = O.read_ascii_index_results(GOLDEN / "index_search" / "expected" /
                                     (name.split(".")[0] + ".txt"))
    assert rows == exp


@pytest.mark.parametrize("p", [0, 1, 7, 12, 14])
def test_positions_seam_matches_oracle_and_reference(p):
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    idx = S.SbwtIndex.open(path, presearch_letters=p)
    chars, ends = mixed_reads(g, 5, 500)
    bits, _ = O.seq_to_bits(chars.tobytes())
    pos = O.positions_of(ends, 31)
    got = idx.search(bits, pos)
    exp = oracle_index(path, 8).search_positions(bits, pos)
    assert np.array_equal(got, exp)
    if O.ref_lib() is not None:
        ref = O.OracleIndex(sb.acgt, sb.num_bits, sb.k, use_ref=True)
        assert np.array_equal(got, ref.search_positions(bits, pos))


@pytest.mark.parametrize("per_kmer", [False, True])
@pytest.mark.parametrize("seed", [11, 12])
@pytest.mark.parametrize("table", [True, False])
def test_reads_match_oracle(per_kmer, seed, table):
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    assert (idx.set_kmer_table(table) > 0) == table
    chars, ends = mixed_reads(g, seed, 2000, median=90, sigma=0.8, len_min=0,
                              len_max=500, sub=0.01, n_rate=0.01)
    got = idx.search_reads(chars, ends, per_kmer_walk=per_kmer)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    assert got.dtype == np.uint64 and np.array_equal(got, exp)
    assert (got < O.INVALID).any() and (got == O.NOT_FOUND).any() and (got == O.INVALID).any()


def test_reads_small_k_and_no_suffix_groups():
    g, path, sb = synthetic(8, 1, 3000, 15)
    chars, ends = mixed_reads(g, 3, 500, median=40, sigma=0.5, len_min=0, len_max=120)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    # from arrays without the suffix-group vector: per-k-mer walks only
    idx = S.SbwtIndex.from_arrays(sb.acgt, sb.num_bits, sb.k)
    assert np.array_equal(idx.search_reads(chars, ends), exp)
    idx2 = S.SbwtIndex.from_arrays(sb.acgt, sb.num_bits, sb.k, sb.suffix_group_starts,
                                   presearch_letters=6)
    assert np.array_equal(idx2.search_reads(chars, ends), exp)


@pytest.mark.parametrize("table", [True, False])
def test_edge_cases_empty_short_invalid(table):
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    idx = S.SbwtIndex.open(path)
    idx.set_kmer_table(table)
    gen = g.seq(0)
    reads = [b"", b"ACGT", gen[:31], gen[100:130], b"N" * 40, gen[:31].lower(),
             gen[500:700] + b"X" + gen[700:900], b"", gen[1000:1031]]
    chars = b"".join(reads)
    ends = np.cumsum([len(r) for r in reads]).astype(np.uint64)
    got = idx.search_reads(chars, ends)
    exp = oracle_results(oracle_index(path, 8), np.frombuffer(chars, np.uint8), ends)
    assert np.array_equal(got, exp)
    # no reads at all
    assert len(idx.search_reads(b"", np.zeros(0, np.uint64))) == 0


def test_device_pointer_path_matches_host_path():
    import torch
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 21, 3000)
    host = idx.search_reads(chars, ends)
    d_chars = torch.from_numpy(chars.copy()).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
    d_out = torch.empty(len(host) + 5, dtype=torch.int64, device="cuda")
    n = idx.search_reads(d_chars, d_ends, out=d_out)
    torch.cuda.synchronize()
    assert n == len(host)
    assert np.array_equal(d_out[:n].cpu().numpy().view(np.uint64), host)


def test_chunked_host_pipeline_matches_single_chunk():
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 31, 4000)
    one = idx.search_reads(chars, ends)
    S.set_launch_config(chunk_chars=5000)
    try:
        many = idx.search_reads(chars, ends)
    finally:
        S.set_launch_config()
    assert np.array_equal(one, many)


@pytest.mark.parametrize("pinned_out", [True, False])
@pytest.mark.parametrize("kernel", [1, 2, 6])
def test_pinned_host_chunks_match_device_path(kernel, pinned_out):
    """Host-pointer calls from pinned inputs, many chunks in flight.  Into a
    pageable output on the walks and k-mers kernels the results cross as
    32-bit codes and are widened on host threads (output start not 16-byte
    aligned); into a pinned output, and on the table kernel, as u64.  All
    equal the oracle, and no slot outside the output is written."""
    import torch
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 33, 30000, sub=0.01, n_rate=0.005)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    S.set_table_kernel(kernel)
    S.set_launch_config(chunk_chars=300_001)
    try:
        assert idx.host_result_bytes() == (4 if kernel != 1 else 8)
        h_chars = torch.from_numpy(chars.copy()).pin_memory()
        h_ends = torch.from_numpy(ends.view(np.int64).copy()).pin_memory()
        h_out = torch.full((len(exp) + 3,), -7, dtype=torch.int64)
        if pinned_out:
            h_out = h_out.pin_memory()
        out = h_out.numpy()[1:1 + len(exp)].view(np.uint64)
        idx.search_reads(h_chars.numpy(), h_ends.numpy().view(np.uint64), out=out)
        assert np.array_equal(out, exp)
        assert h_out[0].item() == -7 and (h_out[1 + len(exp):] == -7).all()
    finally:
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
        S.set_launch_config()


@pytest.mark.parametrize("kernel", [0, 1, 2, 6])
def test_device_batch_in_pieces_matches_one_launch(kernel):
    """A device-pointer batch split into pieces of whole reads (as batches of
    2^32 or more chars are, for the 32-bit kernels; here forced small): the
    same results as one launch, including the capacity error."""
    import torch
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 35, 6000, sub=0.01, n_rate=0.005, len_min=0, len_max=800)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    d_chars = torch.from_numpy(chars.copy()).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
    S.set_table_kernel(kernel)
    try:
        for piece in (700, 50_001):  # 700: pieces of one read each, reads up to 800
            S.set_launch_config(chunk_chars=piece)
            out = torch.full((len(exp) + 8,), -7, dtype=torch.int64, device="cuda")
            assert idx.search_reads(d_chars, d_ends, out=out) == len(exp)
            got = out.cpu().numpy()
            assert np.array_equal(got[:len(exp)].view(np.uint64), exp)
            assert (got[len(exp):] == -7).all()
        small = torch.empty(len(exp) - 1, dtype=torch.int64, device="cuda")
        with pytest.raises(S.SbwtError) as e:
            idx.search_reads(d_chars, d_ends, out=small)
        assert e.value.code == S.E_CAPACITY
    finally:
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
        S.set_launch_config()


@pytest.mark.parametrize("kernel", [0, 1, 2, 6, 8])
def test_128_thread_blocks_match_oracle(kernel):
    """The read search kernels launched with 128-thread blocks (an autotuner
    axis): the oracle's results."""
    g, path, sb = synthetic(41, 3, 5000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 43, 2000, median=90, sigma=0.8, len_min=0, len_max=500,
                              sub=0.01, n_rate=0.01)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    S.set_table_kernel(kernel)
    S.set_block_threads(128)
    try:
        for tile in (0, 64):
            S.set_launch_config(tile=tile)
            assert np.array_equal(idx.search_reads(chars, ends), exp)
    finally:
        S.set_block_threads(256)
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
        S.set_launch_config()
    with pytest.raises(S.SbwtError):
        S.set_block_threads(512)


def test_errors_are_status_codes():
    with pytest.raises(S.SbwtError) as e:
        S.SbwtIndex.open("/nonexistent/file.sbwt")
    assert e.value.code == S.E_IO
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    idx = S.SbwtIndex.open(path)
    with pytest.raises(S.SbwtError) as e:
        idx.search_reads(b"ACGT" * 20, np.array([80], np.uint64), move_to_key_kmer=True)
    assert e.value.code == S.E_INVALID


@pytest.mark.parametrize("probe", [0, 0xFFFFFFFF, 5, 13, 20, 30])
def test_absent_prefix_probe_is_exact(probe):
    """The probe only skips k-mers it proves absent: results are identical
    for every probe length (0 = automatic, 0xFFFFFFFF = off)."""
    g, path, sb = synthetic(7, 4, 6000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    idx.set_kmer_table(False)  # the probe only runs on the search-walk path
    chars, ends = mixed_reads(g, 77, 3000, median=150, sigma=0.5, len_min=20,
                              len_max=600, sub=0.03, n_rate=0.005)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    S.set_probe_length(probe)
    try:
        got = idx.search_reads(chars, ends)
        got2 = idx.search_reads(chars, ends, per_kmer_walk=True)
    finally:
        S.set_probe_length(0)
    assert np.array_equal(got, exp) and np.array_equal(got2, exp)


@pytest.mark.parametrize("d", [2, 7])
@pytest.mark.parametrize("table", [True, False])
def test_move_to_key_kmer_matches_oracle_and_reference(d, table):
    """The d > 1 forward walk to the next key k-mer (reference flag -k)."""
    from helpers import key_marks_for
    g, path, sb = synthetic(9, 2, 3000, 31, 1, 0.02)
    oi = oracle_index(path, 8)
    keys = key_marks_for(oi, d, seed=d)
    idx = S.SbwtIndex.from_arrays(sb.acgt, sb.num_bits, sb.k, sb.suffix_group_starts,
                                  key_kmer_marks=keys)
    idx.set_kmer_table(table)
    chars, ends = mixed_reads(g, 13, 800, sub=0.01, n_rate=0.003)
    exp = np.concatenate(O.index_search_reads(oi, T.split_reads(chars, ends), keys))
    assert np.array_equal(idx.search_reads(chars, ends, move_to_key_kmer=True), exp)
    bits, _ = O.seq_to_bits(chars.tobytes())
    pos = O.positions_of(ends, 31)
    got = idx.search(bits, pos, move_to_key_kmer=True)
    assert np.array_equal(got, oi.search_positions(bits, pos, keys))
    if O.ref_lib() is not None:
        ref = O.OracleIndex(sb.acgt, sb.num_bits, sb.k, use_ref=True)
        assert np.array_equal(got, ref.search_positions(bits, pos, keys))


def test_tdbg_without_variant_string(tmp_path):
    """A .tdbg file is a .sbwt without the leading "plain-matrix" string
    (scripts/modifiers/themisto_tdbg_to_sbwt.py:23-32 of the reference)."""
    import struct
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    data = open(path, "rb").read()
    n = struct.unpack_from("<Q", data, 0)[0]
    assert data[8:8 + n] == b"plain-matrix"
    tdbg = tmp_path / "x.tdbg"
    tdbg.write_bytes(data[8 + n:])
    a, b = S.SbwtIndex.open(path), S.SbwtIndex.open(tdbg)
    chars, ends = mixed_reads(g, 5, 300)
    assert np.array_equal(a.search_reads(chars, ends), b.search_reads(chars, ends))


@pytest.mark.parametrize("p", [13, 14])
def test_deep_presearch_read_search_matches_oracle(p):
    # presearch tables deeper than the reference's 12 letters: same results
    g, path, sb = synthetic(6, 3, 6000, 31, 2, 0.02)
    chars, ends = mixed_reads(g, 9, 800)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    idx = S.SbwtIndex.open(path, presearch_letters=p)
    assert idx.presearch_letters == p
    assert np.array_equal(idx.search_reads(chars, ends), exp)
    with pytest.raises(S.SbwtError):
        S.SbwtIndex.open(path, presearch_letters=15)


def test_host_chunks_capacity_and_order_errors():
    """Host-pointer calls plan each chunk while the previous one runs: a too
    small results buffer and out-of-order read ends in a later chunk are
    still reported (after the chunks in flight finish), with the total k-mer
    count on E_CAPACITY, and the next call is unaffected."""
    import ctypes as C
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 21, 3000)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    L = S.lib()
    n_res = C.c_uint64()
    S.set_launch_config(chunk_chars=4096)  # many chunks
    try:
        out = np.zeros(len(exp), np.uint64)
        rc = L.sbwt_search_reads(idx._h, chars.ctypes.data, len(chars), ends.ctypes.data,
                                 len(ends), out.ctypes.data, len(exp) - 1, C.byref(n_res), 0,
                                 None)
        assert rc == S.E_CAPACITY and n_res.value == len(exp)
        bad = ends.copy()
        bad[-5] = bad[-6] - 1  # decreasing near the end: a later chunk
        rc = L.sbwt_search_reads(idx._h, chars.ctypes.data, len(chars), bad.ctypes.data,
                                 len(bad), out.ctypes.data, len(out), C.byref(n_res), 0, None)
        assert rc == S.E_INVALID
        assert np.array_equal(idx.search_reads(chars, ends), exp)
    finally:
        S.set_launch_config()


@pytest.mark.parametrize("k", [3, 15, 31])
def test_kmer_table_on_and_off(k):
    """The k-mer table (k <= 31) and the search walk give the oracle's results;
    the table can be dropped and rebuilt."""
    g, path, sb = synthetic(12, 2, 5000, k, 1, 0.02)
    idx = S.SbwtIndex.open(path)
    assert idx.set_kmer_table(True) > 0
    chars, ends = mixed_reads(g, 14, 600, median=80, sigma=0.5, len_min=0, len_max=300)
    exp = oracle_results(oracle_index(path, min(8, k)), chars, ends)
    assert np.array_equal(idx.search_reads(chars, ends), exp)
    assert idx.set_kmer_table(False) == 0
    assert np.array_equal(idx.search_reads(chars, ends), exp)
    assert idx.set_kmer_table(True) > 0
    assert np.array_equal(idx.search_reads(chars, ends, per_kmer_walk=True), exp)


@pytest.mark.parametrize("kernel", KERNEL_MODES)
@pytest.mark.parametrize("seed", [21, 22])
@pytest.mark.parametrize("k", [3, 15, 31])
def test_table_kernel_and_general_kernel_match_oracle(kernel, seed, k):
    """With a k-mer table the read search runs on the general kernel, the
    table kernel (stream steps, group scans and table lookups only) or the
    walks kernel (the same steps behind the k-mer filter, several tiles per
    lane, 32-byte result stores); all give the oracle's results on reads
    with errors, N, empty and short reads, at several tile sizes (k-mers of
    one read split across tiles, tiles that are not multiples of 4)."""
    g, path, sb = synthetic(30 + seed, 3, 5000, k, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    assert idx.set_kmer_table(True) > 0
    chars, ends = mixed_reads(g, seed, 1500, median=70, sigma=0.8, len_min=0, len_max=400,
                              sub=0.01, n_rate=0.01)
    exp = oracle_results(oracle_index(path, min(8, k)), chars, ends)
    S.set_table_kernel(kernel)
    try:
        for tile in (0, 16, 37, 100, 5000):
            S.set_launch_config(tile=tile)
            assert np.array_equal(idx.search_reads(chars, ends), exp), tile
    finally:
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
        S.set_launch_config()


@pytest.mark.parametrize("kernel", KERNEL_MODES[1:])
@pytest.mark.parametrize("shift", [0, 1, 3])
def test_table_kernel_device_pointers_and_capacity(kernel, shift):
    """The table and walks kernels through device pointers: exact, they write
    no slot past the k-mer count (the guard slots keep their fill), also
    when the output is not 32-byte aligned (shift: 8-byte elements)."""
    import torch
    g, path, sb = synthetic(31, 3, 5000, 31, 2, 0.02)
    idx = S.SbwtIndex.open(path)
    assert idx.set_kmer_table(True) > 0
    chars, ends = mixed_reads(g, 23, 3000, median=120, sigma=0.6, len_min=0, len_max=600,
                              sub=0.005, n_rate=0.002)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    d_chars = torch.from_numpy(chars.copy()).cuda()
    d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
    buf = torch.full((len(exp) + 64 + shift,), -7, dtype=torch.int64, device="cuda")
    out = buf[shift:]
    S.set_table_kernel(kernel)
    try:
        assert idx.search_reads(d_chars, d_ends, out=out) == len(exp)
    finally:
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
    got = buf.cpu().numpy()
    assert (got[:shift] == -7).all()
    assert np.array_equal(got[shift:shift + len(exp)].view(np.uint64), exp)
    assert (got[shift + len(exp):] == -7).all()


@pytest.mark.parametrize("kernel", [DEFAULT_TABLE_KERNEL, 1, 11, 17])
def test_device_pointers_bad_read_ends(kernel):
    """Device-pointer calls queue the search right after the scan, with no
    host check in between: read ends that decrease or pass n_chars scan to
    zero k-mers, nothing is written, the call returns SBWT_E_INVALID, and the
    next call on the handle is unaffected."""
    import torch
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    idx = S.SbwtIndex.open(path)
    assert idx.set_kmer_table(True) > 0
    chars, ends = mixed_reads(g, 21, 3000)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    d_chars = torch.from_numpy(chars.copy()).cuda()
    decreasing = ends.copy()
    decreasing[len(ends) // 2] = decreasing[len(ends) // 2 - 1] - 1
    past_end = ends.copy()
    past_end[-1] = len(chars) + 100
    S.set_table_kernel(kernel)
    try:
        for bad in (decreasing, past_end):
            d_bad = torch.from_numpy(bad.view(np.int64).copy()).cuda()
            out = torch.full((len(exp) + 8,), -7, dtype=torch.int64, device="cuda")
            with pytest.raises(S.SbwtError) as e:
                idx.search_reads(d_chars, d_bad, out=out)
            assert e.value.code == S.E_INVALID
            assert (out.cpu().numpy() == -7).all()
        d_ends = torch.from_numpy(ends.view(np.int64).copy()).cuda()
        out = torch.empty(len(exp), dtype=torch.int64, device="cuda")
        assert idx.search_reads(d_chars, d_ends, out=out) == len(exp)
        assert np.array_equal(out.cpu().numpy().view(np.uint64), exp)
    finally:
        S.set_table_kernel(DEFAULT_TABLE_KERNEL)
    idx.close()
