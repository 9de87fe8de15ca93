"""Host I/O of the drop-in boundary (no GPU): the FASTA/FASTQ reader, the
index-result writers and the index-file reader reproduce the reference's
formats byte for byte on its own fixtures."""
import ctypes as C
import struct

import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
from helpers import FIXTURE_FILES, GOLDEN, TMP, golden_sbwt_path, oracle_index

U64P = C.POINTER(C.c_uint64)


def lib():
    L = S.lib()
    L.sbwt_fastx_read.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.sbwt_free.argtypes = [C.c_void_p]
    L.sbwt_write_index_results.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_uint64, C.c_uint32]
    L.sbwt_read_index_results.argtypes = [C.c_char_p] + [C.POINTER(C.c_void_p)] * 4 + \
        [C.POINTER(C.c_uint64)]
    L.sbwt_write_color_results.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_uint64, C.c_uint64]
    return L


def fastx_read(path):
    L = lib()
    ch, en = C.c_void_p(), C.c_void_p()
    nc, nr = C.c_uint64(), C.c_uint64()
    S.check(L.sbwt_fastx_read(str(path).encode(), C.byref(ch), C.byref(nc), C.byref(en),
                              C.byref(nr)))
    chars = C.string_at(ch, nc.value) if nc.value else b""
    ends = np.ctypeslib.as_array(C.cast(en, U64P), (max(nr.value, 1),))[:nr.value].copy()
    L.sbwt_free(ch)
    L.sbwt_free(en)
    return chars, ends


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_fastx_reader_matches_kseq_rules(name):
    chars, ends = fastx_read(GOLDEN / "index_search" / name)
    reads = O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    assert chars == b"".join(reads)
    assert ends.tolist() == np.cumsum([len(r) for r in reads]).tolist()


def test_fastx_reader_gzip_and_edge_cases(tmp_path):
    import gzip
    data = b">a\r\nAC\r\nGT\n>b\n>c\nTT\n\n@q x\nACG\nT\n+\nII\nII\n@r\n\n+\n\n"
    p = tmp_path / "x.fq.gz"
    with gzip.open(p, "wb") as f:
        f.write(data)
    chars, ends = fastx_read(p)
    assert chars == b"ACGTTTACGT"
    assert ends.tolist() == [4, 4, 6, 10, 10]


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_ascii_writer_reproduces_reference_bytes(name):
    idx = oracle_index(golden_sbwt_path(), 10)
    chars, ends = fastx_read(GOLDEN / "index_search" / name)
    reads = O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    res = np.concatenate(O.index_search_reads(idx, reads) + [np.zeros(0, np.uint64)])
    res = np.ascontiguousarray(res.astype(np.uint64))
    out = TMP / ("w_" + name.split(".")[0])
    S.check(lib().sbwt_write_index_results(str(out).encode(), 0, 1,
                                           res.ctypes.data if len(res) else None,
                                           ends.ctypes.data if len(ends) else None,
                                           len(ends), 30))
    exp = (GOLDEN / "index_search" / "expected" / (name.split(".")[0] + ".txt")).read_bytes()
    assert (TMP / ("w_" + name.split(".")[0] + ".txt")).read_bytes() == exp


def test_binary_and_bool_writers():
    res = np.array([5, O.NOT_FOUND, O.INVALID, 7], np.uint64)
    ends = np.array([33, 33, 64], np.uint64)  # 3 + 0 + 1 k-mers at k=31
    for fmt, ext in ((1, ".bin"), (2, ".bool")):
        out = TMP / f"wb_{fmt}"
        S.check(lib().sbwt_write_index_results(str(out).encode(), fmt, 1, res.ctypes.data,
                                               ends.ctypes.data, 3, 31))
        b = (TMP / f"wb_{fmt}{ext}").read_bytes()
        if fmt == 1:
            assert b[:8 + 6 + 8 + 4] == struct.pack("<Q", 6) + b"binary" + struct.pack("<Q", 4) + b"v1.0"
            vals = np.frombuffer(b[26:], np.uint64).tolist()
            m3 = (1 << 64) - 3
            assert vals == [5, O.NOT_FOUND, O.INVALID, m3, m3, 7, m3]
        else:
            assert b[8 + 4 + 8 + 4:] == b"012\n\n0\n"


def test_index_file_reader_on_reference_fixtures():
    L = lib()
    for name in ("fasta1", "fasta2", "fasta3", "fasta4"):
        path = GOLDEN / "color_search" / f"{name}.indexes.txt"
        ptrs = [C.c_void_p() for _ in range(4)]
        n = C.c_uint64()
        S.check(L.sbwt_read_index_results(str(path).encode(), *[C.byref(p) for p in ptrs],
                                          C.byref(n)))
        nr = n.value
        offs = np.ctypeslib.as_array(C.cast(ptrs[1], U64P), (nr + 1,)).copy()
        found = np.ctypeslib.as_array(C.cast(ptrs[0], U64P), (max(int(offs[-1]), 1),))
        nf = np.ctypeslib.as_array(C.cast(ptrs[2], U64P), (max(nr, 1),))
        inv = np.ctypeslib.as_array(C.cast(ptrs[3], U64P), (max(nr, 1),))
        rows = O.read_ascii_index_results(path)
        assert nr == len(rows)
        for r, toks in enumerate(rows):
            assert found[offs[r]:offs[r + 1]].tolist() == [t for t in toks if t >= 0]
            assert nf[r] == toks.count(-1) and inv[r] == toks.count(-2)
        for p in ptrs:
            L.sbwt_free(p)


def test_color_writers():
    ids = np.array([0, 2, 1], np.uint32)
    offs = np.array([0, 2, 2, 3], np.uint64)
    L = lib()
    for fmt, ext in ((0, ".txt"), (1, ".bin"), (2, ".csv")):
        out = TMP / f"cw_{fmt}"
        S.check(L.sbwt_write_color_results(str(out).encode(), fmt, 1, ids.ctypes.data,
                                           offs.ctypes.data, 3, 3))
        b = (TMP / f"cw_{fmt}{ext}").read_bytes()
        if fmt == 0:
            assert b == struct.pack("<Q", 5) + b"ascii" + struct.pack("<Q", 4) + b"v1.0" + b"0 2\n\n1\n"
        elif fmt == 1:
            vals = np.frombuffer(b[26:], np.uint64).tolist()
            assert vals == [0, 2, O.NOT_FOUND, O.NOT_FOUND, 1, O.NOT_FOUND]
        else:
            assert b == b"1,2,3\n1,0,1\n0,0,0\n0,1,0\n"


@pytest.mark.parametrize("seed", range(6))
def test_fastx_reader_matches_oracle_on_random_text(seed, tmp_path):
    from helpers import host_fastx, random_fastx
    text = random_fastx(seed, 300, final_newline=seed % 2 == 0)
    chars, ends = host_fastx(text, tmp_path / "r.fx")
    reads = O.parse_fastx(text)
    assert chars == b"".join(reads)
    assert ends.tolist() == np.cumsum([len(r) for r in reads]).tolist()


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("tail_newline", [True, False])
def test_index_file_reader_large_file_in_parts(tail_newline, binary):
    """A file over 16 MB is parsed in parts of whole reads on host threads
    (ascii lines, or binary reads ended by -3 words): the joined result
    equals the rows written (values, -1 and -2 counts, empty rows, and an
    unterminated last row)."""
    rng = np.random.default_rng(5)
    n_rows = 600_000
    lens = rng.integers(0, 40, n_rows)
    lens[rng.random(n_rows) < 0.05] = 0
    lens[-2] = 0
    if tail_newline:
        lens[-1] = 0  # trailing empty rows
    vals = rng.integers(0, 1 << 40, int(lens.sum()))
    kinds = rng.random(len(vals))
    vals[kinds < 0.1] = -1
    vals[(kinds >= 0.1) & (kinds < 0.15)] = -2
    starts = np.concatenate([[0], np.cumsum(lens)])
    path = TMP / f"big_index_results_{int(tail_newline)}_{int(binary)}.txt"
    if binary:
        words = np.full(len(vals) + n_rows, np.uint64(2**64 - 3))
        words[np.arange(len(vals)) + np.repeat(np.arange(n_rows), lens)] = vals.astype(np.uint64)
        if not tail_newline:
            words = words[:-1]
            if lens[-1] == 0:
                words = np.concatenate([words, np.array([5], np.uint64)])
        path.write_bytes(struct.pack("<Q", 6) + b"binary" + struct.pack("<Q", 4) + b"v1.0" +
                         words.tobytes())
    else:
        lines = [" ".join(map(str, vals[starts[r]:starts[r + 1]])) for r in range(n_rows)]
        if not tail_newline:
            lines[-1] = lines[-1] or "5"
        body = "\n".join(lines) + ("\n" if tail_newline else "")
        path.write_bytes(struct.pack("<Q", 5) + b"ascii" + struct.pack("<Q", 4) + b"v1.0" +
                         body.encode())
    assert path.stat().st_size > 40 << 20  # several parts
    L = lib()
    ptrs = [C.c_void_p() for _ in range(4)]
    n = C.c_uint64()
    S.check(L.sbwt_read_index_results(str(path).encode(), *[C.byref(p) for p in ptrs],
                                      C.byref(n)))
    try:
        assert n.value == n_rows
        offs = np.ctypeslib.as_array(C.cast(ptrs[1], U64P), (n_rows + 1,)).copy()
        found = np.ctypeslib.as_array(C.cast(ptrs[0], U64P), (max(int(offs[-1]), 1),))
        nf = np.ctypeslib.as_array(C.cast(ptrs[2], U64P), (n_rows,))
        inv = np.ctypeslib.as_array(C.cast(ptrs[3], U64P), (n_rows,))
        if not tail_newline and lens[-1] == 0:
            lens = lens.copy()
            lens[-1] = 1
            vals = np.concatenate([vals, [5]])
        pos = vals >= 0
        row = np.repeat(np.arange(n_rows), lens)
        exp_found_per_row = np.bincount(row[pos], minlength=n_rows)
        exp_nf = np.bincount(row[vals == -1], minlength=n_rows)
        exp_inv = np.bincount(row[vals == -2], minlength=n_rows)
        assert np.array_equal(np.diff(offs), exp_found_per_row)
        assert np.array_equal(nf, exp_nf) and np.array_equal(inv, exp_inv)
        assert np.array_equal(found[:int(offs[-1])], vals[pos].astype(np.uint64))
    finally:
        for p in ptrs:
            L.sbwt_free(p)


def scan_index_body(body: bytes):
    """The ascii index-results body token by token, as the reader specifies
    it: a newline ends a read; '-' counts a not-found / invalid when the next
    byte is '1' / '2' and skips the bytes from '0' up to 0x7f after it; a
    digit run is a found value modulo 2^64; other bytes are skipped; a tail
    with tokens after the last newline is one more read."""
    found, offs, nf, inv = [], [0], [], []
    c_nf = c_inv = 0
    open_read = False
    i, n = 0, len(body)
    while i < n:
        c = body[i]
        if c == 10:
            offs.append(len(found)); nf.append(c_nf); inv.append(c_inv)
            c_nf = c_inv = 0
            open_read = False
            i += 1
        elif c == 45:
            if i + 1 < n and body[i + 1] == 49:
                c_nf += 1
            elif i + 1 < n and body[i + 1] == 50:
                c_inv += 1
            i += 1
            while i < n and 48 <= body[i] < 128:
                i += 1
            open_read = True
        elif 48 <= c <= 57:
            v = 0
            while i < n and 48 <= body[i] <= 57:
                v = (v * 10 + body[i] - 48) % (1 << 64)
                i += 1
            found.append(v)
            open_read = True
        else:
            i += 1
    if open_read:
        offs.append(len(found)); nf.append(c_nf); inv.append(c_inv)
    return found, offs, nf, inv


def random_index_body(rng, n_bytes: int, other: bytes = b"") -> bytes:
    """Lines of numbers of 1..21 digits, -1 / -2 / other negatives, runs of
    spaces, empty lines and stray '-', cut at n_bytes; `other` bytes are
    sprinkled in when given."""
    parts = []
    size = 0
    while size < n_bytes:
        r = rng.random()
        if r < 0.55:
            t = str(int(rng.integers(0, 10 ** int(rng.integers(1, 10)))))
            if rng.random() < 0.05:
                t = "".join(map(str, rng.integers(0, 10, int(rng.integers(10, 22)))))
        elif r < 0.65:
            t = ["-1", "-2", "-3", "-12", "--1", "-", "-21"][int(rng.integers(0, 7))]
        elif r < 0.8:
            t = " " * int(rng.integers(1, 4))
        elif r < 0.9:
            t = "\n"
        else:
            t = " "
        if other and rng.random() < 0.01:
            t += chr(other[int(rng.integers(0, len(other)))])
        parts.append(t)
        size += len(t)
    return "".join(parts).encode("latin-1")[:n_bytes]


@pytest.mark.parametrize("case", [(1, 3000, b""), (2, 5000, b""), (3, 777, b"x\r"),
                                  (4, 12 << 20, b""), (5, 9 << 20, b"\r\t")])
def test_index_file_reader_matches_scanner_rules(case):
    """The reader (a byte-class fast path for bodies of digits, spaces,
    newlines and '-', the byte-by-byte scanner otherwise, parts on host
    threads) equals the token rules on random bodies."""
    seed, n_bytes, other = case
    rng = np.random.default_rng(seed)
    body = random_index_body(rng, n_bytes, other)
    path = TMP / f"index_body_{seed}.txt"
    path.write_bytes(struct.pack("<Q", 5) + b"ascii" + struct.pack("<Q", 4) + b"v1.0" + body)
    found, offs, nf, inv = scan_index_body(body)
    L = lib()
    ptrs = [C.c_void_p() for _ in range(4)]
    n = C.c_uint64()
    S.check(L.sbwt_read_index_results(str(path).encode(), *[C.byref(p) for p in ptrs],
                                      C.byref(n)))
    try:
        nr = n.value
        assert nr == len(nf)
        got_offs = np.ctypeslib.as_array(C.cast(ptrs[1], U64P), (nr + 1,))
        assert got_offs.tolist() == offs
        got_found = np.ctypeslib.as_array(C.cast(ptrs[0], U64P), (max(len(found), 1),))
        assert got_found[:len(found)].tolist() == found
        if nr:
            assert np.ctypeslib.as_array(C.cast(ptrs[2], U64P), (nr,)).tolist() == nf
            assert np.ctypeslib.as_array(C.cast(ptrs[3], U64P), (nr,)).tolist() == inv
    finally:
        for p in ptrs:
            L.sbwt_free(p)


def _read_results(path):
    L = lib()
    ptrs = [C.c_void_p() for _ in range(4)]
    n = C.c_uint64()
    rc = L.sbwt_read_index_results(str(path).encode(), *[C.byref(p) for p in ptrs], C.byref(n))
    if rc == S.OK:
        for p in ptrs:
            L.sbwt_free(p)
    return rc, n.value


def test_index_file_reader_errors():
    """Missing files are SBWT_E_IO; bad headers are SBWT_E_FORMAT; a header
    with an empty body is zero reads (no GPU involved)."""
    hdr = lambda fmt, ver=b"v1.0": (struct.pack("<Q", len(fmt)) + fmt +
                                     struct.pack("<Q", len(ver)) + ver)
    assert _read_results(TMP / "no_such_results.txt")[0] == S.E_IO
    cases = {
        "empty": b"",
        "short_len": b"\x05\x00\x00",
        "long_name": struct.pack("<Q", 1 << 40) + b"ascii",
        "unknown_format": hdr(b"fasta") + b"1 2 3\n",
        "bad_version": hdr(b"ascii", b"v9.9") + b"1 2 3\n",
        "cut_name": struct.pack("<Q", 6) + b"bin",
    }
    for name, data in cases.items():
        p = TMP / f"bad_results_{name}.txt"
        p.write_bytes(data)
        assert _read_results(p)[0] == S.E_FORMAT, name
    for fmt in (b"ascii", b"binary"):
        p = TMP / f"empty_results_{fmt.decode()}.txt"
        p.write_bytes(hdr(fmt))
        assert _read_results(p) == (S.OK, 0)
