"""Malformed .sbwt / .tcolors files are status codes, never crashes: truncated
files at every section, int vectors wider than 64 bits, and color set
indexes, sparse color ids and dense intervals past their arrays (the color
set indexes are range-checked by the device kernel that widens them)."""
import struct

import numpy as np
import pytest

import sbwt_b200 as S
import sbwt_tools as T
from helpers import TMP, synthetic

pytestmark = pytest.mark.gpu


CASES = {12: (41, 12, 3000, 3), 150: (45, 150, 800, 6)}  # colors: seed, genomes, bp, founders


def colored_files(n_colors=12):
    seed, n, length, founders = CASES[n_colors]
    sp, cp = TMP / f"malformed_{n}.sbwt", TMP / f"malformed_{n}.tcolors"
    if not cp.exists():
        g = T.gen_genomes(seed, n, length, founders, 0.01, 0.05, 0.0)
        T.build_colored(g, 31, str(sp), str(cp))
    return sp.read_bytes(), cp.read_bytes()


def tcolors_sections(data: bytes):
    """name -> (offset of the section's u64 length field, offset of its words,
    words, width or None) in the sdsl-hybrid-v4 member order."""
    off = 8 + struct.unpack_from("<Q", data, 0)[0]
    out = {}
    for name, kind in (("dense", "bv"), ("dense_iv", "iv"), ("sparse", "iv"),
                       ("sparse_iv", "iv"), ("is_dense", "bv"), ("is_dense_rank", "bv"),
                       ("key_marks", "bv"), ("key_rank", "bv"), ("csi", "iv")):
        head = off
        bits = struct.unpack_from("<Q", data, off)[0]
        off += 8
        width = None
        if kind == "iv":
            width = data[off]
            off += 1
        nw = (bits + 63) // 64
        out[name] = (head, off, nw, width, bits)
        off += 8 * nw
    return out


def set_entry(data: bytearray, sec, i: int, value: int):
    """Writes entry i of an int vector section (LSB-first packing)."""
    _, at, nw, w, _ = sec
    words = np.frombuffer(bytes(data[at:at + 8 * nw]), dtype=np.uint64).copy()
    bit = i * w
    v = value & ((1 << w) - 1)
    for b in range(w):
        p = bit + b
        word, off = p // 64, p % 64
        if (v >> b) & 1:
            words[word] |= np.uint64(1 << off)
        else:
            words[word] &= ~np.uint64(1 << off)
    data[at:at + 8 * nw] = words.tobytes()


def open_colors_bytes(data: bytes, name: str):
    p = TMP / name
    p.write_bytes(bytes(data))
    return S.ColorIndex.open(str(p))


def expect_format_error(fn, text=None):
    with pytest.raises(S.SbwtError) as e:
        fn()
    assert e.value.code == S.E_FORMAT, (e.value.code, str(e.value))
    if text:
        assert text in str(e.value)


@pytest.mark.parametrize("n_colors", sorted(CASES))
def test_colors_file_opens_and_missing_is_io_error(n_colors):
    _, cdata = colored_files(n_colors)
    ci = open_colors_bytes(cdata, "malformed_ok.tcolors")
    assert ci.num_colors == n_colors
    with pytest.raises(S.SbwtError) as e:
        S.ColorIndex.open(str(TMP / "no_such_file.tcolors"))
    assert e.value.code == S.E_IO


def test_truncated_colors_file():
    _, cdata = colored_files()
    secs = tcolors_sections(cdata)
    cuts = {0, 4, 12, len(cdata) - 1, len(cdata) - 20}
    for head, at, nw, _, _ in secs.values():
        cuts |= {head + 3, at + 4 * nw}
    for cut in sorted(c for c in cuts if 0 <= c < len(cdata)):
        expect_format_error(lambda: open_colors_bytes(cdata[:cut], "malformed_cut.tcolors"))


def test_truncated_index_file():
    _, path, _ = synthetic(43, 2, 3000, 31, 1, 0.02)
    data = open(path, "rb").read()
    for cut in (0, 5, 20, 60, len(data) // 3, len(data) // 2, len(data) - 8, len(data) - 1):
        p = TMP / "malformed_cut.sbwt"
        p.write_bytes(data[:cut])
        expect_format_error(lambda: S.SbwtIndex.open(str(p)))


def test_int_vector_wider_than_64_bits():
    _, cdata = colored_files()
    head = tcolors_sections(cdata)["csi"][0]
    bad = bytearray(cdata)
    bad[head + 8] = 65
    expect_format_error(lambda: open_colors_bytes(bad, "malformed_width.tcolors"),
                        "int vector width")


@pytest.mark.parametrize("n_colors", sorted(CASES))
@pytest.mark.parametrize("entry", [0, 7, -1])
def test_color_set_index_past_the_sets(entry, n_colors):
    _, cdata = colored_files(n_colors)
    secs = tcolors_sections(cdata)
    n_sets = secs["is_dense"][4]
    _, _, _, w, bits = secs["csi"]
    assert (1 << w) - 1 >= n_sets  # an out-of-range value fits the width
    bad = bytearray(cdata)
    set_entry(bad, secs["csi"], entry % (bits // w), (1 << w) - 1)
    expect_format_error(lambda: open_colors_bytes(bad, "malformed_csi.tcolors"),
                        "color set index out of range")


@pytest.mark.parametrize("entry", [0, -1])
def test_sparse_color_id_past_the_colors(entry):
    _, cdata = colored_files(150)
    secs = tcolors_sections(cdata)
    _, _, _, w, bits = secs["sparse"]
    assert bits > 0 and (1 << w) - 1 >= 150
    bad = bytearray(cdata)
    set_entry(bad, secs["sparse"], entry % (bits // w), (1 << w) - 1)
    expect_format_error(lambda: open_colors_bytes(bad, "malformed_sparse.tcolors"),
                        "sparse color id out of range")


@pytest.mark.parametrize("n_colors", sorted(CASES))
def test_dense_interval_past_the_rows(n_colors):
    _, cdata = colored_files(n_colors)
    secs = tcolors_sections(cdata)
    _, _, _, w, bits = secs["dense_iv"]
    assert bits // w >= 2 and (1 << w) - 1 > secs["dense"][4]
    bad = bytearray(cdata)
    set_entry(bad, secs["dense_iv"], 1, (1 << w) - 1)
    expect_format_error(lambda: open_colors_bytes(bad, "malformed_dense.tcolors"),
                        "dense interval out of range")


@pytest.mark.parametrize("section", ["dense", "csi", "key_rank"])
def test_vector_length_past_the_file(section):
    """A length field larger than the rest of the file is a format error
    before anything is allocated for it (not an out-of-memory status)."""
    _, cdata = colored_files()
    head = tcolors_sections(cdata)[section][0]
    for bits in (1 << 40, (1 << 64) - 1):
        bad = bytearray(cdata)
        bad[head:head + 8] = struct.pack("<Q", bits)
        expect_format_error(lambda: open_colors_bytes(bad, "malformed_len.tcolors"),
                            "unexpected end of file")
