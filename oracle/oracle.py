"""Python side of the oracle: loaders for the two CPU checkers.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline / reference legs may import this module.  It wraps

  * oracle/_build/liboracle.so -- the C restatement in oracle/sbwt_oracle.c;
  * oracle/_ref/libsbwt_ref.so -- SBWT-Search's own index kernels compiled for
    the host (oracle/ref_driver.cpp, oracle/Makefile);

and adds plain-Python readers for the reference's file formats that the
checkers need (.sbwt / .tdbg: src/SbwtBuilder/SbwtBuilder.cpp:58-104; FASTA /
FASTQ with kseq record semantics; ascii index results:
src/IndexResultsPrinter/AsciiContinuousIndexResultsPrinter.cpp:50-95).
These readers are independent of the product's C++ loaders on purpose.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import struct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_SO = HERE / "_ref" / "libsbwt_ref.so"

U64P = C.POINTER(C.c_uint64)
NOT_FOUND = (1 << 64) - 1
INVALID = (1 << 64) - 2


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(U64P)


def _ptr_array(arrs):
    return (U64P * 4)(*[_p(a) for a in arrs])


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            raise RuntimeError(f"{ORACLE_SO} missing: run `make -C oracle`")
        L = C.CDLL(str(ORACLE_SO))
        L.oracle_poppy_sizes.argtypes = [C.c_uint64, U64P, U64P]
        L.oracle_poppy_build.argtypes = [U64P, C.c_uint64, U64P, U64P]
        L.oracle_poppy_build.restype = C.c_uint64
        L.oracle_rank.argtypes = [U64P, U64P, U64P, C.c_uint64]
        L.oracle_rank.restype = C.c_uint64
        L.oracle_varint.argtypes = [U64P, C.c_uint32, C.c_uint64]
        L.oracle_varint.restype = C.c_uint64
        L.oracle_presearch.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, U64P,
                                       C.c_uint32, U64P, U64P]
        L.oracle_search.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                    U64P, C.c_uint32, U64P, U64P, U64P, U64P,
                                    C.c_uint64, C.c_void_p, U64P]
        L.oracle_seq_to_bits.argtypes = [C.c_char_p, C.c_uint64, U64P, C.c_void_p]
        L.oracle_positions.argtypes = [U64P, C.c_uint64, C.c_uint32, C.c_void_p]
        L.oracle_positions.restype = C.c_uint64
        L.oracle_mask_invalid.argtypes = [C.c_void_p, U64P, C.c_uint64, C.c_uint32,
                                          U64P]
        L.oracle_walk_sectors.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p,
                                          C.c_void_p, U64P, C.c_uint32, U64P, U64P,
                                          U64P, U64P, C.c_uint64]
        L.oracle_walk_sectors.restype = C.c_uint64
        L.oracle_pseudoalign.argtypes = [C.c_void_p, U64P, U64P, U64P, U64P,
                                         C.c_uint64, C.c_double, C.c_int, C.c_int,
                                         C.c_void_p, U64P, C.c_void_p]
        L.oracle_pseudoalign.restype = C.c_uint64
        L.oracle_pseudoalign_mt.argtypes = [C.c_void_p, U64P, U64P, U64P, U64P,
                                            C.c_uint64, C.c_double, C.c_int, C.c_int,
                                            U64P, U64P, C.c_int]
        L.oracle_pseudoalign_mt.restype = C.c_uint64
        _lib = L
    return _lib


def ref_lib():
    """SBWT-Search's own index and colors kernels compiled for the host (or
    None when oracle/_ref was not built)."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            return None
        L = C.CDLL(str(REF_SO))
        L.ref_poppy_sizes.argtypes = [C.c_uint64, U64P, U64P]
        L.ref_poppy_build.argtypes = [U64P, C.c_uint64, U64P, U64P]
        L.ref_poppy_build.restype = C.c_uint64
        L.ref_presearch.argtypes = [U64P, C.c_void_p, C.c_void_p, C.c_void_p, U64P,
                                    U64P, C.c_int]
        L.ref_search.argtypes = [C.c_uint, U64P, C.c_void_p, C.c_void_p, C.c_void_p,
                                 U64P, U64P, U64P, U64P, C.c_void_p, C.c_uint64,
                                 U64P, C.c_int]
        L.ref_max_threads.restype = C.c_int
        L.ref_color_counts.argtypes = [
            U64P, C.c_uint64, U64P, U64P, U64P, U64P, C.c_uint32, U64P, U64P, U64P,
            U64P, U64P, C.c_uint32, U64P, C.c_uint32, U64P, C.c_uint32, C.c_uint64,
            U64P, C.c_uint64, U64P, C.c_int]
        L.ref_color_counts.restype = C.c_int
        _ref = L
    return _ref


# --------------------------------------------------------------------------
# File readers
# --------------------------------------------------------------------------
class SbwtFile:
    """The parts of a .sbwt/.tdbg file the search uses
    (src/SbwtBuilder/SbwtBuilder.cpp:58-104): the A/C/G/T bitvectors, their
    length in bits and k.  The suffix-group-start bitvector is kept too."""

    def __init__(self, data: bytes):
        off = 0

        def u64():
            nonlocal off
            v = struct.unpack_from("<Q", data, off)[0]
            off += 8
            return v

        def string():
            nonlocal off
            n = u64()
            s = data[off:off + n]
            off += n
            return s

        variant = string()
        if variant != b"v0.1":
            if variant != b"plain-matrix":
                raise ValueError("Error input is not a plain-matrix SBWT")
            if string() != b"v0.1":
                raise ValueError("Error: wrong SBWT version")

        def bitvector():
            nonlocal off
            nb = u64()
            nw = (nb + 63) // 64
            a = np.frombuffer(data, dtype=np.uint64, count=nw, offset=off).copy()
            off += nw * 8
            return nb, a

        self.acgt = []
        for _ in range(4):
            nb, a = bitvector()
            self.acgt.append(a)
        self.num_bits = nb
        for _ in range(4):
            bitvector()  # rank structures (not used)
        _, self.suffix_group_starts = bitvector()
        for _ in range(2):  # C map, k-mer prefix precalc table
            n_bytes = u64()
            off += n_bytes
        self.precalc_k, self.n_nodes, self.n_kmers, self.k = (u64(), u64(), u64(),
                                                             u64())

    @classmethod
    def read(cls, path) -> "SbwtFile":
        path = str(path)
        if path.endswith(".gz"):
            import gzip
            with gzip.open(path, "rb") as f:
                return cls(f.read())
        with open(path, "rb") as f:
            return cls(f.read())


def parse_fastx(data: bytes) -> list[bytes]:
    """FASTA/FASTQ records with kseq semantics: a record starts at '>' or
    '@'; its sequence is the concatenation of the following lines up to a line
    that starts with '>', '+' or '@'; after '+' quality lines are consumed until
    they are at least as long as the sequence.  Empty records are kept."""
    lines = data.split(b"\n")
    seqs = []
    i = 0
    n = len(lines)
    while i < n and not (lines[i][:1] in (b">", b"@")):
        i += 1
    while i < n:
        i += 1  # header
        seq = []
        while i < n and lines[i][:1] not in (b">", b"+", b"@"):
            seq.append(lines[i].rstrip(b"\r"))
            i += 1
        s = b"".join(seq)
        if i < n and lines[i][:1] == b"+":
            i += 1
            q = 0
            while i < n and q < len(s):
                q += len(lines[i].rstrip(b"\r"))
                i += 1
        seqs.append(s)
        while i < n and lines[i][:1] not in (b">", b"@"):
            i += 1
    return seqs


def read_ascii_index_results(path) -> list[list[int]]:
    """Ascii index results (header "ascii"/"v1.0" length-prefixed strings,
    then one line per read of space-separated tokens)."""
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    for expect in (b"ascii", b"v1.0"):
        n = struct.unpack_from("<Q", data, off)[0]
        assert data[off + 8:off + 8 + n] == expect
        off += 8 + n
    body = data[off:].decode()
    lines = body.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    return [[int(t) for t in ln.split()] for ln in lines]


# --------------------------------------------------------------------------
# Index step
# --------------------------------------------------------------------------
class OracleIndex:
    """Poppy layers + C-map + presearch table over an SBWT, computed by the C
    restatement (or, with use_ref=True, by the reference's own code)."""

    def __init__(self, acgt, num_bits: int, k: int, presearch_letters: int = 12,
                 use_ref: bool = False):
        self.acgt = [np.ascontiguousarray(a, dtype=np.uint64) for a in acgt]
        self.num_bits = int(num_bits)
        self.k = int(k)
        self.use_ref = use_ref
        L = ref_lib() if use_ref else lib()
        if L is None:
            raise RuntimeError("reference CPU build missing: run `make -C oracle ref`")
        sizes = (L.ref_poppy_sizes if use_ref else L.oracle_poppy_sizes)
        build = (L.ref_poppy_build if use_ref else L.oracle_poppy_build)
        n0, n12 = C.c_uint64(), C.c_uint64()
        sizes(self.num_bits, C.byref(n0), C.byref(n12))
        self.l0, self.l12, self.acgt_pad, totals = [], [], [], []
        for a in self.acgt:
            # pad each vector: the reference kernel reads the whole 256-bit basic
            # block that contains position num_bits.
            a_pad = np.zeros(((self.num_bits + 255) // 256) * 4 + 4, dtype=np.uint64)
            a_pad[:len(a)] = a
            l0 = np.zeros(n0.value, dtype=np.uint64)
            l12 = np.zeros(n12.value, dtype=np.uint64)
            totals.append(build(_p(a_pad), self.num_bits, _p(l0), _p(l12)))
            self.acgt_pad.append(a_pad)
            self.l0.append(l0)
            self.l12.append(l12)
        self.totals = totals
        c = [1]
        for t in totals:
            c.append(c[-1] + int(t))
        self.c_map = np.array(c, dtype=np.uint64)
        self.p = 12 if use_ref else int(presearch_letters)
        n = 1 << (2 * self.p)
        self.pre_left = np.zeros(n, dtype=np.uint64)
        self.pre_right = np.zeros(n, dtype=np.uint64)
        if use_ref:
            L.ref_presearch(_p(self.c_map), _ptr_array(self.acgt_pad),
                            _ptr_array(self.l0), _ptr_array(self.l12),
                            _p(self.pre_left), _p(self.pre_right),
                            L.ref_max_threads())
        else:
            L.oracle_presearch(_ptr_array(self.acgt_pad), _ptr_array(self.l0),
                               _ptr_array(self.l12), _p(self.c_map), self.p,
                               _p(self.pre_left), _p(self.pre_right))

    def search_positions(self, bit_seqs: np.ndarray, positions: np.ndarray,
                         key_marks: np.ndarray | None = None,
                         threads: int | None = None) -> np.ndarray:
        """Raw kernel output over packed sequences + k-mer positions: the
        node index or UINT64_MAX (invalid chars are searched as 'A')."""
        bit_seqs = np.ascontiguousarray(bit_seqs, dtype=np.uint64)
        bit_seqs = np.concatenate([bit_seqs, np.zeros(2, np.uint64)])
        positions = np.ascontiguousarray(positions, dtype=np.uint64)
        n = len(positions)
        out = np.zeros(max(n, 1), dtype=np.uint64)
        km = None
        if key_marks is not None:
            key_marks = np.ascontiguousarray(key_marks, dtype=np.uint64)
            km = key_marks.ctypes.data_as(C.c_void_p)
        if self.use_ref:
            L = ref_lib()
            L.ref_search(self.k, _p(self.c_map), _ptr_array(self.acgt_pad),
                         _ptr_array(self.l0), _ptr_array(self.l12),
                         _p(self.pre_left), _p(self.pre_right), _p(positions),
                         _p(bit_seqs), km, n, _p(out),
                         threads or L.ref_max_threads())
        else:
            lib().oracle_search(self.k, _ptr_array(self.acgt_pad),
                                _ptr_array(self.l0), _ptr_array(self.l12),
                                _p(self.c_map), self.p, _p(self.pre_left),
                                _p(self.pre_right), _p(bit_seqs), _p(positions), n,
                                km, _p(out))
        return out[:n]

    def walk_sectors(self, bit_seqs, positions) -> int:
        bit_seqs = np.concatenate([np.ascontiguousarray(bit_seqs, np.uint64),
                                   np.zeros(2, np.uint64)])
        positions = np.ascontiguousarray(positions, dtype=np.uint64)
        return lib().oracle_walk_sectors(
            self.k, _ptr_array(self.acgt_pad), _ptr_array(self.l0),
            _ptr_array(self.l12), _p(self.c_map), self.p, _p(self.pre_left),
            _p(self.pre_right), _p(bit_seqs), _p(positions), len(positions))


def seq_to_bits(chars: bytes):
    n = len(chars)
    bits = np.zeros((n + 31) // 32 + 1, dtype=np.uint64)
    invalid = np.zeros(max(n, 1), dtype=np.uint8)
    lib().oracle_seq_to_bits(chars, n, _p(bits), invalid.ctypes.data_as(C.c_void_p))
    return bits, invalid[:n]


def positions_of(read_ends: np.ndarray, k: int) -> np.ndarray:
    read_ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
    n = lib().oracle_positions(_p(read_ends), len(read_ends), k, None)
    pos = np.zeros(max(n, 1), dtype=np.uint64)
    lib().oracle_positions(_p(read_ends), len(read_ends), k,
                           pos.ctypes.data_as(C.c_void_p))
    return pos[:n]


def index_search_reads(index: OracleIndex, reads: list[bytes],
                       key_marks=None) -> list[np.ndarray]:
    """The index step over whole reads: per read, one u64 per k-mer with
    UINT64_MAX-1 (-2) for k-mers holding an invalid char, UINT64_MAX (-1) for
    k-mers not found, else the SBWT index."""
    chars = b"".join(reads)
    read_ends = np.cumsum([len(r) for r in reads], dtype=np.uint64)
    bits, invalid = seq_to_bits(chars)
    pos = positions_of(read_ends, index.k)
    res = index.search_positions(bits, pos, key_marks)
    if len(pos):
        lib().oracle_mask_invalid(invalid.ctypes.data_as(C.c_void_p), _p(pos),
                                  len(pos), index.k, _p(res))
    out = []
    start = 0
    t = 0
    for r in reads:
        m = max(0, len(r) - index.k + 1)
        out.append(res[t:t + m])
        t += m
    return out


def as_signed_tokens(row: np.ndarray) -> list[int]:
    return [int(v) if v < INVALID else (-1 if v == NOT_FOUND else -2) for v in row]


# --------------------------------------------------------------------------
# Colors step
# --------------------------------------------------------------------------
class ColorsFile:
    """Themisto "sdsl-hybrid-v4" .tcolors file, member order as read by the
    reference (src/ColorIndexBuilder/ColorIndexBuilder.cpp:23-86): dense
    arrays (bit_vector), dense intervals, sparse arrays, sparse intervals
    (int_vector<>), is_dense marks + rank blob, key k-mer marks + rank blob,
    color set indexes (int_vector<>), then three u64 (the second + 1 is the
    number of colors).  sdsl layouts: bit_vector = u64 bits + words;
    int_vector<> = u64 bits + u8 width + words."""

    def __init__(self, data: bytes):
        off = 0

        def u64():
            nonlocal off
            v = struct.unpack_from("<Q", data, off)[0]
            off += 8
            return v

        n = u64()
        if data[off:off + n] != b"sdsl-hybrid-v4":
            raise ValueError("The colors file has an incorrect format. "
                             "Expected 'sdsl-hybrid-v4'")
        off += n

        def words(nbits):
            nonlocal off
            nw = (nbits + 63) // 64
            a = np.frombuffer(data, dtype=np.uint64, count=nw, offset=off).copy()
            off += nw * 8
            return a

        def bitvector():
            nb = u64()
            return nb, words(nb)

        def intvector():
            nonlocal off
            nb = u64()
            w = data[off]
            off += 1
            return nb, w, words(nb)

        _, self.dense_arrays = bitvector()
        nb, self.dense_intervals_width, self.dense_intervals = intvector()
        self.n_dense_intervals = nb // max(1, self.dense_intervals_width)
        nb, self.sparse_arrays_width, self.sparse_arrays = intvector()
        self.n_sparse = nb // max(1, self.sparse_arrays_width)
        nb, self.sparse_intervals_width, self.sparse_intervals = intvector()
        self.is_dense_bits, self.is_dense_marks = bitvector()
        bitvector()  # rank blob
        self.key_kmer_bits, self.key_kmer_marks = bitvector()
        bitvector()  # rank blob
        nb, self.color_set_idxs_width, self.color_set_idxs = intvector()
        self.n_keys = nb // max(1, self.color_set_idxs_width)
        self.max_color_set_idx, largest, self.sum_sizes = u64(), u64(), u64()
        self.num_colors = largest + 1

    @classmethod
    def read(cls, path) -> "ColorsFile":
        with open(path, "rb") as f:
            return cls(f.read())

class _ColorsStruct(C.Structure):
    _fields_ = [
        ("dense_arrays", U64P), ("dense_intervals", U64P),
        ("dense_intervals_width", C.c_uint32), ("sparse_arrays", U64P),
        ("sparse_arrays_width", C.c_uint32), ("sparse_intervals", U64P),
        ("sparse_intervals_width", C.c_uint32), ("is_dense", U64P),
        ("is_dense_l0", U64P), ("is_dense_l12", U64P), ("key_marks", U64P),
        ("key_l0", U64P), ("key_l12", U64P), ("color_set_idxs", U64P),
        ("color_set_idxs_width", C.c_uint32), ("num_colors", C.c_uint64),
    ]


def _pad(a: np.ndarray) -> np.ndarray:
    return np.concatenate([np.ascontiguousarray(a, np.uint64), np.zeros(2, np.uint64)])


class OracleColors:
    """A parsed .tcolors index (see ColorsFile) prepared for the restatement."""

    def __init__(self, tc):
        self.tc = tc
        self.keep = []

        def poppy(bits, nbits):
            n0, n12 = C.c_uint64(), C.c_uint64()
            lib().oracle_poppy_sizes(nbits, C.byref(n0), C.byref(n12))
            b = np.zeros(((nbits + 255) // 256) * 4 + 4, np.uint64)
            b[:len(bits)] = bits
            l0 = np.zeros(n0.value, np.uint64)
            l12 = np.zeros(n12.value, np.uint64)
            lib().oracle_poppy_build(_p(b), nbits, _p(l0), _p(l12))
            self.keep += [b, l0, l12]
            return b, l0, l12

        isd, isd0, isd12 = poppy(tc.is_dense_marks, tc.is_dense_bits)
        km, km0, km12 = poppy(tc.key_kmer_marks, tc.key_kmer_bits)
        arrs = [_pad(tc.dense_arrays), _pad(tc.dense_intervals),
                _pad(tc.sparse_arrays), _pad(tc.sparse_intervals),
                _pad(tc.color_set_idxs)]
        self.keep += arrs
        self.s = _ColorsStruct(
            _p(arrs[0]), _p(arrs[1]), tc.dense_intervals_width, _p(arrs[2]),
            tc.sparse_arrays_width, _p(arrs[3]), tc.sparse_intervals_width,
            _p(isd), _p(isd0), _p(isd12), _p(km), _p(km0), _p(km12), _p(arrs[4]),
            tc.color_set_idxs_width, tc.num_colors)

    def pseudoalign_mt(self, flat_idx, idx_offsets, not_found, invalid, tau=0.7,
                       include_not_found=False, include_invalid=False, threads=None):
        """The same per read, on `threads` host threads: (number of ids,
        ids checksum) per read."""
        idx = np.concatenate([np.ascontiguousarray(flat_idx, np.uint64),
                              np.zeros(1, np.uint64)])
        offs = np.ascontiguousarray(idx_offsets, np.uint64)
        n_reads = len(offs) - 1
        nf = np.ascontiguousarray(not_found, np.uint64)
        inv = np.ascontiguousarray(invalid, np.uint64)
        n_ids = np.zeros(max(1, n_reads), np.uint64)
        ck = np.zeros(max(1, n_reads), np.uint64)
        lib().oracle_pseudoalign_mt(C.byref(self.s), _p(idx), _p(offs), _p(nf), _p(inv),
                                    n_reads, tau, int(include_not_found),
                                    int(include_invalid), _p(n_ids), _p(ck),
                                    threads or os.cpu_count())
        return n_ids[:n_reads], ck[:n_reads]

    def pseudoalign(self, found_lists, not_found, invalid, tau=0.7,
                    include_not_found=False, include_invalid=False,
                    want_counts=False):
        n_reads = len(found_lists)
        offs = np.zeros(n_reads + 1, np.uint64)
        offs[1:] = np.cumsum([len(x) for x in found_lists])
        idx = np.concatenate([np.asarray(x, np.uint64) for x in found_lists] +
                             [np.zeros(1, np.uint64)])
        nf = np.ascontiguousarray(not_found, np.uint64)
        inv = np.ascontiguousarray(invalid, np.uint64)
        if len(nf) == 0:
            nf = np.zeros(1, np.uint64)
            inv = np.zeros(1, np.uint64)
        ids_off = np.zeros(n_reads + 1, np.uint64)
        counts = None
        cptr = None
        if want_counts:
            counts = np.zeros(max(1, n_reads * self.tc.num_colors), np.uint64)
            cptr = counts.ctypes.data_as(C.c_void_p)
        n_ids = lib().oracle_pseudoalign(C.byref(self.s), _p(idx), _p(offs), _p(nf),
                                         _p(inv), n_reads, tau, int(include_not_found),
                                         int(include_invalid), None, _p(ids_off), None)
        ids = np.zeros(max(1, n_ids), np.uint32)
        lib().oracle_pseudoalign(C.byref(self.s), _p(idx), _p(offs), _p(nf), _p(inv),
                                 n_reads, tau, int(include_not_found),
                                 int(include_invalid), ids.ctypes.data_as(C.c_void_p),
                                 _p(ids_off), cptr)
        rows = [ids[int(ids_off[r]):int(ids_off[r + 1])].tolist() for r in range(n_reads)]
        if want_counts:
            return rows, counts[:n_reads * self.tc.num_colors].reshape(
                n_reads, self.tc.num_colors)
        return rows


class RefColors:
    """A parsed .tcolors index (see ColorsFile) prepared for the reference's
    own colors kernels built for the host (oracle/ref_colors.cpp): Poppy
    layers from the reference's PoppyBuilder, arrays padded as the
    reference's GpuColorIndexContainer pads them (one extra word)."""

    def __init__(self, tc):
        L = ref_lib()
        if L is None:
            raise RuntimeError("reference CPU build missing: run `make -C oracle ref`")
        self.tc = tc
        self.keep = []

        def poppy(bits, nbits):
            n0, n12 = C.c_uint64(), C.c_uint64()
            L.ref_poppy_sizes(nbits, C.byref(n0), C.byref(n12))
            b = np.zeros(((nbits + 255) // 256) * 4 + 4, np.uint64)
            b[:len(bits)] = bits
            l0 = np.zeros(n0.value, np.uint64)
            l12 = np.zeros(n12.value, np.uint64)
            L.ref_poppy_build(_p(b), nbits, _p(l0), _p(l12))
            self.keep += [b, l0, l12]
            return b, l0, l12

        self.is_dense = poppy(tc.is_dense_marks, tc.is_dense_bits)
        self.key = poppy(tc.key_kmer_marks, tc.key_kmer_bits)
        self.dense_arrays, self.dense_intervals, self.sparse_arrays, \
            self.sparse_intervals, self.color_set_idxs = (
                _pad(tc.dense_arrays), _pad(tc.dense_intervals), _pad(tc.sparse_arrays),
                _pad(tc.sparse_intervals), _pad(tc.color_set_idxs))

    def color_counts(self, warped: np.ndarray, warp_intervals: np.ndarray,
                     threads: int | None = None) -> np.ndarray:
        """Counts of the reference's d_color_search + d_post_process over one
        batch: warped indexes (found indexes only, each read's count a
        multiple of 32) and the warps before each read (n_reads + 1 entries).
        Returns a (n_reads, num_colors) u64 array."""
        L = ref_lib()
        tc = self.tc
        warped = np.ascontiguousarray(warped, np.uint64)
        wi = np.ascontiguousarray(warp_intervals, np.uint64)
        n_reads = len(wi) - 1
        counts = np.zeros(max(1, n_reads * tc.num_colors), np.uint64)
        if len(warped) == 0:
            return counts[:0].reshape(0, tc.num_colors)
        rc = L.ref_color_counts(
            _p(warped), len(warped), _p(self.key[0]), _p(self.key[1]), _p(self.key[2]),
            _p(self.color_set_idxs), tc.color_set_idxs_width, _p(self.is_dense[0]),
            _p(self.is_dense[1]), _p(self.is_dense[2]), _p(self.dense_arrays),
            _p(self.dense_intervals), tc.dense_intervals_width, _p(self.sparse_arrays),
            tc.sparse_arrays_width, _p(self.sparse_intervals), tc.sparse_intervals_width,
            tc.num_colors, _p(wi), n_reads, _p(counts), threads or L.ref_max_threads())
        if rc != 0:
            raise ValueError("reference color kernel: a warp held padding lanes")
        return counts[:n_reads * tc.num_colors].reshape(n_reads, tc.num_colors)


def padding_free_batch(found_lists, batch_multiple: int = 1024):
    """Trims per-read found-index lists so that the reference's colors kernel
    sees no padding lane: every kept read keeps a positive multiple of 32 of
    its found indexes (reads with fewer than 32 are dropped), and the batch
    total is a multiple of batch_multiple (the reference pads its batch to
    1024 with -1, ColorSearcher.cpp:68-78).  Returns (kept read numbers,
    trimmed lists, warped indexes, warp intervals)."""
    lists = [np.asarray(x, np.uint64)[: (len(x) // 32) * 32] for x in found_lists]
    keep = [i for i, x in enumerate(lists) if len(x) >= 32]
    lists = [lists[i] for i in keep]
    total = sum(len(x) for x in lists)
    excess = total % batch_multiple
    j = len(lists) - 1
    while excess and j >= 0:  # take whole warps off the longest-tail reads
        can = min(excess, len(lists[j]) - 32)
        if can > 0:
            lists[j] = lists[j][:len(lists[j]) - can]
            excess -= can
        j -= 1
    while excess and lists:  # drop whole reads from the end
        excess = (excess - len(lists[-1])) % batch_multiple
        lists.pop()
        keep.pop()
    warped = np.concatenate(lists) if lists else np.zeros(0, np.uint64)
    wi = np.zeros(len(lists) + 1, np.uint64)
    wi[1:] = np.cumsum([len(x) // 32 for x in lists])
    return keep, lists, warped, wi


def ids_checksum(rows) -> np.ndarray:
    """Per read, the checksum oracle_pseudoalign_mt reports: sum over the
    read's ascending ids c of (c + 1) * (position in the list, from 1)."""
    return np.array([sum((c + 1) * (i + 1) for i, c in enumerate(r)) for r in rows],
                    dtype=np.uint64)


def threshold_minimum(seq_size: int, tau: float) -> int:
    """(u64)ceil((double)seq_size * tau), as the reference printer computes it."""
    return int(math.ceil(float(seq_size) * tau))
