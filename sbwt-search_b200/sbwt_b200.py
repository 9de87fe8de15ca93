"""Python host binding of the C ABI in include/sbwt_b200.h (ctypes).

Mirrors the reference's in-process seams so that tests read like the
reference's own:

  * SbwtIndex.search(bit_seqs, positions)  ~ IndexSearcher::search
    (src/IndexSearcher/IndexSearcher.h:41-46);
  * SbwtIndex.search_reads(chars, read_ends) ~ the index step over a batch
    (SeqToBits + PositionsBuilder + search + -1/-2 mapping);
  * ColorIndex.counts / ColorIndex.pseudoalign ~ ColorSearcher::search
    (src/ColorSearcher/ColorSearcher.h:43-48) + the printer's threshold.

Device arrays are torch tensors (only for memory and streams); host arrays
are numpy.  Every call raises SbwtError carrying the library's status code
and message.  There is no CPU fallback: a missing library raises at import
of the handle classes.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libsbwt_b200.so"

OK, E_IO, E_FORMAT, E_OOM, E_CUDA, E_TIMEOUT, E_INVALID, E_CAPACITY = range(8)
DEVICE_POINTERS = 0x1
MOVE_TO_KEY_KMER = 0x2
PER_KMER_WALK = 0x4
INCLUDE_NOT_FOUND = 0x8
INCLUDE_INVALID = 0x10
NOT_FOUND = (1 << 64) - 1
INVALID = (1 << 64) - 2


class SbwtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class IndexInfo(C.Structure):
    _fields_ = [("num_bits", C.c_uint64), ("k", C.c_uint32),
                ("presearch_letters", C.c_uint32), ("c_map", C.c_uint64 * 5),
                ("device_bytes", C.c_uint64), ("device", C.c_int),
                ("has_key_kmer_marks", C.c_int), ("kmer_table_bytes", C.c_uint64),
                ("kmer_filter_bytes", C.c_uint64), ("host_result_bytes", C.c_uint32),
                ("reserved", C.c_uint32)]


_L = None


def lib():
    """Loads _build/libsbwt_b200.so (raises if it was not built)."""
    global _L
    if _L is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: build with sbwt-search_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        vp, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
        L.sbwt_last_error.restype = C.c_char_p
        L.sbwt_version.restype = C.c_char_p
        L.sbwt_index_open.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_uint,
                                      C.POINTER(vp)]
        L.sbwt_index_from_arrays.argtypes = [vp, u64, u32, vp, vp, C.c_int, C.c_uint,
                                             C.POINTER(vp)]
        L.sbwt_index_free.argtypes = [vp]
        L.sbwt_index_free.restype = None
        L.sbwt_index_get_info.argtypes = [vp, C.POINTER(IndexInfo)]
        L.sbwt_index_set_kmer_table.argtypes = [vp, C.c_int, C.POINTER(u64)]
        L.sbwt_search_positions.argtypes = [vp, vp, u64, vp, u64, vp, u32, vp]
        L.sbwt_count_kmers.argtypes = [vp, u64, u32]
        L.sbwt_count_kmers.restype = u64
        L.sbwt_search_reads.argtypes = [vp, vp, u64, vp, u64, vp, u64,
                                        C.POINTER(u64), u32, vp]
        L.sbwt_set_launch_config.argtypes = [u32, u32, u64, u64]
        L.sbwt_set_probe_length.argtypes = [u32]
        L.sbwt_set_l2_window.argtypes = [C.c_int]
        if hasattr(L, "sbwt_colors_open"):
            L.sbwt_colors_open.argtypes = [C.c_char_p, C.c_int, C.POINTER(vp)]
            L.sbwt_colors_free.argtypes = [vp]
            L.sbwt_colors_free.restype = None
            L.sbwt_colors_num_colors.argtypes = [vp]
            L.sbwt_colors_num_colors.restype = u64
            L.sbwt_color_counts.argtypes = [vp, vp, vp, u64, vp, u32, vp]
            L.sbwt_pseudoalign.argtypes = [vp, vp, vp, vp, vp, u64, C.c_double, u32,
                                           vp, u64, vp, vp]
            L.sbwt_colors_set_node_table.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.sbwt_pipeline_create.argtypes = [vp, vp, u64, u64, u32, C.c_double,
                                           C.POINTER(vp)]
        L.sbwt_pipeline_free.argtypes = [vp]
        L.sbwt_pipeline_free.restype = None
        L.sbwt_pipeline_run.argtypes = [vp, vp, u64, vp, u64, vp, u64, C.POINTER(u64),
                                        vp, u64, vp]
        L.sbwt_server_create.argtypes = [vp, vp, u64, u64, C.c_int, u32, C.c_double,
                                         C.POINTER(vp)]
        L.sbwt_server_free.argtypes = [vp]
        L.sbwt_server_free.restype = None
        L.sbwt_server_submit.argtypes = [vp, vp, u64, vp, u64, C.POINTER(u64)]
        L.sbwt_server_wait.argtypes = [vp, u64, C.c_double, C.POINTER(vp), C.POINTER(u64),
                                       C.POINTER(vp), C.POINTER(u64), C.POINTER(vp),
                                       C.POINTER(u64)]
        L.sbwt_get_launch_config.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_int), vp]
        L.sbwt_set_block_threads.argtypes = [u32]
        L.sbwt_server_slots.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(u64), C.POINTER(u64)]
        L.sbwt_server_stats.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(u64), C.POINTER(u64), C.POINTER(u64),
                                        C.POINTER(C.c_double), C.c_int]
        L.sbwt_free.argtypes = [vp]
        L.sbwt_fastx_parse.argtypes = [vp, u64, vp, u64, vp, u64, C.POINTER(u64),
                                       C.POINTER(u64), u32, C.c_int, vp]
        L.sbwt_build_index.argtypes = [vp, u64, vp, u64, u32, C.c_int, C.c_char_p, C.c_int,
                                       C.POINTER(u64)]
        L.sbwt_build_colored_index.argtypes = [vp, u64, vp, u64, u32, C.c_int, C.c_char_p,
                                               C.c_char_p, C.c_int, C.POINTER(u64)]
        L.sbwt_format_index_results.argtypes = [vp, vp, u64, u32, C.c_int, vp, u64,
                                                C.POINTER(u64), u32, C.c_int, vp]
        L.sbwt_format_color_results.argtypes = [vp, vp, u64, u64, C.c_int, vp, u64,
                                                C.POINTER(u64), u32, C.c_int, vp]
        L.sbwt_free.restype = None
        L.sbwt_autotune.argtypes = [vp, vp, u64, vp, u64, u64, C.POINTER(u32),
                                    C.POINTER(u32), C.POINTER(u64), C.POINTER(C.c_double)]
        _L = L
    return _L


def check(rc: int) -> None:
    if rc != OK:
        raise SbwtError(rc, lib().sbwt_last_error().decode(errors="replace"))


def _ptr(a) -> int | None:
    """Address of a numpy array or a torch tensor (None for empty/None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _is_dev(a) -> bool:
    return not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


def set_launch_config(presearch_letters: int = 0, blocks_per_sm: int = 0,
                      tile: int = 0, chunk_chars: int = 0) -> None:
    check(lib().sbwt_set_launch_config(presearch_letters, blocks_per_sm, tile,
                                       chunk_chars))


def set_probe_length(probe_len: int = 0) -> None:
    """0 = automatic, 0xFFFFFFFF = off (results never depend on it)."""
    check(lib().sbwt_set_probe_length(probe_len))


TABLE_KERNEL_DEFAULT = -1


def set_block_threads(threads: int = 256) -> None:
    """Threads per block of the read search kernels (128 or 256)."""
    check(lib().sbwt_set_block_threads(int(threads)))


def set_table_kernel(mode: int = TABLE_KERNEL_DEFAULT) -> None:
    """Read search kernel of an index with a k-mer table: 0 general, 1 table
    (True), 2..5 walks kernel with (walks per lane, blocks per SM) = (1, 5),
    (2, 4), (2, 3), (4, 2), 6 k-mers kernel, 7 automatic (11 for small
    tables, else 17), 8/9 walks kernel without filter and staging (1/2
    walks), 10 the same with 1 walk and a one-k-mer filter, 11/12 k-mers
    kernel with 2/8 k-mers per lane, 13/14 = 8/10 with staged stores,
    15 k-mers kernel over consecutive slots, 16/17 = 13 staging 8/16 slots,
    18 = 14 staging 16 slots, 19 k-mers kernel without the filter, -1 the
    library default (sbwt_set_table_kernel).  Results never depend on it."""
    check(lib().sbwt_set_table_kernel(int(mode)))


def set_l2_window(enabled: bool = True) -> None:
    check(lib().sbwt_set_l2_window(int(enabled)))


class SbwtIndex:
    """A resident SBWT on one GPU (rank blocks + presearch pyramid)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        info = IndexInfo()
        check(lib().sbwt_index_get_info(self._h, C.byref(info)))
        self.k = info.k
        self.num_bits = info.num_bits
        self.presearch_letters = info.presearch_letters
        self.c_map = list(info.c_map)
        self.device_bytes = info.device_bytes
        self.device = info.device
        self.has_key_kmer_marks = bool(info.has_key_kmer_marks)

    @classmethod
    def open(cls, sbwt_path, colors_path=None, device: int = 0,
             presearch_letters: int = 0) -> "SbwtIndex":
        h = C.c_void_p()
        check(lib().sbwt_index_open(str(sbwt_path).encode(),
                                    None if colors_path is None else str(colors_path).encode(),
                                    device, presearch_letters, C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, acgt, num_bits: int, k: int, suffix_group_starts=None,
                    key_kmer_marks=None, device: int = 0,
                    presearch_letters: int = 0) -> "SbwtIndex":
        arrs = [np.ascontiguousarray(a, dtype=np.uint64) for a in acgt]
        ptrs = (C.c_void_p * 4)(*[a.ctypes.data for a in arrs])
        sg = None if suffix_group_starts is None else np.ascontiguousarray(
            suffix_group_starts, dtype=np.uint64)
        km = None if key_kmer_marks is None else np.ascontiguousarray(
            key_kmer_marks, dtype=np.uint64)
        h = C.c_void_p()
        check(lib().sbwt_index_from_arrays(ptrs, num_bits, k, _ptr(sg), _ptr(km), device,
                                           presearch_letters, C.byref(h)))
        return cls(h.value)

    def close(self) -> None:
        if self._h:
            lib().sbwt_index_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- IndexSearcher::search seam ------------------------------------------
    def search(self, bit_seqs, positions, out=None, move_to_key_kmer: bool = False,
               stream: int = 0):
        """bit_seqs: u64 2-bit MSB-first packed chars; positions: u64 k-mer
        starts.  Host numpy in -> numpy out (synchronous); CUDA tensors in ->
        results written into `out` (a CUDA int64/uint64 tensor)."""
        flags = MOVE_TO_KEY_KMER if move_to_key_kmer else 0
        if _is_dev(positions):
            flags |= DEVICE_POINTERS
            assert out is not None
            check(lib().sbwt_search_positions(self._h, _ptr(bit_seqs), bit_seqs.numel(),
                                              _ptr(positions), positions.numel(),
                                              _ptr(out), flags, stream or None))
            return out
        bit_seqs = np.ascontiguousarray(bit_seqs, dtype=np.uint64)
        positions = np.ascontiguousarray(positions, dtype=np.uint64)
        res = np.empty(max(len(positions), 1), dtype=np.uint64)
        check(lib().sbwt_search_positions(self._h, _ptr(bit_seqs), len(bit_seqs),
                                          _ptr(positions), len(positions), _ptr(res),
                                          flags, None))
        return res[:len(positions)]

    # -- fused read path ------------------------------------------------------
    def count_kmers(self, read_ends: np.ndarray) -> int:
        read_ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
        return int(lib().sbwt_count_kmers(_ptr(read_ends), len(read_ends), self.k))

    def set_kmer_table(self, enable: bool) -> int:
        """Builds (kept when present) or drops the k-mer -> node table (same
        results either way); returns its size in bytes, 0 when absent."""
        nb = C.c_uint64(0)
        check(lib().sbwt_index_set_kmer_table(self._h, int(enable), C.byref(nb)))
        info = IndexInfo()
        check(lib().sbwt_index_get_info(self._h, C.byref(info)))
        self.device_bytes = info.device_bytes
        return nb.value

    def host_result_bytes(self) -> int:
        """Bytes per k-mer a host-pointer search_reads moves device -> host
        into a pageable results buffer (a pinned one always takes 8)."""
        info = IndexInfo()
        check(lib().sbwt_index_get_info(self._h, C.byref(info)))
        return int(info.host_result_bytes)

    def filter_bytes(self) -> int:
        """Size of the k-mer filter in front of the k-mer table (0 when absent)."""
        info = IndexInfo()
        check(lib().sbwt_index_get_info(self._h, C.byref(info)))
        return int(info.kmer_filter_bytes)

    def search_reads(self, chars, read_ends, out=None, move_to_key_kmer: bool = False,
                     per_kmer_walk: bool = False, stream: int = 0):
        """chars: reads back to back (bytes / uint8); read_ends: cumulative
        exclusive ends.  Host in -> numpy u64 per k-mer (NOT_FOUND / INVALID
        markers).  CUDA tensors in -> fills `out`, returns the k-mer count."""
        flags = (MOVE_TO_KEY_KMER if move_to_key_kmer else 0) | \
            (PER_KMER_WALK if per_kmer_walk else 0)
        n_res = C.c_uint64(0)
        if _is_dev(read_ends):
            flags |= DEVICE_POINTERS
            check(lib().sbwt_search_reads(self._h, _ptr(chars), chars.numel(),
                                          _ptr(read_ends), read_ends.numel(), _ptr(out),
                                          out.numel(), C.byref(n_res), flags,
                                          stream or None))
            return int(n_res.value)
        if isinstance(chars, (bytes, bytearray)):
            chars = np.frombuffer(chars, dtype=np.uint8)
        chars = np.ascontiguousarray(chars, dtype=np.uint8)
        read_ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
        if out is None:
            out = np.empty(max(self.count_kmers(read_ends), 1), dtype=np.uint64)
        check(lib().sbwt_search_reads(self._h, _ptr(chars) if len(chars) else None,
                                      len(chars), _ptr(read_ends), len(read_ends),
                                      _ptr(out), len(out), C.byref(n_res), flags, None))
        return out[:n_res.value]


class ColorIndex:
    """A resident .tcolors color index on one GPU."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)
        self.num_colors = int(lib().sbwt_colors_num_colors(self._h))

    @classmethod
    def open(cls, tcolors_path, device: int = 0) -> "ColorIndex":
        h = C.c_void_p()
        check(lib().sbwt_colors_open(str(tcolors_path).encode(), device, C.byref(h)))
        return cls(h.value)

    def close(self) -> None:
        if self._h:
            lib().sbwt_colors_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_node_table(self, enable: bool) -> bool:
        """Builds or drops the per-node color set table (same results either
        way); returns whether the table is in use."""
        built = C.c_int(0)
        check(lib().sbwt_colors_set_node_table(self._h, int(enable), C.byref(built)))
        return bool(built.value)

    def counts(self, sbwt_idxs: np.ndarray, idx_offsets: np.ndarray) -> np.ndarray:
        sbwt_idxs = np.ascontiguousarray(sbwt_idxs, dtype=np.uint64)
        idx_offsets = np.ascontiguousarray(idx_offsets, dtype=np.uint64)
        n = len(idx_offsets) - 1
        out = np.zeros((max(n, 1), self.num_colors), dtype=np.uint32)
        check(lib().sbwt_color_counts(self._h, _ptr(sbwt_idxs) if len(sbwt_idxs) else None,
                                      _ptr(idx_offsets), n, _ptr(out), 0, None))
        return out[:n]

    def pseudoalign(self, sbwt_idxs, idx_offsets, not_found=None, invalid=None,
                    tau: float = 0.7, include_not_found: bool = False,
                    include_invalid: bool = False):
        """Per read, the ascending color ids whose count passes tau."""
        sbwt_idxs = np.ascontiguousarray(sbwt_idxs, dtype=np.uint64)
        idx_offsets = np.ascontiguousarray(idx_offsets, dtype=np.uint64)
        n = len(idx_offsets) - 1
        nf = None if not_found is None else np.ascontiguousarray(not_found, np.uint64)
        inv = None if invalid is None else np.ascontiguousarray(invalid, np.uint64)
        flags = (INCLUDE_NOT_FOUND if include_not_found else 0) | \
            (INCLUDE_INVALID if include_invalid else 0)
        offs = np.zeros(n + 1, dtype=np.uint64)
        cap = max(1, len(sbwt_idxs))
        while True:
            ids = np.zeros(cap, dtype=np.uint32)
            rc = lib().sbwt_pseudoalign(self._h, _ptr(sbwt_idxs) if len(sbwt_idxs) else None,
                                        _ptr(idx_offsets), _ptr(nf), _ptr(inv), n, tau,
                                        flags, _ptr(ids), cap, _ptr(offs), None)
            if rc == E_CAPACITY:
                cap = int(offs[n]) + 1
                continue
            check(rc)
            break
        return [ids[int(offs[r]):int(offs[r + 1])].tolist() for r in range(n)], offs, ids


def _np_chars(chars):
    if isinstance(chars, (bytes, bytearray)):
        chars = np.frombuffer(chars, dtype=np.uint8)
    return np.ascontiguousarray(chars, dtype=np.uint8)


class Pipeline:
    """A reusable device pipeline (one CUDA graph per batch): index step, and
    the colors step too when a ColorIndex is given."""

    def __init__(self, index: SbwtIndex, colors: "ColorIndex | None", max_chars: int,
                 max_reads: int, tau: float = 0.7, include_not_found: bool = False,
                 include_invalid: bool = False, move_to_key_kmer: bool = False):
        flags = (INCLUDE_NOT_FOUND if include_not_found else 0) | \
            (INCLUDE_INVALID if include_invalid else 0) | \
            (MOVE_TO_KEY_KMER if move_to_key_kmer else 0)
        h = C.c_void_p()
        check(lib().sbwt_pipeline_create(index._h, colors._h if colors else None, max_chars,
                                         max_reads, flags, tau, C.byref(h)))
        self._h = h
        self.index, self.colors = index, colors

    def close(self):
        if self._h:
            lib().sbwt_pipeline_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, chars, read_ends, raw: bool = False):
        """Index mode: u64 per k-mer.  Colors mode: per-read id lists, or with
        raw=True the (ids, offsets) arrays without building Python lists."""
        chars = _np_chars(chars)
        read_ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
        n = len(read_ends)
        nres = C.c_uint64(0)
        if self.colors is None:
            out = np.empty(max(self.index.count_kmers(read_ends), 1), np.uint64)
            check(lib().sbwt_pipeline_run(self._h, _ptr(chars) if len(chars) else None,
                                          len(chars), _ptr(read_ends) if n else None, n,
                                          _ptr(out), len(out), C.byref(nres), None, 0, None))
            return out[:nres.value]
        offs = np.zeros(n + 1, np.uint64)
        cap = max(1, n * 8)
        while True:
            ids = np.zeros(cap, np.uint32)
            rc = lib().sbwt_pipeline_run(self._h, _ptr(chars) if len(chars) else None,
                                         len(chars), _ptr(read_ends) if n else None, n, None, 0,
                                         C.byref(nres), _ptr(ids), cap, _ptr(offs))
            if rc == E_CAPACITY:
                cap = int(offs[n]) + 1
                continue
            check(rc)
            if raw:
                return ids[:int(offs[n])], offs
            return [ids[int(offs[r]):int(offs[r + 1])].tolist() for r in range(n)]


class Server:
    """Continuous-batching serving loop over resident indexes."""

    def __init__(self, index: SbwtIndex, colors: "ColorIndex | None" = None,
                 batch_chars: int = 32 << 20, batch_reads: int = 1 << 18, slots: int = 3,
                 tau: float = 0.7, include_not_found: bool = False,
                 include_invalid: bool = False):
        flags = (INCLUDE_NOT_FOUND if include_not_found else 0) | \
            (INCLUDE_INVALID if include_invalid else 0)
        h = C.c_void_p()
        check(lib().sbwt_server_create(index._h, colors._h if colors else None, batch_chars,
                                       batch_reads, slots, flags, tau, C.byref(h)))
        self._h = h
        self.colors = colors

    def close(self):
        if self._h:
            lib().sbwt_server_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, chars, read_ends) -> int:
        chars = _np_chars(chars)
        read_ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
        rid = C.c_uint64(0)
        check(lib().sbwt_server_submit(self._h, _ptr(chars) if len(chars) else None,
                                       len(chars), _ptr(read_ends) if len(read_ends) else None,
                                       len(read_ends), C.byref(rid)))
        return rid.value

    def wait(self, rid: int, timeout_ms: float = -1.0, raw: bool = False):
        """Index mode: (values, offsets).  Colors mode: per-read id lists, or
        with raw=True the (ids, offsets) arrays."""
        vals, ids, offs = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nv, ni, nr = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().sbwt_server_wait(self._h, rid, timeout_ms, C.byref(vals), C.byref(nv),
                                     C.byref(ids), C.byref(ni), C.byref(offs), C.byref(nr)))
        L = lib()
        try:
            o = np.ctypeslib.as_array(C.cast(offs, C.POINTER(C.c_uint64)),
                                      (nr.value + 1,)).copy()
            if self.colors is None:
                v = np.ctypeslib.as_array(C.cast(vals, C.POINTER(C.c_uint64)),
                                          (max(nv.value, 1),))[:nv.value].copy()
                return v, o
            i = np.ctypeslib.as_array(C.cast(ids, C.POINTER(C.c_uint32)),
                                      (max(ni.value, 1),))[:ni.value].copy()
            if raw:
                return i, o
            return [i[int(o[r]):int(o[r + 1])].tolist() for r in range(nr.value)]
        finally:
            for p in (vals, ids, offs):
                L.sbwt_free(p)

    def stats(self, reset: bool = False) -> dict:
        p50, p99, el = C.c_double(), C.c_double(), C.c_double()
        nd, rd, nb = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().sbwt_server_stats(self._h, C.byref(p50), C.byref(p99), C.byref(nd),
                                      C.byref(rd), C.byref(nb), C.byref(el), int(reset)))
        return {"p50_s": p50.value, "p99_s": p99.value, "requests": nd.value,
                "reads": rd.value, "batches": nb.value, "elapsed_s": el.value}

    def slots(self) -> dict:
        """Slots open now, device bytes per slot, and how often a waiting
        batch found too little free device memory to open one."""
        n, b, d = C.c_int(), C.c_uint64(), C.c_uint64()
        check(lib().sbwt_server_slots(self._h, C.byref(n), C.byref(b), C.byref(d)))
        return {"open": n.value, "slot_bytes": b.value, "denied": d.value}


AUTOTUNE_CACHE = HERE / "_build" / "autotune.json"


def autotune(index: SbwtIndex, d_chars, d_read_ends, sample_chars: int = 256 << 20,
             use_cache: bool = True) -> dict:
    """Chooses the read search kernel (walks per lane) or presearch depth,
    tile size and blocks per SM for this GPU and index with the library's
    autotuner (sbwt_autotune) and applies them; the choice is cached per
    (GPU name, SBWT nodes, k, k-mer table present) in _build/autotune.json."""
    import json
    try:
        import torch
        gpu = torch.cuda.get_device_name(index.device)
    except Exception:
        gpu = "cuda"
    info = IndexInfo()
    check(lib().sbwt_index_get_info(index._h, C.byref(info)))
    key = f"{gpu}|{index.num_bits}|{index.k}|table={int(info.kmer_table_bytes > 0)}"
    cache = {}
    if use_cache and AUTOTUNE_CACHE.exists():
        try:
            cache = json.loads(AUTOTUNE_CACHE.read_text())
        except Exception:
            cache = {}
    if use_cache and key in cache:
        c = cache[key]
        set_launch_config(c["presearch"], c["blocks_per_sm"], c["tile"], 0)
        set_table_kernel(c.get("table_kernel", TABLE_KERNEL_DEFAULT))
        set_block_threads(c.get("block_threads", 256))
        return dict(c, cached=True)
    p, b = C.c_uint32(), C.c_uint32()
    t, ms = C.c_uint64(), C.c_double()
    check(lib().sbwt_autotune(index._h, _ptr(d_chars), d_chars.numel(), _ptr(d_read_ends),
                              d_read_ends.numel(), sample_chars, C.byref(p), C.byref(b),
                              C.byref(t), C.byref(ms)))
    mode, bt = C.c_int(), C.c_uint32()
    check(lib().sbwt_get_launch_config(None, None, None, None, C.byref(mode), C.byref(bt)))
    c = {"presearch": p.value, "blocks_per_sm": b.value, "tile": t.value,
         "table_kernel": mode.value, "block_threads": bt.value, "sample_ms": ms.value}
    if use_cache:
        cache[key] = c
        AUTOTUNE_CACHE.parent.mkdir(parents=True, exist_ok=True)
        AUTOTUNE_CACHE.write_text(json.dumps(cache, indent=1))
    return dict(c, cached=False)


def fastx_parse(text, device: int = 0):
    """FASTA/FASTQ text (bytes or np.uint8) parsed on the GPU: returns
    (chars np.uint8, read_ends np.uint64), the same as fastx_read on a file."""
    text = _np_chars(text)
    n = len(text)
    nc, nr = C.c_uint64(), C.c_uint64()
    chars = np.zeros(max(n, 1), dtype=np.uint8)
    rc = lib().sbwt_fastx_parse(_ptr(text) if n else None, n, _ptr(chars), n, None, 0,
                                C.byref(nc), C.byref(nr), 0, device, None)
    if rc == E_CAPACITY:
        ends = np.zeros(max(nr.value, 1), dtype=np.uint64)
        rc = lib().sbwt_fastx_parse(_ptr(text) if n else None, n, _ptr(chars), n, _ptr(ends),
                                    len(ends), C.byref(nc), C.byref(nr), 0, device, None)
    else:
        ends = np.zeros(1, dtype=np.uint64)
    check(rc)
    return chars[:nc.value], ends[:nr.value]


def _format(fn, *args, device=0):
    nb = C.c_uint64()
    rc = fn(*args, None, 0, C.byref(nb), 0, device, None)
    if rc == OK:
        return b""
    if rc != E_CAPACITY:
        check(rc)
    out = np.zeros(max(nb.value, 1), dtype=np.uint8)
    check(fn(*args, _ptr(out), len(out), C.byref(nb), 0, device, None))
    return out[:nb.value].tobytes()


def format_index_results(results, read_ends, k: int, fmt: int = 0, device: int = 0) -> bytes:
    """Index results of one batch formatted on the GPU (0 ascii, 1 binary,
    2 bool), byte for byte what the host writers emit after the header."""
    res = np.ascontiguousarray(results, dtype=np.uint64)
    ends = np.ascontiguousarray(read_ends, dtype=np.uint64)
    return _format(lib().sbwt_format_index_results, _ptr(res) if len(res) else None,
                   _ptr(ends) if len(ends) else None, len(ends), k, fmt, device=device)


def format_color_results(ids, ids_offsets, num_colors: int, fmt: int = 0,
                         device: int = 0) -> bytes:
    """Pseudoalignment ids formatted on the GPU (0 ascii, 1 binary, 2 csv)."""
    ids = np.ascontiguousarray(ids, dtype=np.uint32)
    offs = np.ascontiguousarray(ids_offsets, dtype=np.uint64)
    return _format(lib().sbwt_format_color_results, _ptr(ids) if len(ids) else None,
                   _ptr(offs), len(offs) - 1, num_colors, fmt, device=device)


def build_index(seqs, k: int, out_path, add_rc: bool = True, device: int = 0) -> int:
    """SBWT of every k-mer of `seqs` (a list of bytes, or (chars, ends)) built
    on the GPU and written to out_path; returns the node count."""
    if isinstance(seqs, tuple):
        chars, ends = _np_chars(seqs[0]), np.ascontiguousarray(seqs[1], dtype=np.uint64)
    else:
        chars = _np_chars(b"".join(seqs))
        ends = np.cumsum([len(x) for x in seqs]).astype(np.uint64)
    nn = C.c_uint64()
    check(lib().sbwt_build_index(_ptr(chars) if len(chars) else None, len(chars),
                                 _ptr(ends) if len(ends) else None, len(ends), k, int(add_rc),
                                 str(out_path).encode(), device, C.byref(nn)))
    return nn.value


def build_colored_index(chars, genome_ends, k: int, sbwt_path, tcolors_path,
                        add_rc: bool = True, device: int = 0) -> int:
    """SBWT + .tcolors of genomes (chars back to back, cumulative ends) built
    on the GPU; returns the node count."""
    chars = _np_chars(chars)
    ends = np.ascontiguousarray(genome_ends, dtype=np.uint64)
    nn = C.c_uint64()
    check(lib().sbwt_build_colored_index(_ptr(chars) if len(chars) else None, len(chars),
                                         _ptr(ends), len(ends), k, int(add_rc),
                                         str(sbwt_path).encode(), str(tcolors_path).encode(),
                                         device, C.byref(nn)))
    return nn.value
