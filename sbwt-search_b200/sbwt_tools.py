"""ctypes wrapper of the project's index-construction and synthetic-data tools
(csrc/tools/sbwt_build.cpp, built into _build/libsbwt_tools.so).

SBWT-Search itself does not build indexes (Themisto does); these tools write
the reference's .sbwt and .tcolors formats so that tests and benchmarks can
make seeded inputs of any size.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
TOOLS_SO = HERE / "_build" / "libsbwt_tools.so"
_L = None


def _lib():
    global _L
    if _L is None:
        if not TOOLS_SO.exists():
            raise RuntimeError(f"{TOOLS_SO} missing: run __graft_entry__.build()")
        L = C.CDLL(str(TOOLS_SO))
        u64 = C.c_uint64
        L.sbwt_tools_last_error.restype = C.c_char_p
        L.sbwt_tools_build_sbwt.argtypes = [C.c_void_p, C.c_void_p, u64, C.c_int,
                                            C.c_int, C.c_char_p]
        L.sbwt_tools_build_sbwt.restype = u64
        L.sbwt_tools_build_colored.argtypes = [C.c_void_p, C.c_void_p, u64, C.c_int,
                                               C.c_int, C.c_char_p, C.c_char_p]
        L.sbwt_tools_build_colored.restype = u64
        L.sbwt_tools_gen_genomes.argtypes = [u64, u64, u64, u64, C.c_double,
                                             C.c_double, C.c_double, C.c_void_p, u64,
                                             C.c_void_p]
        L.sbwt_tools_gen_genomes.restype = u64
        L.sbwt_tools_gen_reads.argtypes = [u64, C.c_void_p, C.c_void_p, u64, u64,
                                           C.c_double, u64, C.c_double, u64, u64,
                                           C.c_double, C.c_double, C.c_void_p, u64,
                                           C.c_void_p]
        L.sbwt_tools_gen_reads.restype = u64
        _L = L
    return _L


class Genomes:
    """Genomes stored back to back: chars (np.uint8) + lens (np.uint64)."""

    def __init__(self, chars: np.ndarray, lens: np.ndarray):
        self.chars = chars
        self.lens = lens
        self.starts = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)

    def __len__(self):
        return len(self.lens)

    def seq(self, i: int) -> bytes:
        return self.chars[int(self.starts[i]):int(self.starts[i + 1])].tobytes()

    def _ptrs(self):
        base = self.chars.ctypes.data
        arr = (C.c_void_p * len(self.lens))(*[base + int(s) for s in self.starts[:-1]])
        return arr


def gen_genomes(seed: int, n_genomes: int, length: int, n_founders: int = 0,
                sub_lo: float = 0.0, sub_hi: float = 0.0,
                indel: float = 0.0) -> Genomes:
    cap = n_genomes * (length + length // 8 + 64)
    chars = np.zeros(cap, dtype=np.uint8)
    lens = np.zeros(n_genomes, dtype=np.uint64)
    total = _lib().sbwt_tools_gen_genomes(seed, n_genomes, length, n_founders, sub_lo,
                                          sub_hi, indel, chars.ctypes.data, cap,
                                          lens.ctypes.data)
    return Genomes(chars[:total].copy(), lens)


def gen_reads(seed: int, genomes: Genomes | None, n_reads: int,
              frac_from_genome: float, len_median: int, len_sigma: float = 0.0,
              len_min: int = 1, len_max: int = 1 << 20, sub: float = 0.0,
              n_rate: float = 0.0):
    """Returns (chars np.uint8, read_ends np.uint64)."""
    if len_sigma == 0:
        cap = n_reads * len_median
    else:
        cap = n_reads * len_max
        cap = min(cap, int(n_reads * len_median * 8) + len_max)
    chars = np.zeros(max(cap, 1), dtype=np.uint8)
    ends = np.zeros(max(n_reads, 1), dtype=np.uint64)
    if genomes is None:
        gptr, lptr, ng = None, None, 0
    else:
        gptr, lptr, ng = genomes.chars.ctypes.data, genomes.lens.ctypes.data, len(genomes)
    total = _lib().sbwt_tools_gen_reads(seed, gptr, lptr, ng, n_reads,
                                        frac_from_genome, len_median, len_sigma,
                                        len_min, len_max, sub, n_rate,
                                        chars.ctypes.data, cap, ends.ctypes.data)
    if total == 0 and n_reads > 0 and cap > 0:
        raise RuntimeError("read buffer too small")
    return chars[:total], ends[:n_reads]


def build_sbwt(genomes: Genomes, k: int, path: str, add_rc: bool = True) -> int:
    n = _lib().sbwt_tools_build_sbwt(genomes._ptrs(), genomes.lens.ctypes.data,
                                     len(genomes), k, int(add_rc), str(path).encode())
    if n == 0:
        raise RuntimeError(_lib().sbwt_tools_last_error().decode())
    return n


def build_colored(genomes: Genomes, k: int, sbwt_path: str, tcolors_path: str,
                  add_rc: bool = True) -> int:
    n = _lib().sbwt_tools_build_colored(genomes._ptrs(), genomes.lens.ctypes.data,
                                        len(genomes), k, int(add_rc),
                                        str(sbwt_path).encode(),
                                        str(tcolors_path).encode())
    if n == 0:
        raise RuntimeError(_lib().sbwt_tools_last_error().decode())
    return n


def split_reads(chars: np.ndarray, ends: np.ndarray) -> list[bytes]:
    out = []
    s = 0
    b = chars.tobytes()
    for e in ends.tolist():
        out.append(b[s:e])
        s = e
    return out
