"""Shared test inputs: seeded synthetic SBWTs and reads (built with the
project's own tools) and the golden fixtures of the reference."""
from __future__ import annotations

import gzip
import shutil
import tempfile
from functools import lru_cache
from pathlib import Path

import numpy as np

import oracle as O
import sbwt_tools as T

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
TMP = Path(tempfile.mkdtemp(prefix="sbwt_tests_"))
FIXTURE_FILES = ["fasta1.fna", "fasta2.fna", "fasta3.fna", "fasta4.fna", "fastq1.fnq"]


@lru_cache(None)
def golden_sbwt_path() -> str:
    out = TMP / "search_test_index.sbwt"
    with gzip.open(GOLDEN / "index_search" / "search_test_index.sbwt.gz", "rb") as f_in:
        with open(out, "wb") as f_out:
            shutil.copyfileobj(f_in, f_out)
    return str(out)


@lru_cache(None)
def synthetic(seed: int = 1, n_genomes: int = 1, length: int = 20000, k: int = 31,
              n_founders: int = 0, sub: float = 0.0):
    """(genomes, sbwt_path, SbwtFile) for a seeded synthetic reference."""
    g = T.gen_genomes(seed, n_genomes, length, n_founders, sub, sub, 0.0)
    path = TMP / f"syn_{seed}_{n_genomes}_{length}_{k}_{n_founders}_{sub}.sbwt"
    T.build_sbwt(g, k, str(path))
    return g, str(path), O.SbwtFile.read(path)


@lru_cache(None)
def oracle_index(path: str, p: int = 8):
    sb = O.SbwtFile.read(path)
    return O.OracleIndex(sb.acgt, sb.num_bits, sb.k, p)


def mixed_reads(genomes, seed: int, n: int, median: int = 100, sigma: float = 0.6,
                sub: float = 0.01, n_rate: float = 0.005, frac: float = 0.6,
                len_min: int = 0, len_max: int = 400):
    chars, ends = T.gen_reads(seed, genomes, n, frac, median, sigma, len_min, len_max,
                              sub, n_rate)
    return chars, ends


def oracle_results(index, chars: np.ndarray, ends: np.ndarray) -> np.ndarray:
    reads = T.split_reads(chars, ends)
    rows = O.index_search_reads(index, reads)
    return np.concatenate(rows) if rows else np.zeros(0, np.uint64)


def key_marks_for(index, d: int, seed: int = 0) -> np.ndarray:
    """Key k-mer marks for the d > 1 forward walk (IndexSearcher.cuh:60-70 of
    the reference): about one node in d is a key, every node without an
    outgoing edge bit is a key, and every cycle of first-edge successors holds
    a key, so the walk from any node ends."""
    import oracle as O
    N = index.num_bits
    rng = np.random.default_rng(seed)
    key = rng.random(N) < 1.0 / d
    succ = np.full(N, -1, np.int64)
    bits = [np.unpackbits(a.view(np.uint8), bitorder="little")[:N] for a in index.acgt]
    L = O.lib()
    for i in range(N):
        for c in range(4):
            if bits[c][i]:
                succ[i] = int(index.c_map[c]) + L.oracle_rank(
                    O._p(index.acgt_pad[c]), O._p(index.l0[c]), O._p(index.l12[c]), i)
                break
    key |= succ < 0
    state = np.zeros(N, np.int8)  # 0 new, 1 on stack, 2 resolved
    for s in range(N):
        path = []
        x = s
        while not key[x] and state[x] == 0:
            state[x] = 1
            path.append(x)
            x = int(succ[x])
        if not key[x] and state[x] == 1:  # a cycle without a key
            key[x] = True
        for y in path:
            state[y] = 2
    words = np.packbits(key.astype(np.uint8), bitorder="little")
    words = np.concatenate([words, np.zeros((-len(words)) % 8, np.uint8)])
    return words.view(np.uint64)


def random_fastx(seed: int, n_records: int, fastq_frac: float = 0.5, max_line: int = 80,
                 junk: bool = True, final_newline: bool = True) -> bytes:
    """Seeded FASTA/FASTQ text that exercises the record rules: CRLF and LF
    line ends, blank lines, empty records, multi-line sequences and qualities,
    quality lines starting with '@', '>' or '+', zero-length FASTQ sequences,
    leading junk lines and (optionally) no final newline."""
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"ACGTACGTACGTacgtN", dtype=np.uint8)
    qual = np.frombuffer(b"IIII#@>+!5", dtype=np.uint8)
    lines: list[bytes] = []
    if junk:
        for _ in range(int(rng.integers(0, 4))):
            lines.append(bytes(rng.choice(alphabet, int(rng.integers(0, 20)))))
        if rng.random() < 0.5:
            lines.append(b"+junk")
    for r in range(n_records):
        n = int(rng.integers(0, 400)) if rng.random() < 0.9 else 0
        seq = bytes(rng.choice(alphabet, n))
        width = int(rng.integers(1, max_line + 1)) if rng.random() < 0.6 else max(n, 1)
        seq_lines = [seq[i:i + width] for i in range(0, n, width)] or ([] if rng.random() < 0.5
                                                                       else [b""])
        if rng.random() < 0.1:
            seq_lines.insert(int(rng.integers(0, len(seq_lines) + 1)), b"")
        if rng.random() < fastq_frac:
            lines.append(b"@r%d" % r)
            lines += seq_lines
            lines.append(b"+" if rng.random() < 0.7 else b"+r%d" % r)
            q = bytes(rng.choice(qual, n))
            if n and rng.random() < 0.3:
                q = bytes([int(rng.choice(np.frombuffer(b"@>+", np.uint8)))]) + q[1:]
            qw = int(rng.integers(1, max_line + 1)) if rng.random() < 0.4 else max(n, 1)
            lines += [q[i:i + qw] for i in range(0, n, qw)]
        else:
            lines.append(b">r%d some description" % r)
            lines += seq_lines
    out = bytearray()
    for i, ln in enumerate(lines):
        out += ln
        out += b"\r\n" if rng.random() < 0.2 else b"\n"
    if not final_newline and out.endswith(b"\n"):
        out = out[:-2] if out.endswith(b"\r\n") else out[:-1]
    return bytes(out)


def host_fastx(text: bytes, path) -> tuple[bytes, np.ndarray]:
    """The host reader (sbwt_fastx_read) on `text` written to `path`."""
    import ctypes as C
    import sbwt_b200 as S
    Path(path).write_bytes(text)
    L = S.lib()
    L.sbwt_fastx_read.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.sbwt_free.argtypes = [C.c_void_p]
    ch, en = C.c_void_p(), C.c_void_p()
    nc, nr = C.c_uint64(), C.c_uint64()
    S.check(L.sbwt_fastx_read(str(path).encode(), C.byref(ch), C.byref(nc), C.byref(en),
                              C.byref(nr)))
    chars = C.string_at(ch, nc.value) if nc.value else b""
    ends = np.ctypeslib.as_array(C.cast(en, C.POINTER(C.c_uint64)),
                                 (max(nr.value, 1),))[:nr.value].copy()
    L.sbwt_free(ch)
    L.sbwt_free(en)
    return chars, ends


def small_sbwt(seqs: list[bytes], k: int, add_rc: bool = True):
    """A plain-matrix SBWT of the k-mers of seqs (any k), built by brute force
    from the definition, for indexes the project's builder does not make
    (k > 31).  Nodes are the k-mers plus, for every k-mer x without a
    predecessor, the dummies $^(k-i) x[0..i) (i < k); nodes are in colex
    order ($ < A < C < G < T, last char first); the first node of each suffix
    group (nodes sharing their last k-1 chars) carries bit c iff its last
    k-1 chars followed by c is a node.  Returns (acgt words, suffix-group-start
    words, number of nodes, number of k-mers)."""
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    kmers = set()
    for s in seqs:
        s = s.upper()
        strands = [s, s.translate(comp)[::-1]] if add_rc else [s]
        for t in strands:
            for i in range(len(t) - k + 1):
                x = t[i:i + k]
                if all(ch in b"ACGT" for ch in x):
                    kmers.add(x.decode())
    nodes = set(kmers)
    for x in kmers:
        if not any(c + x[:-1] in kmers for c in "ACGT"):
            for i in range(k):
                nodes.add("$" * (k - i) + x[:i])
    order = str.maketrans("$ACGT", "01234")
    ordered = sorted(nodes, key=lambda x: x.translate(order)[::-1])
    n = len(ordered)
    bits = np.zeros((4, n), np.uint8)
    sg = np.zeros(n, np.uint8)
    prev = None
    for i, x in enumerate(ordered):
        if x[1:] != prev:
            sg[i] = 1
            prev = x[1:]
            for ci, c in enumerate("ACGT"):
                if x[1:] + c in nodes:
                    bits[ci, i] = 1

    def words(b):
        w = np.packbits(b, bitorder="little")
        w = np.concatenate([w, np.zeros((-len(w)) % 8, np.uint8)])
        return w.view(np.uint64).copy()

    return [words(bits[c]) for c in range(4)], words(sg), n, len(kmers)
