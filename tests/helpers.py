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
