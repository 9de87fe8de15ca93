"""k beyond one 64-bit word (the reference's walk takes any k >= 12 and reads
each char from the packed sequence per step, IndexSearcher.cuh:37-55):
indexes built by brute force from the SBWT definition (helpers.small_sbwt),
the oracle against the reference's own d_search built for the host on the
CPU, and the GPU read search, positions seam and key-k-mer walk against
both on the GPU."""
from __future__ import annotations

from functools import lru_cache

import numpy as np
import pytest

import oracle as O
import sbwt_tools as T
from helpers import key_marks_for, mixed_reads, small_sbwt

KS = [32, 33, 47, 63, 64, 100]


@lru_cache(None)
def large_k_index(k: int):
    g = T.gen_genomes(40 + k, 2, 3000, 1, 0.02, 0.02, 0.0)
    acgt, sg, n, nk = small_sbwt([g.seq(i) for i in range(len(g))], k)
    return g, acgt, sg, n, nk


@lru_cache(None)
def large_k_oracle(k: int):
    g, acgt, sg, n, nk = large_k_index(k)
    return O.OracleIndex(acgt, n, k, 8)


def reads_for(g, k, seed):
    return mixed_reads(g, seed, 300, median=max(120, k + 60), sub=0.01, n_rate=0.003,
                       len_max=max(400, 3 * k))


@pytest.mark.parametrize("k", [15, 31])
def test_small_sbwt_equals_project_builder(k, tmp_path):
    g = T.gen_genomes(3, 2, 3000, 1, 0.02, 0.02, 0.0)
    acgt, sg, n, nk = small_sbwt([g.seq(i) for i in range(len(g))], k)
    path = tmp_path / "x.sbwt"
    assert T.build_sbwt(g, k, str(path)) == n
    sb = O.SbwtFile.read(path)
    assert sb.num_bits == n
    for a, b in zip(acgt, sb.acgt):
        assert np.array_equal(a[:len(b)], b[:len(a)])
    assert np.array_equal(sg[:len(sb.suffix_group_starts)], sb.suffix_group_starts[:len(sg)])


@pytest.mark.skipif(O.ref_lib() is None, reason="reference CPU build (oracle/_ref) missing")
@pytest.mark.parametrize("k", [33, 47, 63, 100])
def test_oracle_matches_reference_large_k(k):
    g, acgt, sg, n, nk = large_k_index(k)
    oi = large_k_oracle(k)
    ref = O.OracleIndex(acgt, n, k, use_ref=True)
    chars, ends = reads_for(g, k, 7)
    bits, _ = O.seq_to_bits(chars.tobytes())
    pos = O.positions_of(ends, k)
    exp = oi.search_positions(bits, pos)
    assert np.array_equal(exp, ref.search_positions(bits, pos))
    assert (exp != O.NOT_FOUND).mean() > 0.1  # genome k-mers are found
    keys = key_marks_for(oi, 3, seed=k)
    assert np.array_equal(oi.search_positions(bits, pos, keys),
                          ref.search_positions(bits, pos, keys))


@pytest.mark.gpu
@pytest.mark.parametrize("k", KS)
def test_gpu_reads_and_positions_large_k(k):
    import sbwt_b200 as S
    g, acgt, sg, n, nk = large_k_index(k)
    oi = large_k_oracle(k)
    idx = S.SbwtIndex.from_arrays(acgt, n, k, sg)
    chars, ends = reads_for(g, k, 11)
    exp = np.concatenate(O.index_search_reads(oi, T.split_reads(chars, ends)))
    assert (exp < O.INVALID).any() and (exp == O.NOT_FOUND).any() and (exp == O.INVALID).any()
    assert np.array_equal(idx.search_reads(chars, ends), exp)
    assert np.array_equal(idx.search_reads(chars, ends, per_kmer_walk=True), exp)
    bits, _ = O.seq_to_bits(chars.tobytes())
    pos = O.positions_of(ends, k)
    got = idx.search(bits, pos)
    assert np.array_equal(got, oi.search_positions(bits, pos))
    if O.ref_lib() is not None:
        ref = O.OracleIndex(acgt, n, k, use_ref=True)
        assert np.array_equal(got, ref.search_positions(bits, pos))
    idx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("k", [33, 63])
def test_gpu_move_to_key_kmer_large_k(k):
    import sbwt_b200 as S
    g, acgt, sg, n, nk = large_k_index(k)
    oi = large_k_oracle(k)
    keys = key_marks_for(oi, 4, seed=k)
    idx = S.SbwtIndex.from_arrays(acgt, n, k, sg, key_kmer_marks=keys)
    chars, ends = reads_for(g, k, 13)
    exp = np.concatenate(O.index_search_reads(oi, T.split_reads(chars, ends), keys))
    assert np.array_equal(idx.search_reads(chars, ends, move_to_key_kmer=True), exp)
    bits, _ = O.seq_to_bits(chars.tobytes())
    pos = O.positions_of(ends, k)
    got = idx.search(bits, pos, move_to_key_kmer=True)
    assert np.array_equal(got, oi.search_positions(bits, pos, keys))
    if O.ref_lib() is not None:
        ref = O.OracleIndex(acgt, n, k, use_ref=True)
        assert np.array_equal(got, ref.search_positions(bits, pos, keys))
    idx.close()
