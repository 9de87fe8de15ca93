"""Bounded device waits and concurrent use of shared handles.

* The key-k-mer walk (reference IndexSearcher.cuh:60-70) loops forever in the
  reference when a non-key node has no outgoing edge or when first-edge
  successors form a cycle without a key node.  The walk here stops (at once
  on a dead end, after 2^16 steps on a cycle) and the call returns
  SBWT_E_TIMEOUT; the device stays usable.  Neither the oracle nor the
  reference is run on these marks: both would not return.
* Index and color handles are immutable after open: host threads that call
  sbwt_search_reads / sbwt_pseudoalign on one shared handle get the results
  of single-threaded calls."""
import threading

import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
import sbwt_tools as T
from helpers import TMP, mixed_reads, oracle_index, oracle_results

pytestmark = pytest.mark.gpu


def genome_with_poly_a(seed=61):
    g = T.gen_genomes(seed, 2, 3000, 1, 0.02, 0.02, 0.0)
    seqs = [g.seq(0)[:1500] + b"A" * 40 + g.seq(0)[1500:], g.seq(1)]
    lens = np.array([len(s) for s in seqs], np.uint64)
    chars = np.frombuffer(b"".join(seqs), np.uint8).copy()
    return T.Genomes(chars, lens)


def node_of(oi, kmer: bytes) -> int:
    bits, _ = O.seq_to_bits(kmer)
    return int(oi.search_positions(bits, np.zeros(1, np.uint64))[0])


def bit(words, i):
    return (int(words[i >> 6]) >> (i & 63)) & 1


def all_but(n, v):
    keys = np.full((n + 63) // 64, ~np.uint64(0), np.uint64)
    keys[v >> 6] &= ~np.uint64(1 << (v & 63))
    return keys


def one_read(kmer: bytes):
    return np.frombuffer(kmer, np.uint8).copy(), np.array([len(kmer)], np.uint64)


def check_device_still_usable(path, g):
    idx = S.SbwtIndex.open(path)
    chars, ends = mixed_reads(g, 5, 200)
    assert np.array_equal(idx.search_reads(chars, ends), oracle_results(oracle_index(path, 8),
                                                                        chars, ends))
    idx.close()


@pytest.fixture(scope="module")
def poly_a_index():
    g = genome_with_poly_a()
    path = str(TMP / "poly_a.sbwt")
    T.build_sbwt(g, 31, path)
    return g, path, O.SbwtFile.read(path), oracle_index(path, 8)


def test_key_walk_dead_end_times_out(poly_a_index):
    g, path, sb, oi = poly_a_index
    chars, ends = mixed_reads(g, 3, 50, sub=0.0, n_rate=0.0, frac=1.0)
    res = oracle_results(oi, chars, ends)
    reads = T.split_reads(chars, ends)
    starts = np.concatenate([[0], np.cumsum([max(0, len(r) - 30) for r in reads])])
    # a found k-mer whose node starts no suffix group: it has no outgoing edge
    for r, read in enumerate(reads):
        hit = [j for j in range(int(starts[r + 1] - starts[r]))
               if res[starts[r] + j] < O.INVALID and not bit(sb.suffix_group_starts,
                                                              int(res[starts[r] + j]))]
        if hit:
            kmer, v = read[hit[0]:hit[0] + 31], int(res[starts[r] + hit[0]])
            break
    assert all(bit(a, v) == 0 for a in sb.acgt)
    idx = S.SbwtIndex.from_arrays(sb.acgt, sb.num_bits, 31, sb.suffix_group_starts,
                                  key_kmer_marks=all_but(sb.num_bits, v))
    c1, e1 = one_read(kmer)
    with pytest.raises(S.SbwtError) as ex:
        idx.search_reads(c1, e1, move_to_key_kmer=True)
    assert ex.value.code == S.E_TIMEOUT
    bits, _ = O.seq_to_bits(kmer)
    with pytest.raises(S.SbwtError) as ex:
        idx.search(bits, np.zeros(1, np.uint64), move_to_key_kmer=True)
    assert ex.value.code == S.E_TIMEOUT
    # without the walk the same handle answers, and the error was cleared
    assert int(idx.search_reads(c1, e1)[0]) == v
    idx.close()
    check_device_still_usable(path, g)


def test_key_walk_cycle_times_out(poly_a_index):
    g, path, sb, oi = poly_a_index
    v = node_of(oi, b"A" * 31)
    assert v < O.INVALID
    # A^31 starts its suffix group and its first edge (A) leads back to it
    assert bit(sb.suffix_group_starts, v) and bit(sb.acgt[0], v)
    idx = S.SbwtIndex.from_arrays(sb.acgt, sb.num_bits, 31, sb.suffix_group_starts,
                                  key_kmer_marks=all_but(sb.num_bits, v))
    c1, e1 = one_read(b"A" * 33)  # three k-mers, all A^31
    with pytest.raises(S.SbwtError) as ex:
        idx.search_reads(c1, e1, move_to_key_kmer=True)
    assert ex.value.code == S.E_TIMEOUT
    bits, _ = O.seq_to_bits(b"A" * 31)
    with pytest.raises(S.SbwtError) as ex:
        idx.search(bits, np.zeros(1, np.uint64), move_to_key_kmer=True)
    assert ex.value.code == S.E_TIMEOUT
    assert list(idx.search_reads(c1, e1)) == [v, v, v]
    idx.close()
    check_device_still_usable(path, g)


def run_threads(fns, rounds=3):
    errors, out = [], [None] * len(fns)

    def work(i):
        try:
            for _ in range(rounds):
                r = fns[i]()
                if out[i] is None:
                    out[i] = r
                elif not (r == out[i] if isinstance(r, list) else np.array_equal(r, out[i])):
                    errors.append(f"thread {i}: results changed between rounds")
        except Exception as e:  # reported below
            errors.append(f"thread {i}: {e!r}")

    ts = [threading.Thread(target=work, args=(i,)) for i in range(len(fns))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors
    return out


@pytest.mark.parametrize("table", [True, False])
def test_concurrent_search_reads_on_one_handle(table):
    g = T.gen_genomes(71, 3, 20000, 1, 0.02, 0.02, 0.0)
    path = str(TMP / "threads.sbwt")
    T.build_sbwt(g, 31, path)
    idx = S.SbwtIndex.open(path)
    idx.set_kmer_table(table)
    inputs = [mixed_reads(g, 100 + i, 3000 + 500 * i) for i in range(4)]
    single = [idx.search_reads(c, e) for c, e in inputs]
    got = run_threads([lambda c=c, e=e: idx.search_reads(c, e) for c, e in inputs])
    for a, b in zip(got, single):
        assert np.array_equal(a, b)
    oi = oracle_index(path, 8)
    assert np.array_equal(single[0], oracle_results(oi, *inputs[0]))
    idx.close()


def test_concurrent_pseudoalign_on_one_handle():
    g = T.gen_genomes(73, 40, 2000, 4, 0.01, 0.04, 0.0)
    sp, cp = str(TMP / "threads_col.sbwt"), str(TMP / "threads_col.tcolors")
    T.build_colored(g, 31, sp, cp)
    idx = S.SbwtIndex.open(sp)
    ci = S.ColorIndex.open(cp)
    batches = []
    for i in range(4):
        chars, ends = T.gen_reads(200 + i, g, 600 + 100 * i, 0.9, 120, 0.3, 31, 300, 0.01,
                                  0.002)
        res = idx.search_reads(chars, ends)
        per, t = [], 0
        for r in T.split_reads(chars, ends):
            m = max(0, len(r) - 30)
            per.append(res[t:t + m])
            t += m
        found = [p[p < O.INVALID] for p in per]
        offs = np.zeros(len(found) + 1, np.uint64)
        offs[1:] = np.cumsum([len(f) for f in found])
        nf = np.array([(p == O.NOT_FOUND).sum() for p in per], np.uint64)
        inv = np.array([(p == O.INVALID).sum() for p in per], np.uint64)
        batches.append((np.concatenate(found).astype(np.uint64), offs, nf, inv, found))
    single = [ci.pseudoalign(b[0], b[1], b[2], b[3], 0.7)[0] for b in batches]
    got = run_threads([lambda b=b: ci.pseudoalign(b[0], b[1], b[2], b[3], 0.7)[0]
                       for b in batches])
    assert got == single
    oc = O.OracleColors(O.ColorsFile.read(cp))
    b = batches[0]
    assert single[0] == oc.pseudoalign(b[4], b[2], b[3], 0.7)
    idx.close()
    ci.close()
