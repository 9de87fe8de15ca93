"""The oracle (CPU restatement) and the reference's own index kernels
compiled for the host are pinned against the reference's golden fixtures
(test_objects/full_pipeline/index_search/expected/*.txt) and against each
other; the project's SBWT builder is checked for SBWT invariants."""
import numpy as np
import pytest

import oracle as O
from helpers import FIXTURE_FILES, GOLDEN, golden_sbwt_path, synthetic, oracle_index, \
    mixed_reads, oracle_results


def _expected(name):
    return O.read_ascii_index_results(GOLDEN / "index_search" / "expected" /
                                      (name.split(".")[0] + ".txt"))


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_oracle_reproduces_reference_fixture(name):
    sb = O.SbwtFile.read(golden_sbwt_path())
    assert (sb.k, sb.num_bits, sb.n_nodes, sb.n_kmers) == (30, 236, 236, 177)
    idx = oracle_index(golden_sbwt_path(), 10)
    reads = O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    got = [O.as_signed_tokens(r) for r in O.index_search_reads(idx, reads)]
    assert got == _expected(name)


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_reference_cpu_build_reproduces_fixture(name):
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    sb = O.SbwtFile.read(golden_sbwt_path())
    idx = O.OracleIndex(sb.acgt, sb.num_bits, sb.k, use_ref=True)
    reads = O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    got = [O.as_signed_tokens(r) for r in O.index_search_reads(idx, reads)]
    assert got == _expected(name)


def test_presearch_depth_does_not_change_results():
    g, path, sb = synthetic(2, 1, 5000)
    chars, ends = mixed_reads(g, 3, 300)
    base = oracle_results(oracle_index(path, 10), chars, ends)
    for p in (1, 5, 8):
        assert np.array_equal(oracle_results(oracle_index(path, p), chars, ends), base)


def test_oracle_matches_reference_kernels_on_synthetic():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    g, path, sb = synthetic(4, 2, 4000, 31, 1, 0.02)
    ref = O.OracleIndex(sb.acgt, sb.num_bits, sb.k, use_ref=True)
    chars, ends = mixed_reads(g, 5, 400)
    assert np.array_equal(oracle_results(ref, chars, ends),
                          oracle_results(oracle_index(path, 8), chars, ends))


def test_builder_sbwt_invariants():
    g, path, sb = synthetic(6, 3, 3000, 31, 1, 0.03)
    idx = oracle_index(path, 8)
    # every non-root node has exactly one incoming marked edge
    assert int(idx.c_map[4]) == sb.num_bits
    # every k-mer of every genome (both strands) is found, and distinct k-mers
    # get distinct nodes
    comp = bytes.maketrans(b"ACGT", b"TGCA")
    seqs = [g.seq(i) for i in range(len(g))]
    seqs += [s.translate(comp)[::-1] for s in seqs]
    rows = O.index_search_reads(idx, seqs)
    allv = np.concatenate(rows)
    assert (allv < O.INVALID).all()
    kmers = set()
    for s in seqs:
        for i in range(len(s) - 30):
            kmers.add(s[i:i + 31])
    assert len(np.unique(allv)) == len(kmers) == sb.n_kmers
    # the suffix-group starts: root is a start; every node with an edge is one
    sg = sb.suffix_group_starts
    assert sg[0] & 1
    for c in range(4):
        assert not np.any(sb.acgt[c] & ~sg)


def test_fastx_parser_kseq_semantics():
    data = b">a\nAC\nGT\n>b\n>c\nTT\n@q\nACG\nT\n+\nIIII\n@r\n\n+\n\n"
    assert O.parse_fastx(data) == [b"ACGT", b"", b"TT", b"ACGT", b""]
