"""The read search kernels' shortcuts, restated on the CPU and checked against
the oracle's full searches (no GPU).

The table kernel (csrc/index.cu, search_table_kernel) resolves a k-mer in one
of three ways, and each one must give what a full backward search
(src/IndexSearcher/IndexSearcher.cuh:22-72 of the reference) gives:

* stream step: the k-mer follows a found k-mer with node v.  If bit c of v
  is set (c = the new last char), the node is C[c] + rank_c(v).  Otherwise
  the highest suffix-group start g <= v decides.  g == v means not found;
  else bit c of g gives C[c] + rank_c(g), or not found.  On the one-node
  interval [x, x] a backward step (IndexSearcher.cuh:52-54) is nonempty iff
  bit c of x is set.
* table lookup: every other k-mer is looked up in the k-mer -> node table.
  The table is built from the SBWT's own labels: the last char of node v is
  the c with C[c] <= v < C[c + 1]; its predecessor is the (v - C[c])-th set
  bit of vector c.  Chains that reach the root within k chars are dummies.
* invalid char: -2, and the stream restarts.

These tests build the table by that rule and run the rule per read.  Both
are compared with the oracle on the reference's golden index and on
synthetic indexes (k = 3, 15, 31).
"""
import numpy as np
import pytest

import oracle as O
import sbwt_tools as T
from helpers import (FIXTURE_FILES, GOLDEN, golden_sbwt_path, mixed_reads, oracle_index,
                     oracle_results, synthetic)

CODE = {ord("A"): 0, ord("C"): 1, ord("G"): 2, ord("T"): 3,
        ord("a"): 0, ord("c"): 1, ord("g"): 2, ord("t"): 3}


class BitVectors:
    """A/C/G/T bits, C-map and suffix-group starts of an SBWT, with rank."""

    def __init__(self, sb: O.SbwtFile):
        self.n = int(sb.num_bits)
        self.k = int(sb.k)
        self.bits = [np.unpackbits(a.view(np.uint8), bitorder="little")[:self.n]
                     .astype(bool) for a in sb.acgt]
        self.cum = [np.concatenate([[0], np.cumsum(b, dtype=np.int64)]) for b in self.bits]
        c = [1]
        for b in self.bits:
            c.append(c[-1] + int(b.sum()))
        self.c_map = c
        self.sg = np.unpackbits(sb.suffix_group_starts.view(np.uint8),
                                bitorder="little")[:self.n].astype(bool)
        self.ones = [np.flatnonzero(b) for b in self.bits]

    def rank(self, c: int, i: int) -> int:
        return int(self.cum[c][i])

    def bit(self, c: int, i: int) -> bool:
        return bool(self.bits[c][i])

    def group_start(self, v: int) -> int:
        """Highest suffix-group start <= v (-1 if none)."""
        starts = np.flatnonzero(self.sg[:v + 1])
        return int(starts[-1]) if len(starts) else -1

    def last_char(self, v: int):
        for c in range(4):
            if self.c_map[c] <= v < self.c_map[c + 1]:
                return c
        return None  # node 0: the root

    def predecessor(self, v: int) -> int:
        c = self.last_char(v)
        return int(self.ones[c][v - self.c_map[c]])


def kmer_table(bv: BitVectors) -> dict:
    """k-mer (first char on top, 2 bits each) -> node, from the labels."""
    table = {}
    for v in range(bv.n):
        key, u, ok = 0, v, True
        for i in range(bv.k):
            c = bv.last_char(u)
            if c is None:
                ok = False  # reached the root: a $-padded dummy node
                break
            key |= c << (2 * i)
            u = bv.predecessor(u)
        if ok:
            assert key not in table, "a k-mer has one node"
            table[key] = v
    return table


def stream_step(bv: BitVectors, v: int, c: int):
    if bv.bit(c, v):
        return bv.c_map[c] + bv.rank(c, v)
    g = bv.group_start(v)
    if g < 0 or g == v or not bv.bit(c, g):
        return None
    return bv.c_map[c] + bv.rank(c, g)


def table_rule_search(bv: BitVectors, table: dict, read: bytes) -> list:
    """One read through the table kernel's rules: per k-mer the node,
    NOT_FOUND or INVALID."""
    k, out, v = bv.k, [], None
    codes = [CODE.get(ch) for ch in read]
    for pos in range(len(read) - k + 1):
        window = codes[pos:pos + k]
        if any(x is None for x in window):
            out.append(O.INVALID)
            v = None
            continue
        if v is not None:
            v = stream_step(bv, v, window[-1])
        else:
            key = 0
            for x in window:
                key = (key << 2) | x
            v = table.get(key)
        out.append(O.NOT_FOUND if v is None else v)
    return out


def _check(path, chars, ends, p=8):
    sb = O.SbwtFile.read(path)
    bv = BitVectors(sb)
    table = kmer_table(bv)
    exp = oracle_results(oracle_index(path, min(p, sb.k)), chars, ends)
    got = []
    for r in T.split_reads(chars, ends):
        got.extend(table_rule_search(bv, table, bytes(r)))
    assert np.array_equal(np.array(got, dtype=np.uint64), exp)
    return table, exp


def test_table_holds_every_kmer_with_its_searched_node():
    """Every k-mer spelled by a label is found by the oracle's full search at
    that node, and the table is as large as the index's k-mer count."""
    path = golden_sbwt_path()
    sb = O.SbwtFile.read(path)
    bv = BitVectors(sb)
    table = kmer_table(bv)
    assert len(table) == sb.n_kmers
    k = sb.k
    keys = sorted(table)
    chars = b"".join("".join("ACGT"[(key >> (2 * (k - 1 - i))) & 3] for i in range(k)).encode()
                     for key in keys)
    ends = np.arange(1, len(keys) + 1, dtype=np.uint64) * k
    exp = oracle_results(oracle_index(path, 8), np.frombuffer(chars, np.uint8), ends)
    assert np.array_equal(exp, np.array([table[key] for key in keys], dtype=np.uint64))


def test_table_rule_on_golden_index():
    """The reference's fixture reads (k = 30) on its golden index."""
    reads = []
    for name in FIXTURE_FILES:
        reads += O.parse_fastx((GOLDEN / "index_search" / name).read_bytes())
    path = golden_sbwt_path()
    chars = np.frombuffer(b"".join(reads), np.uint8)
    ends = np.cumsum([len(r) for r in reads]).astype(np.uint64)
    _check(path, chars, ends)


@pytest.mark.parametrize("k", [3, 15, 31])
def test_table_rule_on_synthetic_indexes(k):
    g, path, sb = synthetic(40 + k, 3, 1500, k, 2, 0.02)
    chars, ends = mixed_reads(g, 50 + k, 120, median=70, sigma=0.8, len_min=0,
                              len_max=250, sub=0.02, n_rate=0.01)
    _, exp = _check(path, chars, ends)
    # the reads exercise found, not-found and invalid k-mers (at k = 3 every
    # 3-mer is in the index, so none is not found)
    assert (exp < O.INVALID).any() and (exp == O.INVALID).any()
    assert (exp == O.NOT_FOUND).any() or k < 8


@pytest.mark.parametrize("k", [9, 15])
def test_stream_rule_reaches_every_branch(k, monkeypatch):
    """On branchy indexes (two founders at 5 % divergence) and reads with 3 %
    substitutions, the stream step takes all four branches: bit set at v;
    bit clear, v starts its group (not found); bit clear, edge at the group
    start g < v; bit clear, no edge at g (not found).  Results stay equal to
    the oracle's."""
    seen = {"at_v": 0, "v_starts_group": 0, "at_g": 0, "g_without_edge": 0}
    plain_step = stream_step

    def counting_step(bv, v, c):
        if bv.bit(c, v):
            seen["at_v"] += 1
        else:
            g = bv.group_start(v)
            seen["v_starts_group" if g == v else
                 ("at_g" if bv.bit(c, g) else "g_without_edge")] += 1
        return plain_step(bv, v, c)

    monkeypatch.setitem(globals(), "stream_step", counting_step)
    g, path, sb = synthetic(60 + k, 6 if k > 9 else 4, 2000 if k > 9 else 1500, k, 2, 0.05)
    chars, ends = mixed_reads(g, 70 + k, 200, median=70, sigma=0.8, len_min=0,
                              len_max=250, sub=0.03, n_rate=0.01)
    _check(path, chars, ends)
    assert all(seen.values()), seen


# ---------------------------------------------------------------------------
# The k-mer filter in front of the table (csrc/kmer_table.cu, used by
# search_walks_kernel): a blocked Bloom filter, 10 bits per k-mer, one 64-bit
# word per key (word = the high bits of the key's SplitMix64 hash times the
# word count, >> 64), four bits per key (hash bits 0-5, 6-11, 12-17, 18-23).
# ---------------------------------------------------------------------------
M64 = (1 << 64) - 1


def kmer_mix(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xbf58476d1ce4e5b9) & M64
    z = ((z ^ (z >> 27)) * 0x94d049bb133111eb) & M64
    return z ^ (z >> 31)


def filter_word_bits(key: int, n_words: int):
    z = kmer_mix(key)
    bits = 0
    for sh in (0, 6, 12, 18):
        bits |= 1 << ((z >> sh) & 63)
    return (z * n_words) >> 64, bits


def build_filter(keys, bits_per_kmer: int = 10):
    n_words = max((len(keys) * bits_per_kmer + 63) // 64, 1)
    words = [0] * n_words
    for key in keys:
        w, b = filter_word_bits(key, n_words)
        words[w] |= b
    return words


def filter_passes(words, key: int) -> bool:
    w, b = filter_word_bits(key, len(words))
    return (words[w] & b) == b


def walks_rule_search(bv: BitVectors, table: dict, words, read: bytes, stats) -> list:
    """table_rule_search with the filter in front of every table lookup: a
    key the filter rejects is not found without a lookup."""
    k, out, v = bv.k, [], None
    codes = [CODE.get(ch) for ch in read]
    for pos in range(len(read) - k + 1):
        window = codes[pos:pos + k]
        if any(x is None for x in window):
            out.append(O.INVALID)
            v = None
            continue
        if v is not None:
            v = stream_step(bv, v, window[-1])
        else:
            key = 0
            for x in window:
                key = (key << 2) | x
            if filter_passes(words, key):
                stats["lookups"] += 1
                v = table.get(key)
                stats["false_pass"] += v is None
            else:
                stats["rejected"] += 1
                v = None
        out.append(O.NOT_FOUND if v is None else v)
    return out


@pytest.mark.parametrize("k", [15, 31])
def test_filter_rule_matches_oracle(k):
    """The filter has no false negatives (every table key passes), so the
    walks kernel's rule gives the oracle's results; it rejects most absent
    k-mers before a table lookup."""
    g, path, sb = synthetic(80 + k, 3, 3000, k, 2, 0.02)
    bv = BitVectors(sb)
    table = kmer_table(bv)
    words = build_filter(list(table))
    assert all(filter_passes(words, key) for key in table)
    chars, ends = mixed_reads(g, 90 + k, 300, median=90, sigma=0.6, len_min=0,
                              len_max=300, sub=0.02, n_rate=0.005, frac=0.5)
    exp = oracle_results(oracle_index(path, 8), chars, ends)
    stats = {"lookups": 0, "false_pass": 0, "rejected": 0}
    got = []
    for r in T.split_reads(chars, ends):
        got.extend(walks_rule_search(bv, table, words, bytes(r), stats))
    assert np.array_equal(np.array(got, dtype=np.uint64), exp)
    absent = stats["rejected"] + stats["false_pass"]
    assert absent > 1000
    assert stats["false_pass"] / absent < 0.04  # about 1.5 % at 10 bits per k-mer


def test_filter_false_positive_rate():
    """On random keys the filter passes about 1-2 % (10 bits per key, 4 bits
    in one 64-bit word)."""
    rng = np.random.default_rng(5)
    keys = [int(x) for x in rng.integers(0, 1 << 62, 40000, dtype=np.int64)]
    words = build_filter(keys)
    probes = [int(x) for x in rng.integers(0, 1 << 62, 40000, dtype=np.int64)]
    fp = sum(filter_passes(words, p) for p in probes) / len(probes)
    assert 0.005 < fp < 0.03, fp
