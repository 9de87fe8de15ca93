"""Colors step on the CPU: the .tcolors writer of the project's tools and the
oracle's reader agree, and the oracle's pseudoalignment behaves as the
reference's threshold rule says."""
import math

import numpy as np

import oracle as O
import sbwt_tools as T
from helpers import TMP, oracle_index, oracle_results


def colored(seed=3, n=12, length=3000, founders=3, lo=0.01, hi=0.05):
    g = T.gen_genomes(seed, n, length, founders, lo, hi, 0.0)
    sp = TMP / f"col_{seed}_{n}_{length}.sbwt"
    cp = TMP / f"col_{seed}_{n}_{length}.tcolors"
    T.build_colored(g, 31, str(sp), str(cp))
    return g, str(sp), str(cp)


def found_lists(index, g, seed, n_reads):
    chars, ends = T.gen_reads(seed, g, n_reads, 1.0, 120, 0.0, 120, 120, 0.005, 0.002)
    res = oracle_results(index, chars, ends)
    per, t = [], 0
    for r in T.split_reads(chars, ends):
        m = max(0, len(r) - 30)
        per.append(res[t:t + m])
        t += m
    return per


def test_tcolors_roundtrip_and_membership():
    g, sp, cp = colored()
    tc = O.ColorsFile.read(cp)
    assert tc.num_colors == len(g)
    idx = oracle_index(sp, 8)
    oc = O.OracleColors(tc)
    # every k-mer of genome i has color i in its set
    for gi in (0, 5, 11):
        rows = O.index_search_reads(idx, [g.seq(gi)])
        found = [np.asarray(rows[0], np.uint64)]
        _, counts = oc.pseudoalign(found, [0], [0], 1.0, want_counts=True)
        assert counts[0, gi] == len(rows[0])


def test_threshold_rule():
    g, sp, cp = colored()
    tc = O.ColorsFile.read(cp)
    oc = O.OracleColors(tc)
    per = found_lists(oracle_index(sp, 8), g, 9, 50)
    found = [p[p < O.INVALID] for p in per]
    nf = [int((p == O.NOT_FOUND).sum()) for p in per]
    inv = [int((p == O.INVALID).sum()) for p in per]
    for tau in (0.0, 0.5, 0.7, 1.0):
        rows, counts = oc.pseudoalign(found, nf, inv, tau, True, True, want_counts=True)
        for r in range(len(found)):
            size = len(found[r]) + nf[r] + inv[r]
            m = int(math.ceil(size * tau))
            exp = [] if m == 0 else [c for c in range(tc.num_colors) if counts[r, c] >= m]
            assert rows[r] == exp


def test_multithreaded_restatement_matches_single_thread():
    """The OpenMP form of the restatement (the colors CPU baseline) gives
    the single-thread restatement's ids per read (count and checksum)."""
    g, sp, cp = colored()
    tc = O.ColorsFile.read(cp)
    oc = O.OracleColors(tc)
    per = found_lists(oracle_index(sp, 8), g, 11, 300)
    found = [p[p < O.INVALID] for p in per]
    nf = [int((p == O.NOT_FOUND).sum()) for p in per]
    inv = [int((p == O.INVALID).sum()) for p in per]
    offs = np.zeros(len(found) + 1, np.uint64)
    offs[1:] = np.cumsum([len(f) for f in found])
    rows = oc.pseudoalign(found, nf, inv, 0.7)
    n_ids, ck = oc.pseudoalign_mt(np.concatenate(found), offs, nf, inv, 0.7, threads=4)
    assert list(n_ids) == [len(r) for r in rows]
    assert np.array_equal(ck, O.ids_checksum(rows))
