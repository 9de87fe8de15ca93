"""Colors step on the GPU through the C ABI, bit-exact against the oracle
(counts per read and color, and the thresholded sorted ids)."""
import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
import sbwt_tools as T
from helpers import TMP, oracle_index, oracle_results

pytestmark = pytest.mark.gpu


def colored(seed, n, length, founders, lo=0.01, hi=0.05):
    g = T.gen_genomes(seed, n, length, founders, lo, hi, 0.0)
    sp = TMP / f"gcol_{seed}_{n}_{length}.sbwt"
    cp = TMP / f"gcol_{seed}_{n}_{length}.tcolors"
    T.build_colored(g, 31, str(sp), str(cp))
    return g, str(sp), str(cp)


def index_results(sp, g, seed, n_reads, sigma=0.3):
    idx = S.SbwtIndex.open(sp)
    chars, ends = T.gen_reads(seed, g, n_reads, 0.9, 120, sigma, 31, 400, 0.01, 0.003)
    res = idx.search_reads(chars, ends)
    per, t = [], 0
    for r in T.split_reads(chars, ends):
        m = max(0, len(r) - 30)
        per.append(res[t:t + m])
        t += m
    return per


def split(per):
    found = [p[p < O.INVALID] for p in per]
    nf = np.array([(p == O.NOT_FOUND).sum() for p in per], np.uint64)
    inv = np.array([(p == O.INVALID).sum() for p in per], np.uint64)
    offs = np.zeros(len(found) + 1, np.uint64)
    offs[1:] = np.cumsum([len(f) for f in found])
    flat = np.concatenate(found) if found else np.zeros(0, np.uint64)
    return found, flat, offs, nf, inv


@pytest.mark.parametrize("case", [(3, 12, 3000, 3), (5, 150, 800, 6)])
def test_counts_match_oracle(case):
    seed, n, length, founders = case
    g, sp, cp = colored(seed, n, length, founders)
    per = index_results(sp, g, seed + 1, 400)
    found, flat, offs, nf, inv = split(per)
    ci = S.ColorIndex.open(cp)
    assert ci.num_colors == n
    got = ci.counts(flat, offs)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    _, exp = oc.pseudoalign(found, nf, inv, 0.7, want_counts=True)
    assert np.array_equal(got.astype(np.uint64), exp)


@pytest.mark.parametrize("tau", [0.0, 0.3, 0.7, 1.0])
@pytest.mark.parametrize("flags", [(False, False), (True, False), (True, True)])
def test_pseudoalign_matches_oracle(tau, flags):
    g, sp, cp = colored(5, 150, 800, 6)
    per = index_results(sp, g, 17, 600, sigma=0.6)
    found, flat, offs, nf, inv = split(per)
    ci = S.ColorIndex.open(cp)
    rows, _, _ = ci.pseudoalign(flat, offs, nf, inv, tau, *flags)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    exp = oc.pseudoalign(found, nf, inv, tau, *flags)
    assert rows == exp
    assert any(rows) or tau == 0.0  # minimum = ceil(0) = 0 prints nothing


def test_many_colors_two_words_per_lane():
    # 2100 colors -> 33 row words -> two words per lane
    g, sp, cp = colored(8, 2100, 200, 10, 0.01, 0.03)
    per = index_results(sp, g, 9, 300)
    found, flat, offs, nf, inv = split(per)
    ci = S.ColorIndex.open(cp)
    rows, _, _ = ci.pseudoalign(flat, offs, nf, inv, 0.5)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    assert rows == oc.pseudoalign(found, nf, inv, 0.5)
    got = ci.counts(flat, offs)
    _, exp = oc.pseudoalign(found, nf, inv, 0.5, want_counts=True)
    assert np.array_equal(got.astype(np.uint64), exp)


def test_empty_reads_and_capacity_retry():
    g, sp, cp = colored(3, 12, 3000, 3)
    ci = S.ColorIndex.open(cp)
    offs = np.zeros(4, np.uint64)
    rows, _, _ = ci.pseudoalign(np.zeros(0, np.uint64), offs, tau=0.7)
    assert rows == [[], [], []]


def test_bad_index_is_an_error():
    g, sp, cp = colored(3, 12, 3000, 3)
    ci = S.ColorIndex.open(cp)
    with pytest.raises(S.SbwtError) as e:
        ci.pseudoalign(np.array([1 << 40], np.uint64), np.array([0, 1], np.uint64))
    assert e.value.code == S.E_INVALID
