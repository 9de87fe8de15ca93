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


def open_colors(cp, node_table=True):
    ci = S.ColorIndex.open(cp)
    assert ci.set_node_table(node_table) == node_table
    return ci


def split(per):
    found = [p[p < O.INVALID] for p in per]
    nf = np.array([(p == O.NOT_FOUND).sum() for p in per], np.uint64)
    inv = np.array([(p == O.INVALID).sum() for p in per], np.uint64)
    offs = np.zeros(len(found) + 1, np.uint64)
    offs[1:] = np.cumsum([len(f) for f in found])
    flat = np.concatenate(found) if found else np.zeros(0, np.uint64)
    return found, flat, offs, nf, inv


@pytest.mark.parametrize("case", [(3, 12, 3000, 3), (5, 150, 800, 6)])
@pytest.mark.parametrize("node_table", [True, False])
def test_counts_match_oracle(case, node_table):
    seed, n, length, founders = case
    g, sp, cp = colored(seed, n, length, founders)
    per = index_results(sp, g, seed + 1, 400)
    found, flat, offs, nf, inv = split(per)
    ci = open_colors(cp, node_table)
    assert ci.num_colors == n
    got = ci.counts(flat, offs)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    _, exp = oc.pseudoalign(found, nf, inv, 0.7, want_counts=True)
    assert np.array_equal(got.astype(np.uint64), exp)


@pytest.mark.parametrize("tau", [0.0, 0.3, 0.7, 1.0])
@pytest.mark.parametrize("flags", [(False, False), (True, False), (True, True)])
@pytest.mark.parametrize("node_table", [True, False])
def test_pseudoalign_matches_oracle(tau, flags, node_table):
    g, sp, cp = colored(5, 150, 800, 6)
    per = index_results(sp, g, 17, 600, sigma=0.6)
    found, flat, offs, nf, inv = split(per)
    ci = open_colors(cp, node_table)
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


@pytest.mark.parametrize("node_table", [True, False])
def test_bad_index_is_an_error(node_table):
    g, sp, cp = colored(3, 12, 3000, 3)
    ci = open_colors(cp, node_table)
    with pytest.raises(S.SbwtError) as e:
        ci.pseudoalign(np.array([1 << 40], np.uint64), np.array([0, 1], np.uint64))
    assert e.value.code == S.E_INVALID


@pytest.mark.parametrize("n_colors", [9000, 20000])
@pytest.mark.parametrize("node_table", [True, False])
def test_color_tiles_beyond_8192_colors(n_colors, node_table):
    # more than 8192 colors -> several color tiles per read (row words split
    # across warps), with sparse lists that cross tile boundaries
    g, sp, cp = colored(21, n_colors, 120, 12, 0.01, 0.04)
    per = index_results(sp, g, 22, 200)
    found, flat, offs, nf, inv = split(per)
    ci = open_colors(cp, node_table)
    assert ci.num_colors == n_colors
    oc = O.OracleColors(O.ColorsFile.read(cp))
    for tau in (0.3, 0.8):
        rows, _, _ = ci.pseudoalign(flat, offs, nf, inv, tau)
        assert rows == oc.pseudoalign(found, nf, inv, tau)
    got = ci.counts(flat, offs)
    _, exp = oc.pseudoalign(found, nf, inv, 0.5, want_counts=True)
    assert np.array_equal(got.astype(np.uint64), exp)


@pytest.mark.parametrize("node_table", [True, False])
def test_repeated_indexes_in_a_window(node_table):
    # every found index of a read repeated and shuffled: a 32-k-mer window
    # holds up to 32 copies of one index, not adjacent to each other
    g, sp, cp = colored(5, 150, 800, 6)
    per = index_results(sp, g, 31, 300)
    rng = np.random.default_rng(3)
    found = []
    for p in per:
        f = p[p < O.INVALID]
        rep = np.repeat(f, rng.integers(1, 40, size=len(f))) if len(f) else f
        found.append(rng.permutation(rep).astype(np.uint64))
    found.append(np.full(97, found[0][0] if len(found[0]) else 0, np.uint64))
    nf = np.zeros(len(found), np.uint64)
    offs = np.zeros(len(found) + 1, np.uint64)
    offs[1:] = np.cumsum([len(f) for f in found])
    flat = np.concatenate(found)
    ci = open_colors(cp, node_table)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    got = ci.counts(flat, offs)
    _, exp = oc.pseudoalign(found, nf, nf, 0.5, want_counts=True)
    assert np.array_equal(got.astype(np.uint64), exp)
    rows, _, _ = ci.pseudoalign(flat, offs, nf, nf, 0.6)
    assert rows == oc.pseudoalign(found, nf, nf, 0.6)


@pytest.mark.parametrize("n_reads", [4096, 8192, 12289])
def test_many_reads_multi_block_scan(n_reads):
    # the ids offsets scan runs in blocks of 4096 reads: exact multiples and a
    # ragged tail, through host buffers and through device pointers
    import torch
    g, sp, cp = colored(5, 150, 800, 6)
    per = index_results(sp, g, 41, 200)
    pool = [p[p < O.INVALID] for p in per]
    rng = np.random.default_rng(n_reads)
    found = [pool[i][:int(rng.integers(0, len(pool[i]) + 1))]
             for i in rng.integers(0, len(pool), n_reads)]
    nf = np.zeros(n_reads, np.uint64)
    offs = np.zeros(n_reads + 1, np.uint64)
    offs[1:] = np.cumsum([len(f) for f in found])
    flat = np.concatenate(found).astype(np.uint64)
    ci = S.ColorIndex.open(cp)
    oc = O.OracleColors(O.ColorsFile.read(cp))
    rows, ids_off, ids = ci.pseudoalign(flat, offs, nf, nf, 0.5)
    assert rows == oc.pseudoalign(found, nf, nf, 0.5)
    d_flat = torch.from_numpy(flat.view(np.int64)).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    cap = int(ids_off[-1]) + 1
    d_ids = torch.zeros(cap, dtype=torch.int32, device="cuda")
    d_ids_off = torch.zeros(n_reads + 1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    S.check(S.lib().sbwt_pseudoalign(ci._h, d_flat.data_ptr(), d_offs.data_ptr(), None, None,
                                     n_reads, 0.5, S.DEVICE_POINTERS, d_ids.data_ptr(), cap,
                                     d_ids_off.data_ptr(), stream.cuda_stream))
    torch.cuda.synchronize()
    assert np.array_equal(d_ids_off.cpu().numpy().view(np.uint64), ids_off)
    n_ids = int(ids_off[-1])
    assert np.array_equal(d_ids[:n_ids].cpu().numpy().view(np.uint32), ids[:n_ids])


def test_device_offsets_must_not_decrease():
    import torch
    g, sp, cp = colored(3, 12, 3000, 3)
    ci = S.ColorIndex.open(cp)
    d_flat = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_offs = torch.tensor([0, 3, 2, 4], dtype=torch.int64, device="cuda")
    d_ids = torch.zeros(16, dtype=torch.int32, device="cuda")
    d_ids_off = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = S.lib().sbwt_pseudoalign(ci._h, d_flat.data_ptr(), d_offs.data_ptr(), None, None, 3,
                                  0.5, S.DEVICE_POINTERS, d_ids.data_ptr(), 16,
                                  d_ids_off.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == S.E_INVALID
