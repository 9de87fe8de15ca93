"""Colors step pinned to the reference's own code on the CPU: the oracle's
restated counts (oracle/sbwt_oracle.c) equal the counts of SBWT-Search's
d_color_search + d_post_process (src/ColorSearcher/ColorSearcher.cuh:68-318,
ColorPostProcessor.cuh:21-43) compiled for the host with a warp-lockstep
shim (oracle/ref_colors.cpp), and the oracle's ids equal the reference
printer's threshold rule (ContinuousColorResultsPrinter.hpp:235-263) applied
to those counts.

Inputs are padding-free (every read keeps a positive multiple of 32 found
indexes, the batch a multiple of 1024): there the reference kernel has no
lane that leaves before its full-mask collectives, so its result is
defined."""
from __future__ import annotations

from functools import lru_cache

import numpy as np
import pytest

import oracle as O
import sbwt_tools as T
from helpers import TMP, oracle_index, oracle_results

pytestmark = pytest.mark.skipif(O.ref_lib() is None,
                                reason="reference CPU build (oracle/_ref) missing")

# (seed, genomes, genome length, founders, divergence lo, hi): 12 and 150
# colors give dense and sparse sets; 2100 and 9000 colors go past the
# reference's 2000-color workload and past one 8192-color tile of the GPU.
INDEXES = {
    12: (3, 12, 4000, 3, 0.01, 0.05),
    150: (5, 150, 1500, 6, 0.01, 0.04),
    2100: (7, 2100, 300, 8, 0.01, 0.03),
    9000: (11, 9000, 250, 8, 0.005, 0.02),
}


@lru_cache(None)
def colored_index(n_colors: int):
    seed, n, length, founders, lo, hi = INDEXES[n_colors]
    g = T.gen_genomes(seed, n, length, founders, lo, hi, 0.0)
    sp = TMP / f"refcol_{n_colors}.sbwt"
    cp = TMP / f"refcol_{n_colors}.tcolors"
    T.build_colored(g, 31, str(sp), str(cp))
    return g, str(sp), str(cp)


@lru_cache(None)
def padding_free_inputs(n_colors: int, n_reads: int, seed: int):
    """Found-index lists of seeded reads, trimmed to a padding-free batch, and
    each kept read's not-found / invalid counts (from the untrimmed read)."""
    g, sp, cp = colored_index(n_colors)
    chars, ends = T.gen_reads(seed, g, n_reads, 1.0, 150, 0.3, 100, 400, 0.004, 0.002)
    res = oracle_results(oracle_index(sp, 8), chars, ends)
    per, t = [], 0
    for r in T.split_reads(chars, ends):
        m = max(0, len(r) - 30)
        per.append(res[t:t + m])
        t += m
    found = [p[p < O.INVALID] for p in per]
    keep, lists, warped, wi = O.padding_free_batch(found)
    nf = [int((per[i] == O.NOT_FOUND).sum()) for i in keep]
    inv = [int((per[i] == O.INVALID).sum()) for i in keep]
    return lists, warped, wi, nf, inv


def reference_ids(counts_row, seq_size: int, tau: float) -> list[int]:
    m = O.threshold_minimum(seq_size, tau)
    return [] if m == 0 else [int(c) for c in np.nonzero(counts_row >= m)[0]]


@pytest.mark.parametrize("n_colors", [12, 150, 2100, 9000])
def test_oracle_counts_equal_reference_kernels(n_colors):
    g, sp, cp = colored_index(n_colors)
    tc = O.ColorsFile.read(cp)
    assert tc.num_colors == n_colors
    n_reads = 400 if n_colors < 9000 else 300
    lists, warped, wi, nf, inv = padding_free_inputs(n_colors, n_reads, 21)
    assert len(warped) >= 1024 and len(warped) % 1024 == 0
    ref = O.RefColors(tc).color_counts(warped, wi)
    rows, counts = O.OracleColors(tc).pseudoalign(lists, nf, inv, 0.7, want_counts=True)
    assert counts.shape == ref.shape
    assert np.array_equal(counts, ref)
    # dense sets everywhere; sparse ones once sets of size <= C/64 exist
    dense = np.unpackbits(tc.is_dense_marks.view(np.uint8), bitorder="little")
    assert dense[:tc.is_dense_bits].any()
    if n_colors >= 128:
        assert not dense[:tc.is_dense_bits].all()


@pytest.mark.parametrize("n_colors", [12, 150])
def test_oracle_ids_equal_reference_threshold(n_colors):
    g, sp, cp = colored_index(n_colors)
    tc = O.ColorsFile.read(cp)
    lists, warped, wi, nf, inv = padding_free_inputs(n_colors, 400, 22)
    ref = O.RefColors(tc).color_counts(warped, wi)
    oc = O.OracleColors(tc)
    for tau in (0.0, 0.3, 0.7, 1.0):
        for inc_nf, inc_inv in ((False, False), (True, True)):
            rows = oc.pseudoalign(lists, nf, inv, tau, inc_nf, inc_inv)
            for r, row in enumerate(rows):
                size = len(lists[r]) + inc_nf * nf[r] + inc_inv * inv[r]
                assert row == reference_ids(ref[r], size, tau)


def test_reference_kernel_rejects_padding_lanes():
    """A warp with a -1 padding lane is undefined in the reference kernel;
    the host driver reports it instead of guessing."""
    g, sp, cp = colored_index(12)
    tc = O.ColorsFile.read(cp)
    lists, warped, wi, nf, inv = padding_free_inputs(12, 400, 21)
    bad = warped[:64].copy()
    bad[40] = O.NOT_FOUND
    with pytest.raises(ValueError):
        O.RefColors(tc).color_counts(bad, np.array([0, 2], np.uint64))
