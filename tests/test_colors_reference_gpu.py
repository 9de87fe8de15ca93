"""Colors step on the GPU pinned to the reference's own code: the C-ABI
counts (sbwt_color_counts) and ids (sbwt_pseudoalign) equal what
SBWT-Search's d_color_search + d_post_process (ColorSearcher.cuh:68-318,
ColorPostProcessor.cuh:21-43, compiled for the host by oracle/ref_colors.cpp)
and its printer's threshold rule (ContinuousColorResultsPrinter.hpp:235-263)
give on the same padding-free batch, with and without the per-node record
table."""
import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
from test_colors_reference import colored_index, padding_free_inputs, reference_ids

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.ref_lib() is None,
                                 reason="reference CPU build (oracle/_ref) missing")]


def flat(lists):
    offs = np.zeros(len(lists) + 1, np.uint64)
    offs[1:] = np.cumsum([len(x) for x in lists])
    return np.concatenate(lists).astype(np.uint64), offs


@pytest.mark.parametrize("n_colors", [12, 150, 2100, 9000])
@pytest.mark.parametrize("node_table", [True, False])
def test_gpu_counts_equal_reference_kernels(n_colors, node_table):
    g, sp, cp = colored_index(n_colors)
    n_reads = 400 if n_colors < 9000 else 300
    lists, warped, wi, nf, inv = padding_free_inputs(n_colors, n_reads, 21)
    ref = O.RefColors(O.ColorsFile.read(cp)).color_counts(warped, wi)
    ci = S.ColorIndex.open(cp)
    assert ci.set_node_table(node_table) == node_table
    idx, offs = flat(lists)
    got = ci.counts(idx, offs)
    assert np.array_equal(got.astype(np.uint64), ref)
    ci.close()


@pytest.mark.parametrize("tau", [0.0, 0.3, 0.7, 1.0])
@pytest.mark.parametrize("n_colors", [150, 2100])
def test_gpu_ids_equal_reference_threshold(tau, n_colors):
    g, sp, cp = colored_index(n_colors)
    lists, warped, wi, nf, inv = padding_free_inputs(n_colors, 400, 22)
    ref = O.RefColors(O.ColorsFile.read(cp)).color_counts(warped, wi)
    ci = S.ColorIndex.open(cp)
    idx, offs = flat(lists)
    nfa, inva = np.array(nf, np.uint64), np.array(inv, np.uint64)
    for inc_nf, inc_inv in ((False, False), (True, True)):
        rows, _, _ = ci.pseudoalign(idx, offs, nfa, inva, tau, inc_nf, inc_inv)
        exp = [reference_ids(ref[r], len(lists[r]) + inc_nf * nf[r] + inc_inv * inv[r], tau)
               for r in range(len(lists))]
        assert rows == exp
    ci.close()
