"""SBWT construction on the GPU (sbwt_build_index) against the project's host
builder: byte-identical .sbwt files, and the GPU-built index searches like
the oracle."""
import numpy as np
import pytest

import sbwt_b200 as S
import sbwt_tools as T
from helpers import mixed_reads, oracle_index, oracle_results

pytestmark = pytest.mark.gpu


def sequences(seed, k):
    g = T.gen_genomes(seed, 6, 2500, 2, 0.02, 0.03, 0.01)
    rng = np.random.default_rng(seed)
    chars = g.chars.copy()
    chars[rng.integers(0, len(chars), 25)] = ord("N")
    lower = rng.integers(0, len(chars), 200)
    chars[lower] = np.char.lower(chars[lower].view("S1")).view(np.uint8)
    extra = [rng.choice(np.frombuffer(b"ACGT", np.uint8), n) for n in (5, 0, k, k - 1, 3 * k)]
    all_chars = np.concatenate([chars] + extra).astype(np.uint8)
    lens = np.concatenate([g.lens, [len(e) for e in extra]]).astype(np.uint64)
    return all_chars, lens


@pytest.mark.parametrize("k,rc", [(31, True), (31, False), (15, True), (21, False), (3, True)])
def test_gpu_builder_matches_host_builder(k, rc, tmp_path):
    chars, lens = sequences(k, k)
    hp, dp = tmp_path / "host.sbwt", tmp_path / "gpu.sbwt"
    nh = T.build_sbwt(T.Genomes(chars, lens), k, str(hp), rc)
    nd = S.build_index((chars, np.cumsum(lens).astype(np.uint64)), k, dp, rc)
    assert nd == nh
    assert dp.read_bytes() == hp.read_bytes()


def test_empty_input_gives_the_root(tmp_path):
    hp, dp = tmp_path / "host.sbwt", tmp_path / "gpu.sbwt"
    T.build_sbwt(T.Genomes(np.zeros(0, np.uint8), np.zeros(0, np.uint64)), 31, str(hp), True)
    assert S.build_index([], 31, dp) == 1
    assert dp.read_bytes() == hp.read_bytes()


def test_gpu_built_index_searches_like_the_oracle(tmp_path):
    g = T.gen_genomes(77, 8, 20000, 3, 0.02, 0.02, 0.001)
    path = tmp_path / "g.sbwt"
    S.build_index((g.chars, np.cumsum(g.lens).astype(np.uint64)), 31, path)
    chars, ends = mixed_reads(g, 78, 2000)
    exp = oracle_results(oracle_index(str(path), 8), chars, ends)
    assert np.array_equal(S.SbwtIndex.open(path).search_reads(chars, ends), exp)


def test_k_above_31_is_rejected(tmp_path):
    with pytest.raises(S.SbwtError):
        S.build_index([b"ACGT" * 20], 32, tmp_path / "x.sbwt")


@pytest.mark.parametrize("n,length,founders,k,rc", [(12, 3000, 3, 31, True),
                                                    (150, 800, 6, 31, True),
                                                    (3000, 120, 12, 21, False)])
def test_gpu_colored_builder_matches_host_builder(n, length, founders, k, rc, tmp_path):
    # sets of every kind: singletons, sparse lists, dense rows (n > 64)
    g = T.gen_genomes(n + k, n, length, founders, 0.01, 0.05, 0.001)
    hs, hc = tmp_path / "h.sbwt", tmp_path / "h.tcolors"
    ds, dc = tmp_path / "d.sbwt", tmp_path / "d.tcolors"
    nh = T.build_colored(g, k, str(hs), str(hc), add_rc=rc)
    nd = S.build_colored_index(g.chars, np.cumsum(g.lens).astype(np.uint64), k, ds, dc, rc)
    assert nd == nh
    assert ds.read_bytes() == hs.read_bytes()
    assert dc.read_bytes() == hc.read_bytes()
