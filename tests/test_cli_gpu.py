"""The reference-compatible CLI (`sbwt_search index|colors`) end to end on
the GPU: the reference's own index fixtures reproduce byte for byte, and the
colors step matches the oracle."""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle as O
import sbwt_b200 as S
import sbwt_tools as T
from helpers import FIXTURE_FILES, GOLDEN, TMP, golden_sbwt_path, oracle_index

pytestmark = pytest.mark.gpu
CLI = str(S.HERE / "_build" / "sbwt_search")


def run(*args, env=None):
    r = subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def decode_index_file(path, mode):
    b = path.read_bytes()
    if mode == "ascii":
        return O.read_ascii_index_results(path)
    off = 0
    for _ in range(2):
        n = struct.unpack_from("<Q", b, off)[0]
        off += 8 + n
    rows, cur = [], []
    if mode == "binary":
        for v in np.frombuffer(b[off:], np.uint64).tolist():
            if v == (1 << 64) - 3:
                rows.append(cur)
                cur = []
            else:
                cur.append(-1 if v == O.NOT_FOUND else (-2 if v == O.INVALID else v))
        return rows
    for line in b[off:].split(b"\n")[:-1]:
        rows.append([{"0": 0, "1": -1, "2": -2}[chr(c)] for c in line])
    return rows


@pytest.mark.parametrize("piece", [None, "1"])
@pytest.mark.parametrize("mode", ["ascii", "binary", "bool"])
def test_index_cli_on_reference_fixtures(mode, piece, tmp_path):
    """piece "1": every query file is larger than the device piece, so the
    CLI parses it on the host in batches and searches and formats each batch
    on the device; None: whole files go to the device as they are read."""
    ins = tmp_path / "in.list"
    outs = tmp_path / "out.list"
    ins.write_text("\n".join(str(GOLDEN / "index_search" / n) for n in FIXTURE_FILES) + "\n")
    outs.write_text("\n".join(str(tmp_path / n.split(".")[0]) for n in FIXTURE_FILES) + "\n")
    env = None
    if piece is not None:
        env = dict(os.environ, SBWT_CLI_DEVICE_PIECE_BYTES=piece)
    run("index", "-i", golden_sbwt_path(), "-q", ins, "-o", outs, "-p", mode, env=env)
    ext = {"ascii": ".txt", "binary": ".bin", "bool": ".bool"}[mode]
    for n in FIXTURE_FILES:
        stem = n.split(".")[0]
        exp_path = GOLDEN / "index_search" / "expected" / (stem + ".txt")
        got_path = tmp_path / (stem + ext)
        if mode == "ascii":
            assert got_path.read_bytes() == exp_path.read_bytes()
        else:
            exp = O.read_ascii_index_results(exp_path)
            got = decode_index_file(got_path, mode)
            if mode == "bool":  # bool keeps found / not-found / invalid only
                exp = [[0 if t >= 0 else t for t in row] for row in exp]
            assert got == exp


def test_index_cli_missing_flag_prints_help():
    r = subprocess.run([CLI, "index", "-q", "x"], capture_output=True, text=True)
    assert r.returncode == 1 and "Missing option" in r.stdout


def test_colors_cli_matches_oracle(tmp_path):
    g = T.gen_genomes(21, 40, 2000, 4, 0.01, 0.05, 0.0)
    sp, cp = tmp_path / "c.sbwt", tmp_path / "c.tcolors"
    T.build_colored(g, 31, str(sp), str(cp))
    chars, ends = T.gen_reads(22, g, 300, 0.9, 100, 0.4, 20, 300, 0.01, 0.005)
    reads = T.split_reads(chars, ends)
    fq = tmp_path / "q.fna"
    fq.write_bytes(b"".join(b">r%d\n%s\n" % (i, r) for i, r in enumerate(reads)))
    run("index", "-i", sp, "-q", fq, "-o", tmp_path / "idx")
    for mode, ext in (("ascii", ".txt"), ("csv", ".csv"), ("binary", ".bin")):
        run("colors", "-k", cp, "-q", tmp_path / "idx.txt", "-o", tmp_path / ("col_" + mode),
            "-p", mode, "-t", "0.7")
    oi = oracle_index(str(sp), 8)
    per = O.index_search_reads(oi, reads)
    found = [p[p < O.INVALID] for p in per]
    oc = O.OracleColors(O.ColorsFile.read(cp))
    exp = oc.pseudoalign(found, [0] * len(per), [0] * len(per), 0.7)
    body = (tmp_path / "col_ascii.txt").read_bytes()[8 + 5 + 8 + 4:].decode()
    got = [[int(t) for t in ln.split()] for ln in body.split("\n")[:-1]]
    assert got == exp
    csv = (tmp_path / "col_csv.csv").read_text().split("\n")[:-1]
    assert csv[0] == ",".join(str(i) for i in range(1, 41))
    assert [[i for i, x in enumerate(row.split(",")) if x == "1"] for row in csv[1:]] == exp
