"""FASTA/FASTQ parsing on the GPU (sbwt_fastx_parse) against the host reader
(sbwt_fastx_read, pinned to the reference's fixtures): identical chars and
read ends on the fixtures, on seeded adversarial text and on layouts that put
1024-line chunk boundaries inside sequences and qualities."""
import ctypes as C

import numpy as np
import pytest

import sbwt_b200 as S
from helpers import FIXTURE_FILES, GOLDEN, host_fastx, random_fastx

pytestmark = pytest.mark.gpu


def check_same(text, tmp_path):
    hc, he = host_fastx(text, tmp_path / "in.fx")
    dc, de = S.fastx_parse(text)
    assert dc.tobytes() == hc
    assert de.tolist() == he.tolist()
    return len(he)


@pytest.mark.parametrize("name", FIXTURE_FILES)
def test_fixtures(name, tmp_path):
    check_same((GOLDEN / "index_search" / name).read_bytes(), tmp_path)


@pytest.mark.parametrize("seed", range(8))
def test_random_text(seed, tmp_path):
    # ~10-40 k lines: many chunks, boundaries anywhere in the records
    text = random_fastx(100 + seed, 4000, fastq_frac=[0.0, 0.5, 1.0, 0.8][seed % 4],
                        max_line=[80, 7, 200, 3][seed % 4], final_newline=seed % 3 != 0)
    assert check_same(text, tmp_path) > 0


def test_edge_cases(tmp_path):
    cases = [b"", b"\n", b">", b">\n", b"@\n", b"ACGT\n", b">a\nAC\r\nGT\r",
             b">a\r\nAC\r\nGT\n>b\n>c\nTT\n\n@q x\nACG\nT\n+\nII\nII\n@r\n\n+\n\n",
             b"@a\nACGT\n+\n@@\n", b"@a\nACGT\n+\n@@@@\n@b\nA\n+\n>\n",
             b"@a\nAC\n+\nII", b"\r\n\r\n>x\r\n\r\nA\r\n", b"+\n@a\n+\n+\n"]
    for t in cases:
        check_same(t, tmp_path)


def test_long_fasta_records_across_chunks(tmp_path):
    # 3 records of 6000 lines each: whole chunks inside one sequence
    rng = np.random.default_rng(7)
    parts = []
    for r in range(3):
        parts.append(b">chr%d\n" % r)
        body = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 60 * 6000))
        parts += [body[i:i + 60] + b"\n" for i in range(0, len(body), 60)]
    assert check_same(b"".join(parts), tmp_path) == 3


def test_fastq_shifted_by_a_junk_line(tmp_path):
    # 4-line records after one junk line: every chunk starts inside a record
    rng = np.random.default_rng(8)
    lines = [b"junk"]
    for r in range(3000):
        s = bytes(rng.choice(np.frombuffer(b"ACGT", np.uint8), 100))
        q = b"@" + bytes(rng.choice(np.frombuffer(b"I@+>", np.uint8), 99))
        lines += [b"@q%d" % r, s, b"+", q]
    assert check_same(b"\n".join(lines) + b"\n", tmp_path) == 3000


def test_device_pointers_and_capacity():
    import torch
    text = random_fastx(5, 500)
    hc, he = S.fastx_parse(text)
    d_text = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    d_chars = torch.zeros(len(text), dtype=torch.uint8, device="cuda")
    d_ends = torch.zeros(len(he), dtype=torch.int64, device="cuda")
    nc, nr = C.c_uint64(), C.c_uint64()
    L = S.lib()
    rc = L.sbwt_fastx_parse(d_text.data_ptr(), len(text), d_chars.data_ptr(), len(text),
                            d_ends.data_ptr(), len(he) - 1, C.byref(nc), C.byref(nr),
                            S.DEVICE_POINTERS, 0, torch.cuda.current_stream().cuda_stream)
    assert rc == S.E_CAPACITY and nr.value == len(he) and nc.value == len(hc)
    S.check(L.sbwt_fastx_parse(d_text.data_ptr(), len(text), d_chars.data_ptr(), len(text),
                               d_ends.data_ptr(), len(he), C.byref(nc), C.byref(nr),
                               S.DEVICE_POINTERS, 0, torch.cuda.current_stream().cuda_stream))
    assert d_chars[:nc.value].cpu().numpy().tobytes() == hc.tobytes()
    assert d_ends.cpu().numpy().view(np.uint64).tolist() == he.tolist()
