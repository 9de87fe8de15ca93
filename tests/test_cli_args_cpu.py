"""The command line's argument contract, checked without a GPU: usage and
help exit 1, a missing required flag prints the help and exits 1
(ArgumentParser.cpp:20-22 of the reference), and fractions outside [0, 1]
exit 1 with the reference's messages before any work
(IndexSearchArgumentParser.cpp:203-222, ColorSearchArgumentParser.cpp:202-235)."""
import subprocess

import pytest

import sbwt_b200 as S

CLI = str(S.HERE / "_build" / "sbwt_search")


def run(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)


def test_usage_without_or_with_unknown_command():
    for args in ((), ("bogus",)):
        r = run(*args)
        assert r.returncode == 1 and "Usage: sbwt_search" in r.stdout


@pytest.mark.parametrize("cmd", ["index", "colors"])
def test_help_exits_one(cmd):
    for flag in ("-h", "--help"):
        r = run(cmd, flag)
        assert r.returncode == 1 and f"Usage: sbwt_search {cmd}" in r.stdout


@pytest.mark.parametrize("cmd,required", [
    ("index", {"-q": "query-file", "-i": "index-file", "-o": "output-prefix"}),
    ("colors", {"-q": "query-file", "-k": "colors-file", "-o": "output-prefix"}),
])
def test_missing_required_flag_prints_help(cmd, required):
    for left_out, name in required.items():
        args = [x for f in required if f != left_out for x in (f, "x")]
        r = run(cmd, *args)
        assert r.returncode == 1, (left_out, r.returncode)
        assert f"Missing option: {name}" in r.stdout and "Usage:" in r.stdout


@pytest.mark.parametrize("cmd,base", [
    ("index", ["-q", "none.fq", "-i", "none.sbwt", "-o", "out"]),
    ("colors", ["-q", "none.txt", "-k", "none.tcolors", "-o", "out"]),
])
@pytest.mark.parametrize("flag,name", [("-c", "cpu-memory-percentage"),
                                       ("-g", "gpu-memory-percentage")])
def test_memory_fraction_out_of_range(cmd, base, flag, name):
    for value in ("1.5", "-0.1", "abc"):
        r = run(cmd, *base, flag, value)
        assert r.returncode == 1
        assert f"Invalid value for {name}. Must be between 0 and 1." in r.stderr


def test_threshold_out_of_range():
    base = ["-q", "none.txt", "-k", "none.tcolors", "-o", "out"]
    for value in ("1.01", "-1", "x"):
        r = run("colors", *base, "-t", value)
        assert r.returncode == 1
        assert "Invalid value for threshold, must be between 1 and 0 (both included)" in r.stderr


@pytest.mark.parametrize("cmd,index_flag,index_name", [("index", "-i", "none.sbwt"),
                                                       ("colors", "-k", "none.tcolors")])
def test_list_pairing_follows_the_query_name(tmp_path, cmd, index_flag, index_name):
    """A query name ending in .list makes both the query and the output file
    lists of names (whatever the output's name); lists of different lengths
    are an error before anything is opened (FilenamesParser.cpp:19-37 and
    IndexSearchMain.cpp:405-407 of the reference)."""
    q = tmp_path / "queries.list"
    q.write_text("a.fq\nb.fq\n")
    one = tmp_path / "outputs.txt"
    one.write_text("out_a\n")
    two = tmp_path / "outputs2.txt"
    two.write_text("out_a\nout_b\n")
    missing_index = str(tmp_path / index_name)
    r = run(cmd, "-q", str(q), "-o", str(one), index_flag, missing_index)
    assert r.returncode != 0 and "Input and output file sizes differ" in r.stderr
    # equal lengths: the pairing passes and the missing index is the error
    r = run(cmd, "-q", str(q), "-o", str(two), index_flag, missing_index)
    assert r.returncode != 0 and "Unable to open file" in r.stderr and index_name in r.stderr
    # a single query: an output name ending in .list is one name, not read
    r = run(cmd, "-q", str(tmp_path / "a.fq"), "-o", str(tmp_path / "nothere.list"),
            index_flag, missing_index)
    assert r.returncode != 0 and index_name in r.stderr and "nothere.list" not in r.stderr
    # a query list that cannot be read
    r = run(cmd, "-q", str(tmp_path / "absent.list"), "-o", str(two), index_flag, missing_index)
    assert r.returncode != 0 and "absent.list" in r.stderr


@pytest.mark.parametrize("cmd,base", [
    ("index", ["-q", "none.fq", "-i", "none.sbwt", "-o", "out"]),
    ("colors", ["-q", "none.txt", "-k", "none.tcolors", "-o", "out"]),
])
def test_unknown_print_mode(cmd, base):
    """(IndexSearchMain.cpp:213-222, ColorSearchMain.cpp:205-214 of the reference)"""
    r = run(cmd, *base, "-p", "fasta")
    assert r.returncode != 0
    assert "Invalid value passed by user for argument print_mode" in r.stderr
