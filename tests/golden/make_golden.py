"""Copies SBWT-Search's own end-to-end fixtures into tests/golden/.

Run in a checkout that has the reference tree (default /root/reference):

    python tests/golden/make_golden.py [REFERENCE_ROOT]

What is copied (all small; the .sbwt is stored gzip-compressed):
  index_search/search_test_index.sbwt.gz  <- test_objects/search_test_index.sbwt
  index_search/{fasta1..4.fna,fastq1.fnq} <- test_objects/full_pipeline/index_search/
  index_search/expected/*.txt             <- .../index_search/expected/
  color_search/fasta{1..4}.indexes.txt    <- test_objects/full_pipeline/color_search/
  color_search/expected/*.colors.txt      <- .../color_search/expected/
These are the inputs and expected outputs of the reference's pipeline tests
(scripts/test/index_pipeline_test.sh:69-95, color_pipeline_test.sh:67-96).
The colors fixtures cannot be replayed (their .tcolors input is not shipped
with the reference); they are kept as inputs of the index-file parser tests.
"""
import gzip
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def main(ref_root: str = "/root/reference") -> None:
    src = Path(ref_root) / "test_objects"
    out = HERE / "index_search"
    (out / "expected").mkdir(parents=True, exist_ok=True)
    with open(src / "search_test_index.sbwt", "rb") as f_in:
        with gzip.GzipFile(out / "search_test_index.sbwt.gz", "wb", mtime=0) as f_out:
            shutil.copyfileobj(f_in, f_out)
    idx = src / "full_pipeline" / "index_search"
    for p in sorted(idx.iterdir()):
        if p.is_file() and p.suffix in (".fna", ".fnq"):
            shutil.copyfile(p, out / p.name)
    for p in sorted((idx / "expected").iterdir()):
        shutil.copyfile(p, out / "expected" / p.name)
    cout = HERE / "color_search"
    (cout / "expected").mkdir(parents=True, exist_ok=True)
    col = src / "full_pipeline" / "color_search"
    for p in sorted(col.iterdir()):
        if p.is_file() and p.name.endswith(".indexes.txt"):
            shutil.copyfile(p, cout / p.name)
    for p in sorted((col / "expected").iterdir()):
        shutil.copyfile(p, cout / "expected" / p.name)


if __name__ == "__main__":
    main(*sys.argv[1:])
