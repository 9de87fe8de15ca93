"""Builds the library in-tree (no JIT cache): everything lands in _build/.

  _build/libsbwt_b200.so   CUDA kernels (sm_100a) + host C++ + the C ABI
  _build/libsbwt_tools.so  index construction + synthetic data tools (host)
  _build/sbwt_search       the reference-compatible CLI (index | colors)

Run `python sbwt-search_b200/build.py` (or __graft_entry__.build()).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
OUT = HERE / "_build"
CSRC = HERE / "csrc"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-I", str(REPO / "include")]

LIB_SOURCES = ["index.cu", "colors.cu", "measure.cu", "pipeline.cu", "fastx_device.cu", "format_device.cu", "build_device.cu", "kmer_table.cu",
               "capi.cpp", "colors_host.cpp", "formats.cpp", "fastx.cpp", "results_io.cpp"]
CLI_SOURCES = ["cli_main.cpp"]
TOOLS_SOURCES = ["tools/sbwt_build.cpp", "formats.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(Path(d).stat().st_mtime <= t for d in deps)


def _headers():
    return list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + \
        [REPO / "include" / "sbwt_b200.h", Path(__file__)]


def _obj(src: str, verbose: bool = False) -> Path:
    s = CSRC / src
    o = OUT / "obj" / (src.replace("/", "_") + ".o")
    o.parent.mkdir(parents=True, exist_ok=True)
    if _newer(o, [s] + _headers()):
        return o
    if s.suffix == ".cu":
        cmd = [NVCC, *ARCH, "-lineinfo", *COMMON, "-ccbin", HOST_CXX,
               "-Xcompiler", "-fPIC", "-c", str(s), "-o", str(o)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = [HOST_CXX, *COMMON, "-fPIC", "-Wall", "-I", "/usr/local/cuda/include",
               "-c", str(s), "-o", str(o)]
    out = _run(cmd)
    if verbose and out:
        print(out)
    return o


def build(verbose: bool = False) -> None:
    OUT.mkdir(parents=True, exist_ok=True)
    srcs = [s for s in LIB_SOURCES if (CSRC / s).exists()]
    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(lambda s: _obj(s, verbose), srcs))
        cli_objs = list(ex.map(_obj, [s for s in CLI_SOURCES if (CSRC / s).exists()]))
    lib = OUT / "libsbwt_b200.so"
    if not _newer(lib, objs):
        _run([NVCC, *ARCH, "-shared", "-ccbin", HOST_CXX, *map(str, objs), "-o", str(lib),
              "-lz", "-Xlinker", "-soname=libsbwt_b200.so"])
    if cli_objs:
        cli = OUT / "sbwt_search"
        if not _newer(cli, cli_objs + [lib]):
            _run([HOST_CXX, *map(str, cli_objs), "-o", str(cli), "-L", str(OUT),
                  "-lsbwt_b200", f"-Wl,-rpath,{OUT}", "-Wl,-rpath,$ORIGIN",
                  "-L/usr/local/cuda/lib64", "-lcudart", "-lpthread"])
    tools = OUT / "libsbwt_tools.so"
    tsrc = [CSRC / s for s in TOOLS_SOURCES]
    if not _newer(tools, tsrc + _headers()):
        _run([HOST_CXX, "-std=c++17", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared",
              "-fPIC", "-Wall", *map(str, tsrc), "-o", str(tools)])


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", *sorted(p.name for p in OUT.iterdir() if p.is_file()))
