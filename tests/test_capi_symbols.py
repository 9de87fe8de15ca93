"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls are made here)."""
import ctypes
import re
from pathlib import Path

import sbwt_b200 as S

REPO = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (REPO / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(sbwt_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_api():
    names = declared_functions()
    assert "sbwt_search_reads" in names and "sbwt_index_open" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(S.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_gpu():
    assert b"sm_100a" in S.lib().sbwt_version()
    h = ctypes.c_void_p()
    rc = S.lib().sbwt_index_open(None, None, 0, 0, ctypes.byref(h))
    assert rc == S.E_INVALID and S.lib().sbwt_last_error()


def test_table_kernel_mode_range_without_gpu():
    """Modes 0..19 set the read search kernel (no device call); 20 and above
    are SBWT_E_INVALID; a negative mode restores the default."""
    lib = S.lib()
    try:
        for mode in (0, 7, 17, 19):
            assert lib.sbwt_set_table_kernel(mode) == 0
        assert lib.sbwt_set_table_kernel(20) == S.E_INVALID
        assert b"0..19" in lib.sbwt_last_error()
    finally:
        assert lib.sbwt_set_table_kernel(-1) == 0
