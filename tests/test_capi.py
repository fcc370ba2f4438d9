"""CPU checks of the C-ABI library: it loads and exports every entry point
declared in include/tblite_b200.h (no compute calls without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tblite_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("tb_calculator_create", "tb_singlepoint_batch", "tb_batch_run", "tb_sygvd_batch",
                     "tb_get_hamiltonian", "tb_adjacency_list", "tb_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from tblite_b200 import capi
    if not os.path.exists(capi.LIB_PATH):
        pytest.fail(f"CUDA library not built: {capi.LIB_PATH}")
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(capi.EXPORTS) <= set(declared_functions())


def test_library_has_no_cpu_oracle_dependency():
    from tblite_b200 import capi
    data = open(capi.LIB_PATH, "rb").read()
    assert b"orc_singlepoint" not in data and b"liboracle" not in data


def test_params_file_errors_are_reported(tmp_path):
    # parsing happens before any device call; a bad file must fail with TB_PARAM_ERROR
    from tblite_b200 import capi
    bad = tmp_path / "bad.tbp"
    bad.write_text("format tblite-b200-params 1\nelement H 1\n  shell 7 3\n")
    lib = capi.load_library()
    h = ctypes.c_void_p()
    st = lib.tb_calculator_create(str(bad).encode(), ctypes.byref(h))
    assert st == capi.TB_PARAM_ERROR
    assert "unsupported shell" in capi.last_error()


def test_checked_build_exports_and_reports_itself():
    """The checked build (index guards, -DTB_BOUNDS_CHECK) exports the same
    boundary and says it is the checked build; the normal build says it is not."""
    from tblite_b200 import capi
    if not os.path.exists(capi.LIB_CHECK_PATH):
        pytest.fail(f"checked library not built: {capi.LIB_CHECK_PATH}")
    chk = ctypes.CDLL(capi.LIB_CHECK_PATH)
    missing = [n for n in declared_functions() if not hasattr(chk, n)]
    assert not missing, missing
    assert chk.tb_bounds_check_build() == 1
    assert ctypes.CDLL(capi.LIB_PATH).tb_bounds_check_build() == 0
