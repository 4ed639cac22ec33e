"""CPU: the C-ABI library loads and exports every entry point its header
declares (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "wmd_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(wmd_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_drop_in_entry_points():
    names = declared_functions()
    for n in ("wmd_sinkhorn_fused", "wmd_sinkhorn_nonfused",
              "wmd_sinkhorn_fused_csc", "wmd_sinkhorn_nonfused_csc"):
        assert n in names


def test_library_exports_every_declared_symbol(wmd):
    lib = ctypes.CDLL(wmd.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert sorted(wmd.exported_names()) == declared_functions()


def test_abi_version_and_status_strings(wmd):
    L = wmd.lib()
    assert L.wmd_abi_version() == 1
    assert L.wmd_status_string(0) == b"ok"
    assert L.wmd_status_string(2) == b"invalid input data"


def test_struct_layout_mirrors_reference_csr_csc(wmd):
    # puma_csr_double_t / puma_csc_double_t (common.h:38-57): three u64
    # counts followed by three pointers.
    assert ctypes.sizeof(wmd.CSR) == 6 * 8
    assert ctypes.sizeof(wmd.CSC) == 6 * 8
    assert [f[0] for f in wmd.CSR._fields_] == [
        "num_rows", "num_cols", "nnz", "row_ptr", "col_inds", "vals"]
    assert [f[0] for f in wmd.CSC._fields_] == [
        "num_rows", "num_cols", "nnz", "col_ptr", "row_inds", "vals"]


def test_null_arguments_rejected_before_any_device_work(wmd):
    L = wmd.lib()
    st = L.wmd_sinkhorn_fused(None, None, None, -10.0, 15, 10, 10, 300, None)
    assert st == 1  # WMD_ERR_INVALID_ARG
    assert b"null" in L.wmd_last_error()
    st = L.wmd_sinkhorn_nonfused_csc(None, None, None, 10.0, 15, 10, 10, 300, None)
    assert st == 1


def test_create_without_device_reports_no_device(wmd):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert wmd.lib().wmd_create(ctypes.byref(h), 0) == 5  # WMD_ERR_NO_DEVICE
