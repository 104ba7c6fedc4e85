"""The C-ABI library loads without a GPU and exports every symbol the header declares."""
import os
import re
import subprocess

import pytest

from conftest import ROOT


def header_symbols():
    src = open(os.path.join(ROOT, "include", "dftbaby_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dftb_\w+)\s*\(", src)))


def test_library_exports_header_symbols():
    from dftbaby_b200 import build, native
    build.build_native()
    out = subprocess.check_output(["nm", "-D", "--defined-only", native.LIB_PATH]).decode()
    exported = set(re.findall(r"\bT (dftb_\w+)", out))
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    assert set(native.exported_symbols()) == set(header_symbols())


def test_library_loads_and_answers_size_queries():
    from dftbaby_b200 import native
    L = native.load(require_cuda=False)
    assert b"sm_100a" in L.dftb_version()
    assert L.dftb_trans_charges_workspace_size(102, 51, 51) >= 8 * 102 * 102
    assert L.dftb_hermitian_rv_workspace_size(42, 10) >= 2 * 8 * 42 * 10
    assert L.dftb_apbv_workspace_size(42, 51, 51, 10) >= 8 * 42 * 51 * 51 * 10


def test_entry_points_reject_bad_sizes_without_touching_the_gpu():
    from dftbaby_b200 import native
    L = native.load(require_cuda=False)
    assert L.dftb_directional_cosines(0, None, None, None, None, None, None) == -1
    assert L.dftb_monopoles(10, 0, None, None, None, None, None, None, None) == -1
    assert L.dftb_trans_charges(10, 2, 3, 3, None, None, None, None, None, None, None, None, 0, None) == -2
    assert L.dftb_hermitian_rv(4, 2, 2, 1, None, None, None, None, None, None, 0, None) == -2
    assert b"null" in L.dftb_last_error()


def test_package_fails_loudly_without_cuda():
    import torch
    from dftbaby_b200 import native
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    with pytest.raises(native.NativeUnavailable):
        native.load()
