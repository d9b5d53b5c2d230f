"""C-ABI checks that need no GPU: the library loads and exports every entry
point declared in include/iblgf_b200.h; a context request without a usable
device fails with a status code, not an exception or a crash."""
import ctypes
import os
import re

import pytest

import iblgf_b200 as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "iblgf_b200.h")).read()
    return sorted(set(re.findall(r"\b(iblgf_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_binding_list():
    assert declared() == sorted(B.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = B.lib()
    for name in declared():
        assert hasattr(L, name), name


def test_create_without_device_reports_status():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(B.IblgfError):
        B.Solver((-24,) * 3, (48,) * 3, 6, 1.0, [((-24,) * 3, (48,) * 3)])


def test_null_config_is_rejected():
    h = ctypes.c_void_p()
    assert B.lib().iblgf_create(None, ctypes.byref(h)) == 1


def test_cpp_adapter_builds():
    """include/iblgf_b200/adapter.hpp (reference-style PoissonSolver<Setup>)
    compiles against a stand-in of the reference's domain types and links to
    the library."""
    import subprocess
    subprocess.run(["make", "-s", "-B", "-C", os.path.join(ROOT, "tests", "cpp")], check=True)
    assert os.path.exists(os.path.join(ROOT, "tests", "cpp", "adapter_mock"))
