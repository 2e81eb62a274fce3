"""The C ABI library: it loads, and exports every entry point include/*.h declares (CPU only)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def declared():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^\s*(?:int|void|const char|double)\s*\*?\s*(sci_cuda_\w+)\s*\(",
                                header.read_text(), re.M))
    return names


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(ROOT / "libsci_b200" / "libsci_cuda.so"))
    names = declared()
    assert {"sci_cuda_open", "sci_cuda_execute", "sci_cuda_reduce"} <= names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_open_without_a_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        return
    from libsci_b200.native import DEVICE, lib

    handle = ctypes.c_void_p()
    assert lib.sci_cuda_open(0, ctypes.byref(handle)) == DEVICE
    assert not handle.value


def test_the_product_path_refuses_to_import_without_the_library(tmp_path, monkeypatch):
    """native.py raises instead of falling back when libsci_cuda.so is absent."""
    import importlib

    import libsci_b200.native as native

    monkeypatch.setattr(native, "LIBRARY", tmp_path / "missing.so")
    try:
        native._load()
    except ImportError as error:
        assert "not built" in str(error)
    else:
        raise AssertionError("loading a missing library did not raise")
    importlib.reload(native)
