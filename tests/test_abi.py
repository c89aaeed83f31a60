"""The C ABI library loads (no GPU needed) and exports every entry point include/grabnes_gpu.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grabnes_gpu.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gbn_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "gbn_lanczos" in names and "gbn_cf_dos" in names and len(names) >= 20


def test_library_exports_every_declared_symbol():
    import grabnes_b200 as G
    lib = ctypes.CDLL(G.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared()) == set(G.EXPORTS)


def test_version_string_without_gpu():
    import grabnes_b200 as G
    assert "sm_100a" in G.version()


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import grabnes_b200 as G
    with pytest.raises(G.GbnError):
        G.Context(0)
