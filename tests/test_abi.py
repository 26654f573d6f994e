"""The C-ABI library loads and exports every entry point include/gpl.h declares (no GPU work)."""
import ctypes
import os
import re

import pytest

from gaspacho2_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^GPL_API\s+[\w\s\*]+?\b(gpl_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared()
    assert "gpl_create" in names and "gpl_evaluate" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_signatures_cover_the_header():
    assert set(declared()) <= set(_lib.SIGNATURES), set(declared()) - set(_lib.SIGNATURES)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.GplError):
        _lib.load()


def test_error_codes_without_device():
    """Argument checks run before any device work, so they answer without a GPU."""
    L = _lib.load()
    assert L.gpl_create(None, 0, None) == -1
