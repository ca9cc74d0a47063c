"""The C-ABI library loads and exports every symbol include/emagddm_b200.h
declares (no device work)."""
import ctypes as C
import os
import re

from emagddm_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "emagddm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(emg_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = C.CDLL(_abi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) == set(_abi.SIGNATURES)


def test_version_and_error_string():
    L = _abi.lib()
    assert L.emg_abi_version() == 1
    assert isinstance(L.emg_last_error(), bytes)
