"""The C-ABI library loads and exports every entry point that include/pdgpu.h declares (no GPU needed)."""
import os
import re

from conftest import ROOT


def declared_functions():
    with open(os.path.join(ROOT, "include", "pdgpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(pdg_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "pdg_fock_two_electron" in names and "pdg_scf_run" in names


def test_library_exports_every_declared_symbol():
    from pdynamo3_b200 import lib
    L = lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert set(declared_functions()) <= set(lib.EXPORTS) | set(declared_functions())


def test_version_and_error_string():
    from pdynamo3_b200 import lib
    L = lib.load()
    assert L.pdg_version() >= 100
    assert isinstance(L.pdg_last_error(), bytes)
