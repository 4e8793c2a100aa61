"""The C-ABI library: it loads without a GPU and exports every entry point the header declares."""

import os
import re

import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "nebula_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"NB_API\s+[\w\s\*]+?\b(nb_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared()
    assert "nb_block_advance" in names and "nb_find_neighbours" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    import ctypes

    from blackhole_nebula_simulator_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libnebula_b200.so not built")
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, f"not exported: {missing}"
    assert L.nb_version() == 1
    # the Python binding declares a signature for every header entry point
    assert set(_declared()) == set(_lib.EXPORTED)


def test_struct_mirrors_match_the_library():
    """nb_state and nb_params as the ctypes binding lays them out are the library's own."""
    import ctypes

    from blackhole_nebula_simulator_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libnebula_b200.so not built")
    L = _lib.lib()
    assert ctypes.sizeof(_lib.NbState) == L.nb_state_size()
    assert ctypes.sizeof(_lib.NbParams) == L.nb_params_size()


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "blackhole_nebula_simulator_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                text = open(os.path.join(dirpath, f)).read()
                assert not re.search(r"^\s*(from|import)\s+oracle", text, re.M), f
