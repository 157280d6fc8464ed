"""The C-ABI library loads and exports every entry point declared in
include/ptb200.h (no device calls: runs without a GPU)."""
import os
import re

from particle_transport_b200 import _lib, build

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "ptb200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(pt_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared()
    assert "pt_push_run" in names and "pt_dmumu_accumulate" in names
    assert set(names) == set(_lib.EXPORTS), set(names) ^ set(_lib.EXPORTS)


def test_library_builds_and_exports_every_symbol():
    path = build.build()
    assert os.path.exists(path)
    L = _lib.load()
    for name in declared():
        assert hasattr(L, name), name
    assert L.pt_version() == 1


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    pkg = os.path.dirname(_lib.__file__)
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                src = open(os.path.join(root, f)).read()
                assert "import oracle" not in src and "from oracle" not in src, f
                assert "libptoracle" not in src, f
