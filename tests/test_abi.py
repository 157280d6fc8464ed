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


def test_header_is_plain_c(tmp_path):
    """A C host (Julia's ccall, cgo, ctypes) sees the header as C: it compiles
    as pedantic C99, and the structs the host fills keep their field names."""
    import shutil
    import subprocess

    import pytest

    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "use_header.c"
    src.write_text('#include "ptb200.h"\n'
                   "int main(void) {\n"
                   "    pt_campaign_desc d = {0};\n"
                   "    pt_push_params p = {0};\n"
                   "    d.sort_every = 2; d.n_mom = 1; p.sort_every = 64;\n"
                   "    return PT_FIELD_BRICK_F64 - 4 + (int)(d.sort_every - 2) + (int)(p.sort_every - 64);\n"
                   "}\n")
    out = subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                          "-I" + os.path.dirname(HEADER), "-c", str(src), "-o", str(tmp_path / "use_header.o")],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
