"""The Julia shim's ccall argument lists and structs against the C header.

``particle_transport_b200/julia/PtB200.jl`` is how the reference's Julia
pipeline reaches the library; there is no Julia here to run it, so this test
reads it as text.  Every ``ccall`` must name an entry point declared in
``include/ptb200.h`` with the same number of arguments and the same kind of
each argument (pointer, 64-bit integer, 32-bit integer, double) and return
type, and the shim's ``PtGrid`` / ``PtPushParams`` must have the header
structs' fields in the same order with the same sizes and offsets.  The
ctypes binding used by the Python host is checked against the same
prototypes.  Runs without a GPU."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from particle_transport_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ptb200.h")
SHIM = os.path.join(ROOT, "particle_transport_b200", "julia", "PtB200.jl")


def _strip_c_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def _c_kind(param: str) -> str:
    p = param.strip()
    if "*" in p or "[" in p or p.startswith("pt_save_fn"):
        return "ptr"
    t = p.rsplit(None, 1)[0] if len(p.split()) > 1 else p
    t = t.replace("const ", "").strip()
    return {"int64_t": "i64", "uint64_t": "i64", "int": "i32", "int32_t": "i32", "double": "f64"}[t]


def header_prototypes():
    """name -> (return kind, [parameter kinds]) for every pt_* function."""
    text = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"(?:^|(?<=[;}]))\s*((?:const\s+)?(?:int|int64_t|char)\s*\*?)\s*(pt_\w+)\s*\(([^)]*)\)\s*(?=;)",
                         text):
        ret, name, params = m.group(1), m.group(2), m.group(3).strip()
        rk = "ptr" if "*" in ret else {"int": "i32", "int64_t": "i64"}[ret.strip()]
        kinds = [] if params in ("", "void") else [_c_kind(p) for p in params.split(",")]
        out[name] = (rk, kinds)
    return out


def _split_top(s: str):
    """Split on commas that are not inside (), {} or []."""
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    tail = "".join(cur).strip()
    if tail:
        parts.append(tail)
    return [p for p in parts if p]


def _balanced(text: str, start: int) -> str:
    """The contents of the parenthesis opened at text[start]."""
    assert text[start] == "("
    depth = 0
    for i in range(start, len(text)):
        depth += {"(": 1, ")": -1}.get(text[i], 0)
        if depth == 0:
            return text[start + 1:i]
    raise ValueError("unbalanced")


def _jl_kind(t: str) -> str:
    t = t.strip()
    if t.startswith(("Ptr{", "Ref{")) or t in ("Cstring", "Ptr"):
        return "ptr"
    return {"Int64": "i64", "UInt64": "i64", "Cint": "i32", "Int32": "i32", "Float64": "f64"}[t]


def shim_ccalls():
    """[(name, return kind, [argument kinds], number of argument values)]"""
    text = re.sub(r"#[^\n]*", "", open(SHIM).read())
    calls = []
    for m in re.finditer(r"ccall\(", text):
        body = _balanced(text, m.end() - 1)
        parts = _split_top(body)
        name = re.match(r"\(\s*:(\w+)\s*,", parts[0]).group(1)
        types = parts[2]
        assert types.startswith("(") and types.endswith(")"), types
        kinds = [_jl_kind(t) for t in _split_top(types[1:-1])]
        calls.append((name, _jl_kind(parts[1]), kinds, len(parts) - 3))
    return calls


def test_shim_ccalls_match_header():
    protos = header_prototypes()
    assert {"pt_push_run", "pt_dmumu_accumulate", "pt_dpp_accumulate", "pt_last_error"} <= set(protos)
    calls = shim_ccalls()
    names = {c[0] for c in calls}
    # the seams the shim replaces, plus the handle lifecycle
    assert {"pt_ctx_create", "pt_ctx_destroy", "pt_field_upload", "pt_field_destroy", "pt_push_run",
            "pt_dmumu_accumulate", "pt_dpp_accumulate", "pt_energy_snapshots", "pt_last_error"} <= names
    for name, rk, kinds, nvals in calls:
        assert name in protos, f"{name} is not declared in the header"
        hret, hkinds = protos[name]
        assert rk == hret, (name, rk, hret)
        assert kinds == hkinds, (name, kinds, hkinds)
        assert nvals == len(kinds), (name, nvals, len(kinds))


def test_ctypes_signatures_match_header():
    protos = header_prototypes()
    L = _lib.load()

    def kind(t):
        if t in (C.c_int64, C.c_uint64):
            return "i64"
        if t in (C.c_int, C.c_int32):
            return "i32"
        if t is C.c_double:
            return "f64"
        return "ptr"

    assert set(protos) == set(_lib.EXPORTS)
    for name, (hret, hkinds) in protos.items():
        f = getattr(L, name)
        assert [kind(t) for t in (f.argtypes or [])] == hkinds, name
        assert kind(f.restype) == hret, name


_JL_SIZES = {"Int64": 8, "UInt64": 8, "Float64": 8, "Int32": 4, "Cint": 4}


def shim_struct(name):
    text = open(SHIM).read()
    body = re.search(r"struct\s+%s\s*\n(.*?)\nend" % name, text, re.S).group(1)
    fields = []
    for line in body.splitlines():
        for item in line.split(";"):
            m = re.match(r"\s*(\w+)::(\w+)\s*$", item)
            if m:
                fields.append((m.group(1), m.group(2)))
    off, out = 0, []
    for fname, jt in fields:  # Julia isbits structs use the C layout: natural alignment
        sz = _JL_SIZES[jt]
        off = (off + sz - 1) // sz * sz
        out.append((fname, off, sz))
        off += sz
    return out, (off + 7) // 8 * 8


def c_struct_layout(tmp_path, cname, fields):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ptb200.h"', "int main(void) {",
             f'    printf("sizeof %zu\\n", sizeof({cname}));']
    for f in fields:
        lines.append(f'    printf("{f} %zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname}*)0)->{f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / f"{cname}.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / cname
    subprocess.run([cc, "-std=c99", "-I" + os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    size = int(out[0].split()[1])
    return [(l.split()[0], int(l.split()[1]), int(l.split()[2])) for l in out[1:] if l.strip()], size


@pytest.mark.parametrize("jl, cname, ct", [("PtGrid", "pt_grid", _lib.Grid),
                                            ("PtPushParams", "pt_push_params", _lib.PushParams)])
def test_shim_structs_match_header(tmp_path, jl, cname, ct):
    jfields, jsize = shim_struct(jl)
    cfields, csize = c_struct_layout(tmp_path, cname, [f for f, _, _ in jfields])
    assert jfields == cfields and jsize == csize, (jfields, cfields, jsize, csize)
    assert C.sizeof(ct) == csize
    assert [(f, getattr(ct, f).offset, getattr(ct, f).size) for f, _ in ct._fields_] == cfields
