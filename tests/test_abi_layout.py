"""The ctypes mirror of the C ABI's structs (cudaplasticity_b200/_capi.py)
against the C compiler's layout of include/cuplast.h: every field at the
same offset, every struct the same size. A mismatch would corrupt options
and reports silently, so it is checked on the CPU with gcc."""
import ctypes
import os
import shutil
import subprocess

import pytest

from cudaplasticity_b200 import _capi as C

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = ["cp_material", "cp_mesh_view", "cp_solve_opts", "cp_solve_report", "cp_batch_opts", "cp_server_opts",
           "cp_server_stats"]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cuplast.h"', 'int main(void) {']
    for s in STRUCTS:
        lines.append(f'printf("{s} size %zu\\n", sizeof({s}));')
        for name, _ in getattr(C, s)._fields_:
            lines.append(f'printf("{s} {name} %zu\\n", offsetof({s}, {name}));')
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            s, k, v = ln.split()
            got[(s, k)] = int(v)
    for s in STRUCTS:
        cls = getattr(C, s)
        assert got[(s, "size")] == ctypes.sizeof(cls), s
        for name, _ in cls._fields_:
            assert got[(s, name)] == getattr(cls, name).offset, (s, name)


def test_every_c_field_is_mirrored():
    """The field names of each struct in the header, in order, are the
    ctypes mirror's (read from the header text)."""
    import re

    text = open(os.path.join(ROOT, "include", "cuplast.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    for s in STRUCTS:
        m = re.search(r"typedef struct\s*(?:\w+\s*)?\{([^{}]*)\}\s*" + s + r"\s*;", text)
        assert m, s
        names = []
        for decl in m.group(1).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            body = re.sub(r"^(const\s+)?[\w\s]+?(\*+\s*|\s+)(?=\w+\s*(\[|,|$))", "", decl, count=1)
            for part in body.split(","):
                nm = re.sub(r"\[.*?\]", "", part).strip().lstrip("*").strip()
                if nm:
                    names.append(nm)
        assert names == [n for n, _ in getattr(C, s)._fields_], (s, names)
