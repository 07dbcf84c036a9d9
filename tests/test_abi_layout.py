"""Descriptor layouts: every ctypes mirror in grico_b200/_lib.py has the C header's field
offsets and size (a small C program compiled with gcc prints offsetof/sizeof from
include/grico_b200.h), and the Julia mirrors in INTEGRATION.md list the same fields in the same
order, so a binding copied from there hands the library a complete struct."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

import grico_b200._lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = ["GricoCellBatchDesc", "GricoPointBatchDesc", "GricoPlanDesc", "GricoSolveOptions", "GricoSolveReport",
           "GricoTransferDesc", "GricoMGOptions", "GricoLearnedDesc"]


def _c_layout():
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "grico_b200.h"', "int main(void) {"]
    for name in STRUCTS:
        st = getattr(L, name)
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "layout.c")
        exe = os.path.join(tmp, "layout")
        with open(src, "w") as f:
            f.write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        s, f, v = line.split()
        table[(s, f)] = int(v)
    return table


@pytest.mark.parametrize("name", STRUCTS)
def test_ctypes_mirror_matches_header(name):
    table = _c_layout()
    st = getattr(L, name)
    assert C.sizeof(st) == table[(name, "sizeof")]
    for field, _ in st._fields_:
        assert getattr(st, field).offset == table[(name, field)], field


def _header_fields(name):
    text = open(os.path.join(ROOT, "include", "grico_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.search(r"(\w+)\s*(\[\s*\w+\s*\])?$", decl)
        names.append(m.group(1))
    return names


@pytest.mark.parametrize("c_name,julia_name", [("GricoCellBatchDesc", "CellBatchDesc"),
                                               ("GricoPointBatchDesc", "PointBatchDesc"),
                                               ("GricoPlanDesc", "PlanDesc")])
def test_julia_mirror_lists_every_field(c_name, julia_name):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    body = re.search(r"struct %s\s.*?\n(.*?)\nend" % julia_name, text, flags=re.S).group(1)
    fields = re.findall(r"(\w+)::", body)
    assert fields == _header_fields(c_name)
    assert fields == [f for f, _ in getattr(L, c_name)._fields_]
