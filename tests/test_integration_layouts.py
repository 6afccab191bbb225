"""The Java FFM struct layouts written out in INTEGRATION.md against the C
structs of include/vrgpu.h (through their ctypes mirrors, which every GPU
call uses): the same size and every named field at the same offset, so a
maintainer who copies the Java gets the ABI the library reads."""
import ctypes as C
import os
import re

import pytest

from vecruntime_b200 import native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MIRRORS = {"COLUMN_TYPE": N.ColumnType, "DICTIONARY": N.Dictionary, "COLUMN": N.Column, "TERM": N.Term,
           "AGG_FN": N.AggFn, "SPEC": N.AggSpec, "BATCH": N.Batch, "OUT_COLUMN": N.OutColumn, "PQ_PAGE": N.PqPage}
SIZES = {"JAVA_INT": 4, "JAVA_LONG": 8, "ADDRESS": 8}


def java_layouts():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    out = {}
    for name, body in re.findall(r"StructLayout (\w+) = MemoryLayout\.structLayout\((.*?)\);", text, re.S):
        fields, off = {}, 0
        for m in re.finditer(r"(JAVA_INT|JAVA_LONG|ADDRESS)\.withName\(\"(\w+)\"\)|paddingLayout\((\d+)\)|"
                             r"sequenceLayout\((\d+), (\w+)\)\.withName\(\"(\w+)\"\)", body):
            if m.group(1):
                size = SIZES[m.group(1)]
                assert off % size == 0, f"{name}.{m.group(2)} is not naturally aligned at {off}"
                fields[m.group(2)] = off
                off += size
            elif m.group(3):
                off += int(m.group(3))
            else:
                inner = out[m.group(5)]
                fields[m.group(6)] = off
                off += int(m.group(4)) * inner[1]
        out[name] = (fields, off)
    return out


@pytest.mark.parametrize("name", sorted(MIRRORS))
def test_java_layout_matches_the_c_struct(name):
    layouts = java_layouts()
    assert name in layouts, f"INTEGRATION.md has no {name} layout"
    fields, size = layouts[name]
    mirror = MIRRORS[name]
    assert size == C.sizeof(mirror), (name, size, C.sizeof(mirror))
    c_fields = {f[0]: getattr(mirror, f[0]).offset for f in mirror._fields_}
    assert fields == c_fields, (name, fields, c_fields)


C_NAMES = {"COLUMN_TYPE": "vr_column_type", "DICTIONARY": "vr_dictionary", "COLUMN": "vr_column", "TERM": "vr_term",
           "AGG_FN": "vr_agg_fn", "SPEC": "vr_agg_spec", "BATCH": "vr_batch", "OUT_COLUMN": "vr_out_column",
           "PQ_PAGE": "vr_pq_page"}


def test_ctypes_mirrors_match_the_header(tmp_path):
    """The ctypes mirrors against the header itself, compiled with gcc:
    sizeof and offsetof of every field."""
    import shutil
    import subprocess

    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vrgpu.h"', "int main(void) {"]
    for key, cname in C_NAMES.items():
        lines.append(f'printf("{key} @sizeof %zu\\n", sizeof({cname}));')
        for f in MIRRORS[key]._fields_:
            lines.append(f'printf("{key} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for ln in filter(None, out):
        key, field, value = ln.split()
        mirror = MIRRORS[key]
        want = C.sizeof(mirror) if field == "@sizeof" else getattr(mirror, field).offset
        assert int(value) == want, (key, field, value, want)
