"""The Fortran module include/mpgcr.f90 against the C header include/mpgcr.h, checked as text
(no Fortran compiler on these machines): every bind(C) derived type has the C struct's members in
the same order with the same offsets and total size (C layout rules; offsetof from a C compiler),
every entry point of the header has a bind(C) interface with the same name and argument count,
and the named constants equal the header's."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "mpgcr.f90")
HEADER = os.path.join(ROOT, "include", "mpgcr.h")

FSIZE = {"integer(c_int)": 4, "integer(c_int64_t)": 8, "real(c_double)": 8, "real(c_float)": 4,
         "type(c_ptr)": 8, "character(kind=c_char)": 1}


def fortran_types():
    """{type name: [(member, size, align, count)]} from the module's bind(C) types."""
    txt = open(F90).read()
    out = {}
    for name, body in re.findall(r"type, bind\(C\) :: (\w+)\n(.*?)end type", txt, re.S):
        members = []
        for line in body.splitlines():
            line = line.split("!")[0].strip()
            if not line:
                continue
            ftype, names = [x.strip() for x in line.split("::")]
            size = FSIZE[ftype]
            for m in re.findall(r"(\w+)(?:\((\d+)\))?", names):
                members.append((m[0], size, size, int(m[1]) if m[1] else 1))
        out[name] = members
    return out


def c_layout(tmp_path, types):
    lines = ['#include "mpgcr.h"', "#include <stdio.h>", "#include <stddef.h>", "int main(void){"]
    for t, members in types.items():
        lines.append(f'printf("{t} size %zu\\n", sizeof({t}));')
        for m, *_ in members:
            lines.append(f'printf("{t} {m} %zu\\n", offsetof({t}, {m}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    res = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        t, m, v = ln.split()
        res[(t, m)] = int(v)
    return res


def test_derived_types_match_c_structs(tmp_path):
    types = fortran_types()
    assert set(types) == {"mpg_params", "mpg_mesh_ref", "mpg_gcr_stats", "mpg_diag", "mpg_info", "mpg_ktime"}
    c = c_layout(tmp_path, types)
    for t, members in types.items():
        off = 0
        maxal = 1
        for m, size, align, count in members:
            off = (off + align - 1) // align * align
            assert c[(t, m)] == off, (t, m, c[(t, m)], off)
            off += size * count
            maxal = max(maxal, align)
        total = (off + maxal - 1) // maxal * maxal
        assert c[(t, "size")] == total, (t, c[(t, "size")], total)


def test_every_entry_point_has_an_interface():
    htxt = open(HEADER).read()
    decl = {}
    for m in re.finditer(r"^\s*(?:int|const char \*)\s*(mpg_\w+)\s*\(([^)]*)\)", htxt, re.M):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        decl[m.group(1)] = len(args)
    ftxt = open(F90).read()
    iface = {}
    for m in re.finditer(r"function (mpg_\w+)\(([^)]*)\)\s*(?:&\s*)?bind\(C, name=\"(\w+)\"\)", ftxt):
        assert m.group(1) == m.group(3)
        iface[m.group(1)] = len([a for a in m.group(2).split(",") if a.strip()])
    assert set(iface) == set(decl)
    for name, n in decl.items():
        assert iface[name] == n, name


def test_named_constants_match_header():
    htxt = open(HEADER).read()
    hval = {k: int(v) for k, v in re.findall(r"#define\s+(MPG_\w+)\s+(-?\d+)\b", htxt)}
    hval.update({k: int(v) for k, v in re.findall(r"(MPG_F_\w+)\s*=\s*(\d+)", htxt)})
    ftxt = open(F90).read().replace("&\n", " ")
    fval = {k: int(v) for k, v in re.findall(r"(MPG_\w+)\s*=\s*(-?\d+)", ftxt)}
    assert len(fval) >= 30
    for k, v in fval.items():
        assert hval.get(k) == v, (k, v, hval.get(k))
