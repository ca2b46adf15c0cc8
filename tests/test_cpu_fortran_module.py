"""The Fortran host's ISO_C_BINDING module (include/mrlbm_gpu.f90) against the C header.

No Fortran compiler exists in this image, so the module is checked statically: the components
of its bind(c) types must sit at the offsets the C compiler gives the struct fields of
include/mrlbm.h (bind(c) types follow the C layout rules), every interface must name a
function the header declares, with the same number of arguments, and the built library must
export it.  The module is what a Fortran host of the reference (2d_mrlbm.f90:229-535) would
`use` to call the step.
"""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "mrlbm_gpu.f90")
HDR = os.path.join(ROOT, "include", "mrlbm.h")
SIZES = {"real(c_double)": 8, "integer(c_int64_t)": 8, "integer(c_int32_t)": 4, "integer(c_int)": 4}


def _strip_comments(text):
    return "\n".join(line.split("!")[0] for line in text.splitlines())


def fortran_types():
    src = _strip_comments(open(F90).read())
    types = {}
    for m in re.finditer(r"type\s*,\s*bind\(c\)\s*::\s*(\w+)(.*?)end type", src, re.S | re.I):
        fields = []
        for line in m.group(2).splitlines():
            mm = re.match(r"\s*(real\(c_double\)|integer\(c_int64_t\)|integer\(c_int32_t\)|integer\(c_int\))\s*::\s*(\w+)\s*$",
                          line, re.I)
            if mm:
                fields.append((mm.group(2), SIZES[mm.group(1).lower()]))
            elif line.strip():
                raise AssertionError(f"unparsed component line: {line!r}")
        types[m.group(1)] = fields
    return types


def c_layout(fields):
    off, out, align = 0, {}, 1
    for name, size in fields:
        off = (off + size - 1) // size * size
        out[name] = off
        off += size
        align = max(align, size)
    return out, (off + align - 1) // align * align


def c_offsets(tmp_path, struct, names):
    prog = tmp_path / "off.c"
    lines = [f'printf("{n} %zu\\n", offsetof({struct}, {n}));' for n in names]
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "mrlbm.h"\nint main(void){\n' +
                    "\n".join(lines) + f'\nprintf("sizeof %zu\\n", sizeof({struct}));\nreturn 0;}}\n')
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.parametrize("name", ["mrlbm_config", "mrlbm_geometry_info"])
def test_bind_c_types_match_the_c_structs(tmp_path, name):
    fields = fortran_types()[name]
    f_off, f_size = c_layout(fields)
    c = c_offsets(tmp_path, name, [n for n, _ in fields])
    for n, _ in fields:
        assert f_off[n] == c[n], (name, n, f_off[n], c[n])
    assert f_size == c["sizeof"]


def test_config_type_has_every_c_field(tmp_path):
    """The Fortran type lists every field of the C struct, in order (no field left out)."""
    hdr = open(HDR).read()
    body = re.search(r"typedef struct mrlbm_config \{(.*?)\} mrlbm_config;", hdr, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    c_names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"^(double|uint64_t|int32_t)\s+", "", decl)
        c_names += [x.strip() for x in decl.split(",")]
    f_names = [n for n, _ in fortran_types()["mrlbm_config"]]
    assert [n.lower() for n in f_names] == [n.lower() for n in c_names]


def test_interfaces_match_header_and_library(mrlbm):
    src = _strip_comments(open(F90).read())
    hdr = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(?:int|size_t)\s+(mrlbm_\w+)\s*\(([^)]*)\)\s*;", hdr):
        args = [a for a in m.group(2).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(1)] = len(args)
    funcs = re.findall(r"function\s+(mrlbm_\w+)\s*\(([^)]*)\)\s*bind\(c\)", src.replace("&\n", " "), re.I)
    assert len(funcs) >= 30
    lib = ctypes.CDLL(mrlbm.api.LIB_PATH)
    for name, args in funcs:
        n = len([a for a in args.split(",") if a.strip()])
        assert name in protos, name
        assert protos[name] == n, (name, protos[name], n)
        assert hasattr(lib, name), name


def test_module_constants_match_the_header():
    """Every named constant of the module carries the value of the header's #define."""
    src = _strip_comments(open(F90).read())
    hdr = open(HDR).read()
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(MRLBM_\w+)\s+(-?\d+)", hdr)}
    consts = {}
    for decl in re.findall(r"parameter\s*::\s*(.*)", src, re.I):
        for item in decl.split(","):
            name, _, value = item.partition("=")
            consts[name.strip()] = int(value.strip().split("_")[0])
    assert len(consts) >= 20
    for name, value in consts.items():
        assert name in defs, name
        assert defs[name] == value, (name, defs[name], value)


def test_module_covers_every_header_function():
    src = _strip_comments(open(F90).read())
    hdr = re.sub(r"/\*.*?\*/", "", open(HDR).read(), flags=re.S)
    declared = set(re.findall(r"\b(?:int|size_t)\s+(mrlbm_\w+)\s*\(", hdr))
    bound = set(re.findall(r"function\s+(mrlbm_\w+)\s*\(", src, re.I))
    assert declared == bound, sorted(declared ^ bound)
