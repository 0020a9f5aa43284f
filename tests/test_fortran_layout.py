"""The Fortran interface module (include/hipft_gpu.f90) against the C header.

No Fortran compiler exists in this image, so the module is checked by
reading it: every `type, bind(c)` derived type must have the C struct's
layout (field names, order, offsets and size under the iso_c_binding kinds),
measured by compiling a probe of include/hipft_gpu.h with gcc; every
`bind(c)` interface must name a function the header declares and the
library exports, with the header's argument count, and pass each argument
the way the C prototype takes it (by value or by address).
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F90 = os.path.join(ROOT, "include", "hipft_gpu.f90")
HDR = os.path.join(ROOT, "include", "hipft_gpu.h")

KIND = {"c_int": 4, "c_double": 8, "c_ptr": 8, "c_funptr": 8, "c_int64_t": 8, "c_size_t": 8}


def _fortran_text():
    # join continuation lines and drop comments
    lines = []
    for raw in open(F90):
        line = raw.split("!", 1)[0].rstrip()
        if lines and lines[-1].endswith("&"):
            lines[-1] = lines[-1][:-1] + " " + line.strip()
        else:
            lines.append(line)
    return lines


def fortran_types():
    out, cur = {}, None
    for line in _fortran_text():
        s = line.strip()
        m = re.match(r"type,\s*bind\(c\)\s*::\s*(\w+)", s, re.I)
        if m:
            cur = m.group(1)
            out[cur] = []
            continue
        if cur and re.match(r"end\s+type", s, re.I):
            cur = None
            continue
        if cur:
            m = re.match(r"(integer|real|type)\((c_\w+)\)\s*::\s*(.+)", s, re.I)
            assert m, f"unparsed field line in {cur}: {s}"
            for name in m.group(3).split(","):
                out[cur].append((name.strip(), m.group(2).lower()))
    return out


def c_layout(fields):
    off, offs, align = 0, [], 1
    for name, kind in fields:
        size = KIND[kind]
        off = (off + size - 1) // size * size
        offs.append((name, off))
        off += size
        align = max(align, size)
    return offs, (off + align - 1) // align * align


def fortran_interfaces():
    funcs, cur = {}, None
    for line in _fortran_text():
        s = line.strip()
        m = re.match(r"integer\(c_int\)\s+function\s+(\w+)\(([^)]*)\)\s*bind\(c,\s*name=\"(\w+)\"\)", s, re.I)
        if m:
            cur = m.group(3)
            args = [a.strip() for a in m.group(2).split(",") if a.strip()]
            funcs[cur] = {"args": args, "decl": {}}
            continue
        if cur and re.match(r"end\s+function", s, re.I):
            cur = None
            continue
        if cur:
            m = re.match(r"(integer|real|type|character)\(([^)]*)\)\s*(,[^:]*)?::\s*(.+)", s, re.I)
            if m:
                attrs = (m.group(3) or "").lower()
                kind = m.group(2).lower()
                for name in re.split(r",(?![^(]*\))", m.group(4)):
                    base = re.sub(r"\(.*\)", "", name).strip()
                    funcs[cur]["decl"][base] = (kind, "value" in attrs)
    return funcs


def header_prototypes():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(?:int|const char \*)\s+(hipft_\w+)\s*\(([^;]*?)\)\s*;", text, re.S):
        params = [p.strip() for p in re.split(r",(?![^(]*\))", m.group(2)) if p.strip() and p.strip() != "void"]
        protos[m.group(1)] = params
    return protos


def test_bind_c_types_match_the_header(tmp_path):
    types = fortran_types()
    assert set(types) >= {"hipft_grid", "hipft_params", "hipft_flow_def", "hipft_da_opts", "hipft_diffusion_info",
                          "hipft_info", "hipft_shard"}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HDR}"', "int main(void) {"]
    for t, fields in types.items():
        lines.append(f'  printf("{t} sizeof %zu\\n", sizeof({t}));')
        for name, _ in fields:
            lines.append(f'  printf("{t} {name} %zu\\n", offsetof({t}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], check=True)
    got = {}
    for row in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        t, f, v = row.split()
        got[(t, f)] = int(v)
    for t, fields in types.items():
        offs, size = c_layout(fields)
        for name, off in offs:
            assert got[(t, name)] == off, f"{t}.{name}: Fortran offset {off}, C offset {got[(t, name)]}"
        assert got[(t, "sizeof")] == size, f"{t}: Fortran size {size}, C size {got[(t, 'sizeof')]}"


def test_interfaces_match_prototypes_and_exports():
    from hipft_b200 import gpu
    L = gpu.lib()
    protos = header_prototypes()
    funcs = fortran_interfaces()
    assert len(funcs) >= 30
    for name, f in funcs.items():
        assert name in protos, f"{name} is not declared in hipft_gpu.h"
        assert hasattr(L, name), f"{name} is not exported by libhipft_gpu.so"
        params = protos[name]
        assert len(f["args"]) == len(params), f"{name}: {len(f['args'])} Fortran arguments, {len(params)} in C"
        for a, cp in zip(f["args"], params):
            kind, by_value = f["decl"][a]
            c_is_pointer = "*" in cp or "[" in cp or cp.split()[0].endswith("_cb")
            f_is_pointer = (not by_value) or kind in ("c_ptr", "c_funptr")
            assert c_is_pointer == f_is_pointer, f"{name}({a}): C '{cp}' vs Fortran {kind} value={by_value}"
