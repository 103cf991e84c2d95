"""The Julia structs of the INTEGRATION.md template against the C structs of
include/qem.h: every field's offset and each struct's size, as the C
compiler lays out qem_params and qem_lj_wall and as Julia lays out an
isbits struct (C alignment rules; NTuple{n,T} is n consecutive T).  A
ccall passing Ref{QemParams} reads the wrong fields if these differ."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PRIM = {"Float64": (8, 8), "Int32": (4, 4), "UInt32": (4, 4), "Int64": (8, 8), "UInt64": (8, 8)}


def _julia_block():
    txt = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```julia\n(.*?)```", txt, re.S)
    assert m, "no julia block in INTEGRATION.md"
    return m.group(1)


def _fields(src, name):
    m = re.search(r"\bstruct\s+" + name + r"\b(.*?)\bend\b", src, re.S)
    assert m, name
    body = re.sub(r"#[^\n]*", "", m.group(1))
    out = []
    for part in re.split(r"[;\n]", body):
        part = part.strip()
        if not part:
            continue
        f, t = part.split("::")
        out.append((f.strip(), t.strip()))
    return out


def _layout(fields, types):
    off, align, res = 0, 1, []
    for f, t in fields:
        m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", t)
        if m:
            n, (sz, al) = int(m.group(1)), types[m.group(2)]
            sz *= n
        else:
            sz, al = types[t]
        off = (off + al - 1) // al * al
        res.append((f, off))
        off += sz
        align = max(align, al)
    return res, (off + align - 1) // align * align, align


def _c_layout(struct, fields):
    src = "#include <stddef.h>\n#include <stdio.h>\n#include \"qem.h\"\nint main(void){\n"
    for f in fields:
        src += f'printf("%zu\\n", offsetof({struct}, {f}));\n'
    src += f'printf("%zu\\n", sizeof({struct}));\nreturn 0;}}\n'
    return src


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_julia_structs_match_the_c_abi(tmp_path):
    src = _julia_block()
    types = dict(PRIM)
    wall = _fields(src, "QemLJWall")
    wl, wsize, walign = _layout(wall, types)
    types["QemLJWall"] = (wsize, walign)
    par = _fields(src, "QemParams")
    pl, psize, _ = _layout(par, types)
    for struct, lay, size in (("qem_lj_wall", wl, wsize), ("qem_params", pl, psize)):
        c = tmp_path / f"{struct}.c"
        c.write_text(_c_layout(struct, [f for f, _ in lay]))
        exe = tmp_path / struct
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
        got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
        assert got[:-1] == [o for _, o in lay], (struct, list(zip([f for f, _ in lay], got, [o for _, o in lay])))
        assert got[-1] == size, (struct, got[-1], size)
    assert psize == 200
