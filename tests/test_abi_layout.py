"""The ctypes structures of rome_b200.abi lay out exactly like the C
structures of include/rome_gpu.h: the same member names in the same order,
each at the same byte offset, and the same total size, as the host C
compiler lays them out.  A caller binding the header from C, C++ or any FFI
and the Python host side then pass the same bytes.  CPU only (gcc)."""
import ctypes
import os
import re
import shutil
import subprocess
import tempfile

import pytest

from rome_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rome_gpu.h")


def header_structs():
    """{typedef name: [member names in order]} of the header's typedef'd structs."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    out = {}
    for body, name in re.findall(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
        members = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "type a, b[2]" -> the declarators after the type
            first, *rest = decl.split(",")
            names = [re.findall(r"(\w+)\s*(?:\[[^\]]*\])?\s*$", first)[0]]
            names += [re.findall(r"(\w+)\s*(?:\[[^\]]*\])?\s*$", r)[0] for r in rest]
            members += names
        out[name] = members
    return out


def ctypes_structs():
    return {n: getattr(abi, n) for n in dir(abi)
            if isinstance(getattr(abi, n), type) and issubclass(getattr(abi, n), ctypes.Structure)}


def test_every_header_struct_has_a_binding():
    assert sorted(header_structs()) == sorted(ctypes_structs())


def test_member_names_and_order_match():
    hs, cs = header_structs(), ctypes_structs()
    for name, members in hs.items():
        assert [f[0] for f in cs[name]._fields_] == members, name


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs the host C compiler")
def test_offsets_and_sizes_match_the_c_compiler():
    cs = ctypes_structs()
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{HEADER}"', "int main(void) {"]
    for name, st in sorted(cs.items()):
        lines.append(f'    printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field in st._fields_:
            lines.append(f'    printf("{name} {field[0]} %zu\\n", offsetof({name}, {field[0]}));')
    lines += ["    return 0;", "}"]
    tmp = tempfile.mkdtemp(prefix="rome_abi_")
    try:
        c = os.path.join(tmp, "layout.c")
        exe = os.path.join(tmp, "layout")
        with open(c, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-o", exe, c])
        out = subprocess.check_output([exe], text=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    got = {}
    for line in out.splitlines():
        s, m, v = line.split()
        got[(s, m)] = int(v)
    for name, st in cs.items():
        assert got[(name, "sizeof")] == ctypes.sizeof(st), name
        for field in st._fields_:
            assert got[(name, field[0])] == getattr(st, field[0]).offset, (name, field[0])


def test_pointer_helpers_reject_the_wrong_arrays():
    """Arrays passed to the library as raw pointers must have the element
    type and C-contiguous layout the C side reads; anything else is refused
    before the call (also under python -O)."""
    import numpy as np
    assert abi.dptr(None) is not None and not abi.dptr(None)
    abi.dptr(np.zeros(3))
    abi.iptr(np.zeros(3, np.int32))
    abi.cptr(np.zeros(3, np.int8))
    for bad, fn in ((np.zeros(3, np.float32), abi.dptr), (np.zeros((4, 4))[:, ::2], abi.dptr),
                    (np.zeros(3, np.int64), abi.iptr), (np.zeros(3, np.uint8), abi.cptr)):
        with pytest.raises(TypeError):
            fn(bad)
