"""The C ABI: libmdgpu.so loads without a GPU and exports every entry point include/mdgpu.h
declares; the Python host side declares the same set. No compute calls."""
import ctypes
import os
import re

import pytest

from conftest import ROOT
from madpac_b200 import build as B
from madpac_b200 import mdgpu as M


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "mdgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mdgpu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    B.build()
    return ctypes.CDLL(B.LIB)


def test_library_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name


def test_python_binding_covers_the_header():
    assert set(M.SIGNATURES) == set(declared_symbols())


def test_create_without_gpu_fails_cleanly_or_works():
    # without a device the constructor reports ERR_CUDA (never crashes); with one it succeeds
    from madpac_b200 import workloads as W

    try:
        lc = M.LinkedCells([10.0, 10.0, 10.0], 2.5, [W.Component()])
    except M.MdgpuError as e:
        assert e.code == 2
    else:
        lc.close()


def test_oracle_is_not_imported_by_the_package():
    pkg = os.path.join(ROOT, "madpac_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cuh", ".cpp")):
                src = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in src and "liboracle" not in src, f


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the header's structs have the C compiler's sizes and field offsets."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {"mdgpu_component": M._MdComponent, "mdgpu_site": M._MdSite, "mdgpu_charge": M._MdCharge,
               "mdgpu_oriented": M._MdOriented}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mdgpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out if line}
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)
