"""CPU checks of the C ABI library: it loads, exports every entry point
declared in include/*.h, and the ctypes mirror of PicParams has the C
layout.  No compute call is made (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(REPO, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?(?:int|void|char)\s*\*?\s*(pic_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from pic3d_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_ctypes_mirror_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "pic3d_gpu.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(PicParams), offsetof(PicParams, charge),'
                   ' offsetof(PicParams, capacity), offsetof(PicParams, precision), offsetof(PicParams, tile),'
                   ' offsetof(PicParams, E_schwinger));}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), "-o", str(exe), str(src)], check=True)
    c_vals = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    from pic3d_b200._lib import PicParams
    py_vals = [ctypes.sizeof(PicParams), PicParams.charge.offset, PicParams.capacity.offset,
               PicParams.precision.offset, PicParams.tile.offset, PicParams.E_schwinger.offset]
    assert c_vals == py_vals


def test_default_params_without_gpu():
    from pic3d_b200 import _lib
    lib = _lib.load()
    p = _lib.PicParams()
    lib.pic_default_params(ctypes.byref(p))
    assert p.mem == 4 and p.precision == 64 and p.charge[0] == -1.0 and p.mass[1] == 1836.0


def test_no_oracle_in_product_path():
    """The package never imports the oracle (it is test infrastructure)."""
    pkg = os.path.join(REPO, "pic3d_b200")
    for root, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                text = open(os.path.join(root, f)).read()
                assert "import oracle" not in text and "pic_oracle" not in text and "liboracle" not in text, f


@pytest.mark.parametrize("bad", [dict(mem=3), dict(precision=16), dict(local_xcells=5), dict(dt=2.0)])
def test_create_rejects_bad_params(bad):
    """Parameter validation happens before any device call."""
    from pic3d_b200 import _lib
    lib = _lib.load()
    p = _lib.PicParams()
    lib.pic_default_params(ctypes.byref(p))
    for k, v in bad.items():
        setattr(p, k, v)
    h = ctypes.c_void_p()
    assert lib.pic_create(ctypes.byref(p), 0, ctypes.byref(h)) == _lib.PIC_EINVAL
    assert not h.value
