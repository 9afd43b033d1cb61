"""CPU checks of the C ABI (no GPU): the shared library loads, exports every
function the public headers declare, keeps the reference's struct layout, and
its host-side grid operations behave like the reference's."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from libgrid_b200 import capi

INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for h in ("grid.h", "gb_cuda.h"):
        src = open(os.path.join(INCLUDE, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", src, flags=re.M):
            name = m.group(1)
            if name in ("if", "while", "for", "sizeof", "return"):
                continue
            names.add(name)
    return sorted(names)


def test_exports_every_declared_function(b200):
    missing = [n for n in declared_functions() if not hasattr(b200.lib, n)]
    assert not missing, missing
    assert len(declared_functions()) > 120


def test_struct_layout_matches_header(b200, tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text(
        '#include "grid.h"\n#include <stddef.h>\n#include <stdio.h>\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu\\n\", sizeof(cgrid), sizeof(rgrid), sizeof(wf),"
        " offsetof(cgrid, fft_norm), offsetof(rgrid, fft_norm));return 0;}\n"
    )
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I" + INCLUDE, str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    cs, rs, ws, cfo, rfo = (int(x) for x in out)
    assert C.sizeof(b200.CGrid) == cs
    assert C.sizeof(b200.RGrid) == rs
    assert C.sizeof(b200.WF) == ws
    assert b200.CGrid.fft_norm.offset == cfo
    assert b200.RGrid.fft_norm.offset == rfo


def test_host_side_grid_access(b200):
    g = b200.cgrid(4, 5, 6, 0.5)
    a = (np.arange(120).reshape(4, 5, 6) * (1 + 0.5j)).astype(complex)
    g.set(a)
    assert b200.lib.cgrid_value_at_index(g.ptr, 1, 2, 3).value() == a[1, 2, 3]
    # periodic wrap through value_outside (src/cgrid_bc.c:69-86)
    assert b200.lib.cgrid_value_at_index(g.ptr, -1, 7, 6).value() == a[3, 2, 0]
    b200.lib.cgrid_value_to_index(g.ptr, 0, 0, 0, capi.Complex.of(7 - 1j))
    assert g.get()[0, 0, 0] == 7 - 1j
    d = b200.cgrid(3, 3, 3, 0.5, bc="dirichlet")
    assert b200.lib.cgrid_value_at_index(d.ptr, 5, 0, 0).value() == 0
    n = b200.cgrid(4, 4, 4, 0.5, bc="neumann")
    n.set(np.arange(64).reshape(4, 4, 4).astype(complex))
    # mirror i -> 2 n - i - 2 (src/cgrid_bc.c:45-57)
    assert b200.lib.cgrid_value_at_index(n.ptr, 4, 1, 1).value() == 2 * 16 + 1 * 4 + 1
    for x in (g, d, n):
        b200.free(x)


def test_wf_alloc_validation(b200):
    # Dirichlet only with Crank-Nicolson (src/grid_wf.c:41-44)
    p = b200.lib.grid_wf_alloc(8, 8, 8, 0.1, 1.0, bytes([capi.WF_DIRICHLET_BOUNDARY]), bytes([capi.WF_2ND_ORDER_FFT]), b"x")
    assert not p
    p = b200.lib.grid_wf_alloc(8, 8, 8, 0.1, 1.0, bytes([9]), bytes([capi.WF_2ND_ORDER_FFT]), b"x")
    assert not p
    w = b200.wf(8, 8, 8, 0.1, 1.0, capi.WF_DIRICHLET_BOUNDARY, capi.WF_2ND_ORDER_CN)
    assert w.s.kmax == 9999.0 and w.s.norm == 1.0 and w.s.cfft_width == 1.0
    b200.free(w)


def test_binary_write_format_matches_reference(b200, ref):
    a = (np.arange(60).reshape(3, 4, 5) * (0.25 - 1j)).astype(complex)
    blobs = []
    libc = C.CDLL("libc.so.6")
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    for api in (b200, ref):
        g = api.cgrid(3, 4, 5, 0.7, values=a)
        api.lib.cgrid_write.argtypes = [C.POINTER(api.CGrid), C.c_void_p]
        with tempfile.NamedTemporaryFile(delete=False) as f:
            path = f.name
        fp = libc.fopen(path.encode(), b"wb")
        api.lib.cgrid_write(g.ptr, fp)
        libc.fclose(fp)
        blobs.append(open(path, "rb").read())
        os.unlink(path)
    assert blobs[0] == blobs[1]
    # read it back into a fresh grid
    with tempfile.NamedTemporaryFile(delete=False) as f:
        f.write(blobs[0])
        path = f.name
    b200.lib.cgrid_read.restype = C.POINTER(b200.CGrid)
    b200.lib.cgrid_read.argtypes = [C.POINTER(b200.CGrid), C.c_void_p]
    g = b200.cgrid(3, 4, 5, 0.7)
    fp = libc.fopen(path.encode(), b"rb")
    b200.lib.cgrid_read(g.ptr, fp)
    libc.fclose(fp)
    os.unlink(path)
    assert np.array_equal(g.get(), a)


def test_analyze_method_default_is_finite_difference(b200):
    m = C.c_char.in_dll(b200.lib, "grid_analyze_method")
    g = b200.cgrid(2, 2, 2, 1.0)
    assert m.value in (b"\x00", b"\x01")
    b200.free(g)
