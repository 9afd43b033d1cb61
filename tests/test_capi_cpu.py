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


def _reference_src():
    root = os.environ.get("LIBGRID_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    return os.path.join(root, "src")


STRUCT_FIELDS = {
    "cgrid": ["value", "id", "grid_len", "nx", "ny", "nz", "step", "x0", "y0", "z0", "kx0", "ky0", "kz0", "omega",
              "value_outside", "outside_params_ptr", "default_outside_params", "plan", "iplan", "cufft_handle",
              "host_lock", "fft_norm", "fft_norm2", "flag"],
    "rgrid": ["value", "id", "grid_len", "nx", "ny", "nz", "nz2", "step", "x0", "y0", "z0", "kx0", "ky0", "kz0",
              "value_outside", "outside_params_ptr", "default_outside_params", "plan", "iplan", "cufft_handle_r2c",
              "cufft_handle_c2r", "host_lock", "fft_norm", "fft_norm2", "flag"],
    "wf": ["grid", "mass", "norm", "cfft_width", "boundary", "propagator", "cworkspace", "cworkspace2", "cworkspace3",
           "ts_func", "lx", "hx", "ly", "hy", "lz", "hz", "kmax"],
}


def _layout(tmp_path, name, prelude):
    lines = []
    for st, fields in STRUCT_FIELDS.items():
        lines.append('printf("%s sizeof %%zu\\n", sizeof(%s));' % (st, st))
        for f in fields:
            lines.append('printf("%s.%s %%zu %%zu\\n", offsetof(%s, %s), sizeof(((%s *) 0)->%s));' % (st, f, st, f, st, f))
    prog = tmp_path / (name + ".c")
    prog.write_text(prelude + "\n#include <stddef.h>\n#include <stdio.h>\nint main(void){\n" + "\n".join(lines) +
                    "\nreturn 0;}\n")
    exe = tmp_path / name
    subprocess.run(["gcc", "-std=gnu99", "-I" + INCLUDE, str(prog), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()


def test_struct_layout_matches_reference_structs_h(tmp_path):
    """Every field offset and size of cgrid, rgrid and wf in include/grid.h
    equals the reference's src/structs.h compiled as the reference's CUDA,
    double-precision build sees it (USE_CUDA, DOUBLE_PREC, REAL double, INT
    long, fftw_plan a pointer, cufftHandle an int), so existing callers
    recompile unchanged."""
    src = _reference_src()
    if not os.path.exists(os.path.join(src, "structs.h")):
        pytest.skip("reference sources not present (set LIBGRID_REFERENCE)")
    ref_prelude = (
        "#include <complex.h>\n#include <sys/time.h>\n#include <time.h>\n"
        "#define REAL double\n#define INT long\n#define DOUBLE_PREC\n#define USE_CUDA\n"
        "typedef struct fftw_plan_s *fftw_plan;\ntypedef int cufftHandle;\n"
        '#include "%s"\n' % os.path.join(src, "structs.h")
    )
    ours = _layout(tmp_path, "ours", '#include "grid.h"')
    theirs = _layout(tmp_path, "theirs", ref_prelude)
    assert ours == theirs
    assert len(ours) == 3 + sum(len(f) for f in STRUCT_FIELDS.values())
