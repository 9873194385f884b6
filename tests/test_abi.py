"""The C-ABI library loads, exports every entry point that include/mh_darcy.h declares, and
behaves as documented without a GPU (no compute calls on the CPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import mhdarcy
from mhdarcy import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(mh_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) >= 20
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.EXPORTED) | set(names)


def test_version_and_status_strings():
    assert b"sm_100a" in _lib.lib.mh_version()
    assert _lib.lib.mh_status_string(_lib.MH_ERR_SINGULAR) == b"singular local matrix"
    assert _lib.lib.mh_status_string(12345) == b"unknown status"


def test_default_options():
    o = mhdarcy.solve_opts()
    assert o.r_tol == 1e-10 and o.max_it == 20000 and o.method == _lib.MH_SOLVER_PCG64


def test_create_without_device_builds_topology():
    m = mhdarcy.cube_mesh(2, [(2, 1)], [(0, 1, 1)])
    with mhdarcy.MHSystem(m) as s:
        assert s.sizes.n_elements == 6 * 8 + 8 + 2
        t = s.topology()
        assert len(t["side_edge"]) == s.n_sides
        if not mhdarcy.device_available():
            with pytest.raises(mhdarcy.MHError) as ei:
                s.set_coeffs(conductivity=np.ones(s.n_elements))
            assert ei.value.status == _lib.MH_ERR_CUDA


def test_invalid_arguments():
    d = _lib.MeshDesc()
    h = C.c_void_p()
    assert _lib.lib.mh_create(C.byref(d), C.byref(h)) == _lib.MH_ERR_INVALID
    assert _lib.lib.mh_create(None, C.byref(h)) == _lib.MH_ERR_INVALID
    h2 = C.c_void_p()
    assert _lib.lib.mh_cube_mesh_create(0, 0, None, None, 0, None, None, None, C.byref(h2)) == _lib.MH_ERR_INVALID


STRUCTS = {  # C type in include/mh_darcy.h -> ctypes mirror in mhdarcy/_lib.py
    "mh_mesh_desc": "MeshDesc", "mh_mortar_desc": "MortarDesc", "mh_gmsh_info": "GmshInfo",
    "mh_sizes": "Sizes", "mh_coeffs": "Coeffs", "mh_bc": "BC", "mh_solve_opts": "SolveOpts",
    "mh_solve_stats": "SolveStats", "mh_tune_result": "TuneResult", "mh_learn_opts": "LearnOpts",
    "mh_learn_stats": "LearnStats",
}


def test_struct_layouts_match_the_header(tmp_path):
    """Every public struct has the same size and field offsets in the header (compiled with
    gcc) and in the ctypes mirror the Python bindings pass to the library."""
    import ctypes
    import shutil
    import subprocess
    from mhdarcy import _lib
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mh_darcy.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        py = getattr(_lib, pyname)
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for cname, pyname in STRUCTS.items():
        py = getattr(_lib, pyname)
        assert int(out["%s size" % cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out["%s.%s" % (cname, f)]) == getattr(py, f).offset, (cname, f)
