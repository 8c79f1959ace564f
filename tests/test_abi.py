"""The C ABI: the library loads, exports every function include/sgh_b200.h
declares, its struct layouts match the ctypes mirror, and plan validation
rejects bad configurations -- all without touching a GPU."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT, make_context
from spectral_galerkin_heat_b200 import _lib, workloads
from spectral_galerkin_heat_b200.solver import make_config

HEADER = os.path.join(ROOT, "include", "sgh_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sgh_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 16
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTED) == names
    assert L.sgh_abi_version() == _lib.ABI_VERSION == 3


def test_struct_layout_matches_header():
    """Compile a host-only C program against the header and compare offsets."""
    structs = {
        "sgh_config": _lib.SghConfig, "sgh_laser": _lib.SghLaser,
        "sgh_step_out": _lib.SghStepOut, "sgh_program": _lib.SghProgram,
        "sgh_box_geom": _lib.SghBoxGeom,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sgh_b200.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                       check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        cname, field, val = line.split()
        py = structs[cname]
        if field == "size":
            assert C.sizeof(py) == int(val), cname
        else:
            assert getattr(py, field).offset == int(val), (cname, field)


def _cfg(**over):
    cfg, path = workloads.nonlinear_raster(nx=16, ny=8, nz=4)
    c = make_config(make_context(cfg, path), 0.1, 1e-8, 50)
    for k, v in over.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("over", [dict(nx=1), dict(nz=0), dict(dt=0.0), dict(r_x=0.0),
                                  dict(precision=3), dict(max_iter=-1),
                                  dict(cell_integrated=1, order=4.0)])
def test_plan_create_rejects_bad_config(over):
    L = _lib.lib()
    p = C.c_void_p()
    rc = L.sgh_plan_create(C.byref(_cfg(**over)), C.byref(p))
    assert rc < 0
    assert L.sgh_last_error()


def test_plan_create_rejects_bad_program():
    c = _cfg()
    c.k_solid.ops[0] = 99  # unknown opcode
    p = C.c_void_p()
    assert _lib.lib().sgh_plan_create(C.byref(c), C.byref(p)) == -1
    assert b"opcode" in _lib.lib().sgh_last_error()


def test_plan_create_and_workspace_size():
    L = _lib.lib()
    p = C.c_void_p()
    assert L.sgh_plan_create(C.byref(_cfg()), C.byref(p)) == 0
    n = C.c_uint64()
    assert L.sgh_plan_workspace_bytes(p, C.byref(n)) == 0
    assert n.value > 11 * 16 * 8 * 4 * 8
    # unbound plans refuse to run
    out = _lib.SghStepOut()
    las = _lib.SghLaser()
    assert L.sgh_step(p, C.byref(las), C.byref(out), None) == -3
    assert L.sgh_plan_destroy(p) == 0


def test_dctn_workspace_query():
    L = _lib.lib()
    n = C.c_uint64()
    shape = (C.c_int32 * 3)(4, 5, 6)
    assert L.sgh_dctn_workspace_bytes(3, shape, C.byref(n)) == 0
    assert n.value >= 2 * 120 * 8
    assert L.sgh_dctn_workspace_bytes(4, shape, C.byref(n)) == -1
