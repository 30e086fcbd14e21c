"""C ABI: the library loads without a GPU, exports every entry point the
header declares, and the Python mirrors match the C layouts."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from baccolonygrowth_b200 import _abi, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "bcg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(bcg_[a-z0-9_]+)\s*\(", text)
    return sorted(set(n for n in names if not n.endswith("_t")))


def test_header_functions_exported():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # every declared function has a ctypes prototype
    assert not [n for n in names if n not in _abi.PROTOTYPES]


def _c_layout():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "bcg.h"
int main(void) {
  printf("%zu %zu %zu\n", sizeof(bcg_params), sizeof(bcg_cell), sizeof(bcg_rng));
  printf("%zu %zu %zu %zu\n", offsetof(bcg_params, box_length), offsetof(bcg_params, c1_ph),
         offsetof(bcg_params, mg_dt), offsetof(bcg_params, cross_feeding));
  printf("%zu %zu %zu\n", offsetof(bcg_cell, length), offsetof(bcg_cell, velocity), offsetof(bcg_cell, type));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        return subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()


def test_struct_layouts_match_header():
    v = list(map(int, _c_layout()))
    assert v[0] == ctypes.sizeof(_abi.Params)
    assert v[1] == _abi.CELL_DTYPE.itemsize == 208
    assert v[2] == ctypes.sizeof(_abi.Rng)
    assert v[3] == _abi.Params.box_length.offset
    assert v[4] == _abi.Params.c1_ph.offset
    assert v[5] == _abi.Params.mg_dt.offset
    assert v[6] == _abi.Params.cross_feeding.offset
    assert v[7] == _abi.CELL_DTYPE.fields["length"][1]
    assert v[8] == _abi.CELL_DTYPE.fields["velocity"][1]
    assert v[9] == _abi.CELL_DTYPE.fields["type"][1]


def test_params_from_shipped_input():
    p = params.parse_parameters(params.shipped_input_text("small"))
    params.finalize(p)
    # CellMD3D.cpp:52-54 derivations for the shipped input
    assert p.box_length == 4.0
    assert p.max_cells_per_box == 99
    assert (p.box_x, p.box_y, p.box_z, p.box_z_agar, p.max_levels_mg) == (256, 1, 50, 32, 2)
    assert p.q_car_aer_nt == 0.00037      # "0.00037;" parsed with atof semantics
    assert p.cross_feeding == 0 and p.nutrient_gsi == 0


def test_create_without_device_reports_status():
    # on a machine without a GPU bcg_create must fail with a status, not abort
    from tests_util import cuda_count
    if cuda_count() > 0:
        pytest.skip("a device is present")
    p = params.workload_params("small_4k")
    h = ctypes.c_void_p()
    rc = _abi.load().bcg_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == _abi.E_NO_DEVICE
