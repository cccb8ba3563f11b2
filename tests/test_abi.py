"""The C ABI library loads without a GPU and exports every symbol that
include/*.h declares; host-only entry points agree with the oracle."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np

import molmodel_b200
from molmodel_b200 import _lib
from oracle.oracle import port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(mmnb_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = molmodel_b200.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert {n for n, _, _ in _lib.SIGNATURES} == names


def test_config_defaults_are_the_references():
    lib = molmodel_b200.load_library()
    c = _lib.MmnbConfig()
    assert lib.mmnb_config_init(ctypes.byref(c)) == 0
    # src/eleclj.cpp:13-40
    assert (c.rspace_cutoff, c.smoothing_width, c.neighbor_list_width, c.kspace_cutoff) == (0, 1, 0, 5)
    assert c.ewald_screening == -1 and c.use_p3m == 0 and c.p3m_grid_spacing == 0.5
    assert (c.p3m_assignment_order, c.p3m_alias_sum_limit, c.p3m_ik_differentiate) == (3, 2, 0)
    assert c.include_lj_correction == 1 and c.geometric_combining_for_sigma == 0
    assert (c.include_rspace, c.include_kspace, c.include_self) == (1, 1, 1)
    assert c.p3m_grid_density == -1


def test_config_mirror_has_the_headers_layout(tmp_path):
    """Every field of the ctypes mirror sits at the offset the C compiler gives
    it in include/mmnb.h, and the two structs have one size."""
    fields = [f for f, _ in _lib.MmnbConfig._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stdio.h>\n#include <stddef.h>\n#include \"mmnb.h\"\nint main(void) {\n"
                   + "".join('  printf("%%zu\\n", offsetof(mmnb_config, %s));\n' % f for f in fields)
                   + '  printf("%zu\\n", sizeof(mmnb_config));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    want = [getattr(_lib.MmnbConfig, f).offset for f in fields] + [ctypes.sizeof(_lib.MmnbConfig)]
    assert got == want


def test_chebyshev_table_is_the_oracles_bitwise():
    lib = molmodel_b200.load_library()
    for rc, eta in ((9.0, 0.35), (7.0, 0.45), (1.5, 1.2)):
        c = np.zeros(512 * 7)
        mn, mx, inv = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        dp = ctypes.POINTER(ctypes.c_double)
        assert lib.mmnb_chebyshev_table(rc, eta, ctypes.byref(mn), ctypes.byref(mx), ctypes.byref(inv),
                                        c.ctypes.data_as(dp)) == 0
        o = port().chebyshev(rc, eta)
        assert (mn.value, mx.value, inv.value) == o[:3]
        assert np.array_equal(c, o[3].reshape(-1))


def test_mesh_size_rule():
    lib = molmodel_b200.load_library()
    # multiple_of_2357_near (src/pppm.c:277-292): nearest 2^a3^b5^c7^d, first found on ties
    assert lib.mmnb_p3m_mesh_size(99.437, 99.437 / 96) == 96
    assert lib.mmnb_p3m_mesh_size(49.719, 49.719 / 48) == 48
    assert lib.mmnb_p3m_mesh_size(19.731, 1.04) == 18
    assert lib.mmnb_p3m_mesh_size(11.0, 1.0) == 10  # 11 -> 10 and 12 tie; 10 is found first
    assert lib.mmnb_p3m_mesh_size(13.0, 1.0) == 12
    assert lib.mmnb_p3m_mesh_size(-1.0, 1.0) == 0


def test_create_rejects_bad_arguments_without_touching_a_gpu():
    lib = molmodel_b200.load_library()
    c = _lib.MmnbConfig()
    lib.mmnb_config_init(ctypes.byref(c))
    h = ctypes.c_void_p()
    g = np.array([[0, 3]], dtype=np.int32)
    ip = ctypes.POINTER(ctypes.c_int)
    # no box
    assert lib.mmnb_create(ctypes.byref(c), 3, 1, g.ctypes.data_as(ip), 0, None, 0, None, ctypes.byref(h)) == 1
    assert b"box" in lib.mmnb_last_error(None)
    c.box = (ctypes.c_double * 3)(10.0, 10.0, 10.0)
    c.bctype = 5
    assert lib.mmnb_create(ctypes.byref(c), 3, 1, g.ctypes.data_as(ip), 0, None, 0, None, ctypes.byref(h)) == 3
    c.bctype = 1
    c.rspace_cutoff = 6.0  # > 0.49 * 10
    assert lib.mmnb_create(ctypes.byref(c), 3, 1, g.ctypes.data_as(ip), 0, None, 0, None, ctypes.byref(h)) == 4
    bad = np.array([[0, 2]], dtype=np.int32)  # site 2 in no group
    c.rspace_cutoff = 4.0
    assert lib.mmnb_create(ctypes.byref(c), 3, 1, bad.ctypes.data_as(ip), 0, None, 0, None, ctypes.byref(h)) == 1
    assert lib.mmnb_status_string(4) == b"cutoff too large for the box"
