"""C-ABI library checks that need no GPU: it loads, exports every entry point
include/sph/sph.h declares, the ctypes layout matches, presets are sane, and
calls that need a device fail with a status code instead of crashing."""
import ctypes as C
import os
import re

import numpy as np

import sca2012_b200 as sph
from sca2012_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include", "sph")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", "sph", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sph_[a-z_0-9]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    lib = sph.lib()
    names = declared_entry_points()
    assert len(names) >= 19
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    bound = {s[0] for s in _abi.SIGNATURES}
    assert names <= bound, f"declared but not bound in _abi.SIGNATURES: {sorted(names - bound)}"


def test_config_layout():
    assert sph.lib().sph_config_size() == C.sizeof(_abi.Config)


def test_reference_presets_match_constructor_formulas():
    # SPH-3D-2/sph_system.cpp:63-84 with PI = 3.141592f, float products, double pow
    c = sph.preset(sph.PRESET_REF_3D2)
    PI = np.float32(3.141592)
    h = np.float64(np.float32(0.9))
    poly6 = np.float32(315.0 / (np.float64(np.float32(64.0) * PI) * h ** 9))
    assert np.float32(c.poly6[1]) == poly6
    assert list(c.ncell) == [32, 16, 16] and c.world[0] == 32.0
    assert list(c.ndens) == [129, 65, 65]
    c4 = sph.preset(sph.PRESET_REF_3D4)
    assert list(c4.ncell) == [40, 20, 20] and c4.split_ways == 4
    c2 = sph.preset(sph.PRESET_REF_2D)
    assert c2.dim == 2 and list(c2.ncell)[:2] == [32, 32] and c2.merge_rule == _abi.MERGE_WAVELET_CELL


def test_si_presets():
    c = sph.preset(sph.PRESET_DAM_3D4)
    assert list(c.ncell) == [128, 128, 64]
    assert abs(c.mass[0] - 1000 * 0.005 ** 3) < 1e-7 * c.mass[0]
    assert abs(c.kernel[1] - 0.01 / 4 ** (1 / 3)) < 1e-7
    c = sph.preset(sph.PRESET_DAM_2D)
    assert list(c.ncell)[:2] == [64, 64] and c.use_split == 0


def test_unknown_preset_is_an_error():
    c = _abi.Config()
    assert sph.lib().sph_config_preset(99, C.byref(c)) == _abi.SPH_ERR_INVALID


def test_create_without_device_or_bad_config_returns_status():
    lib = sph.lib()
    h = _abi.H()
    bad = sph.preset(sph.PRESET_REF_3D2)
    bad.dim = 5
    assert lib.sph_create(C.byref(bad), C.byref(h)) == _abi.SPH_ERR_INVALID
    bad = sph.preset(sph.PRESET_REF_3D2)
    bad.kernel[0] = 2.0   # longer than a cell: the 27-cell stencil would miss pairs
    assert lib.sph_create(C.byref(bad), C.byref(h)) == _abi.SPH_ERR_INVALID
    assert lib.sph_step(None, 1) == _abi.SPH_ERR_INVALID
    assert lib.sph_destroy(None) == _abi.SPH_ERR_INVALID


def test_reference_scenes_have_reference_counts():
    # counts of the reference's own lattice loops
    assert len(sph.scenes.ref_box_3d2(sph.preset(sph.PRESET_REF_3D2))[0]) == 20 * 19 * 19
    assert len(sph.scenes.ref_init_2d(sph.preset(sph.PRESET_REF_2D))[0]) == 31 * 63
