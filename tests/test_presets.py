"""The oracle's restatement of the parameter presets (oracle/presets.py) equals
the library's sph_config_preset byte for byte, for every preset.  The CPU
reference arm of the benchmark builds its configuration from the restatement,
so it never loads the CUDA library."""
import ctypes as C
import subprocess
import sys

import pytest

import sca2012_b200 as sph
from oracle import presets as P

ALL = [sph.PRESET_REF_2D, sph.PRESET_REF_3D2, sph.PRESET_REF_3D4, sph.PRESET_DAM_2D, sph.PRESET_DAM_3D2,
       sph.PRESET_DAM_3D4, sph.PRESET_ROLLOUT_3D]


@pytest.mark.parametrize("which", ALL)
def test_preset_restatement_is_bit_identical(which):
    lib_cfg = sph.preset(which)
    ora_cfg = P.preset(which)
    a = C.string_at(C.addressof(lib_cfg), C.sizeof(lib_cfg))
    b = C.string_at(C.addressof(ora_cfg), C.sizeof(ora_cfg))
    if a != b:
        diff = [name for name, _ in type(lib_cfg)._fields_
                if C.string_at(C.addressof(lib_cfg) + getattr(type(lib_cfg), name).offset,
                               getattr(type(lib_cfg), name).size)
                != C.string_at(C.addressof(ora_cfg) + getattr(type(lib_cfg), name).offset,
                               getattr(type(lib_cfg), name).size)]
        pytest.fail(f"preset {which}: fields differ: {diff}")


def test_oracle_side_loads_no_product_library():
    # a fresh interpreter: the oracle, its presets and the scene generator
    # (loaded the way the benchmark's reference arm loads them) map no
    # library of the package
    code = (
        "import sys; sys.path.insert(0, '.');"
        "from oracle import presets as P, oracle as O;"
        "import importlib.util as u;"
        "s = u.spec_from_file_location('scn', 'sca2012_b200/scenes.py'); m = u.module_from_spec(s);"
        "s.loader.exec_module(m);"
        "c = P.preset(P.PRESET_DAM_2D); pos, vel, lvl = m.dam_2d(c, seed=0);"
        "st, _ = O.step(c, dict(pos=pos, vel=vel, level=lvl));"
        "maps = open('/proc/self/maps').read();"
        "assert 'libsca2012_b200' not in maps, 'product library mapped';"
        "assert 'sca2012_b200' not in sys.modules;"
        "print(len(st['pos']))")
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    assert int(out.stdout.strip()) == 4096
