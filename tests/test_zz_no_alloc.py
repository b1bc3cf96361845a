"""GPU test of sph_sort_cells_noalloc, the cell sort for callers that cannot
call cudaMalloc (a host program whose device memory belongs to another
allocator, or a loop that cannot afford cudaMalloc's implicit device
synchronisation).  Its scratch lives in a fixed static device array inside
the library; the caller passes only inputs and outputs.

Through the C-ABI, its outputs must equal the cell sort the existing entry
point performs inside sph_step (read back with sph_get_debug) on the same
positions, on two calls in a row (the second call reuses the array the first
one left behind).  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import sca2012_b200 as sph
from sca2012_b200 import _abi, scenes

pytestmark = pytest.mark.gpu


def _existing_sort(cfg, pos, vel, lvl):
    s = sph.Solver(cfg)
    s.set_state(dict(pos=pos, vel=vel, level=lvl))
    s.step(1)
    assert s.sync_status() == 0
    d = s.get_debug()
    s.close()
    return d


def _noalloc_sort(cfg, pos):
    import torch
    n = len(pos)
    ncell = int(np.prod([cfg.ncell[a] for a in range(cfg.dim)]))
    pos_d = torch.from_numpy(np.ascontiguousarray(pos, np.float32)).cuda()
    key = torch.full((n,), 0xDEAD, dtype=torch.int32, device="cuda")
    idx = torch.full((n,), 0xDEAD, dtype=torch.int32, device="cuda")
    cs = torch.full((ncell,), 0xDEAD, dtype=torch.int32, device="cuda")
    ce = torch.full((ncell,), 0xDEAD, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = sph.lib().sph_sort_cells_noalloc(C.byref(cfg), n, pos_d.data_ptr(), key.data_ptr(), idx.data_ptr(),
                                          cs.data_ptr(), ce.data_ptr(), C.c_void_p(stream))
    torch.cuda.synchronize()
    assert rc == _abi.SPH_OK
    as_u32 = lambda t: t.cpu().numpy().view(np.uint32)
    return as_u32(key), as_u32(idx), as_u32(cs), as_u32(ce)


@pytest.mark.parametrize("preset,scene", [(sph.PRESET_REF_3D2, scenes.ref_box_3d2),
                                          (sph.PRESET_REF_2D, scenes.ref_init_2d)])
def test_noalloc_sort_matches_step_sort_twice(preset, scene, gpu):
    cfg = sph.preset(preset)
    pos, vel, lvl = scene(cfg)
    ref = _existing_sort(cfg, pos, vel, lvl)
    for call in range(2):
        key, idx, cs, ce = _noalloc_sort(cfg, pos)
        assert np.array_equal(key, ref["hash"]), f"call {call}: cell keys differ"
        assert np.array_equal(idx, ref["index"]), f"call {call}: sorted index differs"
        assert np.array_equal(cs, ref["cell_start"]), f"call {call}: cell_start differs"
        assert np.array_equal(ce, ref["cell_end"]), f"call {call}: cell_end differs"


def test_noalloc_rejects_sizes_beyond_its_maximum(gpu):
    cfg = sph.preset(sph.PRESET_DAM_3D4)   # 1 048 576 cells > SPH_NOALLOC_MAX_CELLS
    rc = sph.lib().sph_sort_cells_noalloc(C.byref(cfg), 10, None, None, None, None, None, None)
    assert rc == _abi.SPH_ERR_RANGE
    cfg = sph.preset(sph.PRESET_REF_3D2)
    rc = sph.lib().sph_sort_cells_noalloc(C.byref(cfg), _abi.NOALLOC_MAX_PARTICLES + 1, None, None, None, None,
                                          None, None)
    assert rc == _abi.SPH_ERR_RANGE
