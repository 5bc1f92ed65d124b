"""The allocation-free entry point (include/nbody_b200_noalloc.h).

For callers that cannot call cudaMalloc (stream capture, frameworks that own
all device memory, allocation-free loops): nbody_root_cube_noalloc computes
the reference's root cube over the caller's device arrays using scratch that
lives inside the library. Checked through the C ABI against the root cube the
regular entry point reports, on two calls in a row (the scratch is reused).
This file sorts last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out_dev):
    lib = nb.load_library()
    return lib.nbody_root_cube_noalloc(C.c_void_p(pos_dev.data_ptr()), C.c_void_p(mass_dev.data_ptr()), n,
                                       C.c_void_p(out_dev.data_ptr()),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_root_cube_noalloc_matches_regular_entry_point(nb):
    import torch
    lib = nb.load_library()
    for gen_type, n in ((0, 5000), (2, 70000)):
        pos, vel, mass = nb.generate(n, gen_type=gen_type, size=1024.0)
        with nb.Engine() as e:
            e.barnes_hut(pos, mass)
            st = e.stats()
        pos_dev = torch.from_numpy(pos).cuda()
        mass_dev = torch.from_numpy(mass).cuda()
        for call in range(2):  # the second call reuses the scratch left by the first
            out = torch.full((5,), -7.0, dtype=torch.float64, device="cuda")
            assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out) == nb.OK
            torch.cuda.synchronize()
            o = out.cpu().numpy()
            # min/max reductions are exact: the tolerance is zero
            assert np.array_equal(o[:3], np.array(st["root_center"])), (call, o, st["root_center"])
            assert o[3] == st["root_side"], (call, o[3], st["root_side"])
            assert o[4] == 0.0
    assert lib.nbody_root_cube_noalloc_max_n() == 4 * 1024 * 1024


def test_root_cube_noalloc_limits_and_flags(nb):
    import torch
    lib = nb.load_library()
    pos, _, mass = nb.generate(100)
    pos[17, 2] = np.inf
    pos_dev = torch.from_numpy(pos).cuda()
    mass_dev = torch.from_numpy(mass).cuda()
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, 100, out) == nb.OK
    torch.cuda.synchronize()
    assert out[4].item() == 1.0
    too_many = lib.nbody_root_cube_noalloc_max_n() + 1
    assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, too_many, out) == nb.ERR_INVALID
    assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, 0, out) == nb.ERR_INVALID
    assert lib.nbody_root_cube_noalloc(None, C.c_void_p(mass_dev.data_ptr()), 100,
                                       C.c_void_p(out.data_ptr()), None) == nb.ERR_INVALID
