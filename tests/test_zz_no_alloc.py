"""The allocation-free entry point (include/nbody_b200_noalloc.h).

For callers that cannot call cudaMalloc (stream capture, frameworks that own
all device memory, allocation-free loops): nbody_root_cube_noalloc computes
the reference's root cube over the caller's device arrays using scratch that
lives inside the library. Checked through the C ABI against the root cube the
regular entry point reports: on two calls in a row (the scratch is reused),
when captured into a CUDA graph and replayed on new contents, and across a
device reset and new driver-API contexts, which each hold their own instance
of the scratch array. This file sorts last so that a failure here comes after
every other test.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out_dev):
    lib = nb.load_library()
    return lib.nbody_root_cube_noalloc(C.c_void_p(pos_dev.data_ptr()), C.c_void_p(mass_dev.data_ptr()), n,
                                       C.c_void_p(out_dev.data_ptr()),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _regular_root_cube(nb, pos, mass):
    with nb.Engine() as e:
        e.barnes_hut(pos, mass)
        st = e.stats()
    return np.array(list(st["root_center"]) + [st["root_side"], 0.0])


def test_root_cube_noalloc_matches_regular_entry_point(nb):
    import torch
    lib = nb.load_library()
    for gen_type, n in ((0, 5000), (2, 70000)):
        pos, vel, mass = nb.generate(n, gen_type=gen_type, size=1024.0)
        want = _regular_root_cube(nb, pos, mass)
        pos_dev = torch.from_numpy(pos).cuda()
        mass_dev = torch.from_numpy(mass).cuda()
        for call in range(2):  # the second call reuses the scratch left by the first
            out = torch.full((5,), -7.0, dtype=torch.float64, device="cuda")
            assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out) == nb.OK
            torch.cuda.synchronize()
            # min/max reductions are exact: the tolerance is zero
            assert np.array_equal(out.cpu().numpy(), want), (call, out.cpu().numpy(), want)
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
    o = out.cpu().numpy()
    assert o[4] == 1.0 and np.isnan(o[:4]).all(), o  # a poisoned cube cannot be used by mistake
    too_many = lib.nbody_root_cube_noalloc_max_n() + 1
    assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, too_many, out) == nb.ERR_INVALID
    assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, 0, out) == nb.ERR_INVALID
    assert lib.nbody_root_cube_noalloc(None, C.c_void_p(mass_dev.data_ptr()), 100,
                                       C.c_void_p(out.data_ptr()), None) == nb.ERR_INVALID


def test_root_cube_noalloc_in_a_captured_graph(nb):
    """One warm-up call, then one call captured into a CUDA graph; the graph is
    replayed on new particle contents and matches the regular entry point."""
    import torch
    n = 20000
    pos0, _, mass0 = nb.generate(n, gen_type=1, size=512.0)
    pos_dev = torch.from_numpy(pos0).cuda()
    mass_dev = torch.from_numpy(mass0).cuda()
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        assert _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out) == nb.OK
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = _root_cube_noalloc(nb, torch, pos_dev, mass_dev, n, out)
    assert rc == nb.OK
    for seed, gen_type in ((11, 2), (12, 0)):
        pos, _, mass = nb.generate(n, gen_type=gen_type, size=1024.0, seed=seed)
        pos_dev.copy_(torch.from_numpy(pos))
        mass_dev.copy_(torch.from_numpy(mass))
        out.fill_(-7.0)
        g.replay()
        torch.cuda.synchronize()
        want = _regular_root_cube(nb, pos, mass)
        assert np.array_equal(out.cpu().numpy(), want), (seed, out.cpu().numpy(), want)
    del g


# Runs in a fresh process: the caller owns its memory through the shared CUDA
# runtime (as the reference's program does) and resets the device between
# calls; then it runs two calls in contexts it creates with the driver API.
_CHILD = r"""
import ctypes as C, glob, os, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import nbodysim_b200 as nb

lib = nb.load_library()
n = 70000
pos, _, mass = nb.generate(n, gen_type=2, size=1024.0)
with nb.Engine() as e:
    e.barnes_hut(pos, mass)
    st = e.stats()
want = np.array(list(st["root_center"]) + [st["root_side"], 0.0])

cands = sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so.12*"))
rt = C.CDLL(cands[0])
H2D, D2H = 1, 2

def call_runtime():
    p, m, o = C.c_void_p(), C.c_void_p(), C.c_void_p()
    for ptr, size in ((p, pos.nbytes), (m, mass.nbytes), (o, 40)):
        assert rt.cudaMalloc(C.byref(ptr), C.c_size_t(size)) == 0
    assert rt.cudaMemcpy(p, C.c_void_p(pos.ctypes.data), C.c_size_t(pos.nbytes), H2D) == 0
    assert rt.cudaMemcpy(m, C.c_void_p(mass.ctypes.data), C.c_size_t(mass.nbytes), H2D) == 0
    rc = lib.nbody_root_cube_noalloc(p, m, n, o, None)
    assert rt.cudaDeviceSynchronize() == 0
    out = np.zeros(5)
    assert rt.cudaMemcpy(C.c_void_p(out.ctypes.data), o, C.c_size_t(40), D2H) == 0
    for ptr in (p, m, o):
        rt.cudaFree(ptr)
    return rc, out

cu = C.CDLL("libcuda.so.1")
assert cu.cuInit(0) == 0
dev = C.c_int()
assert cu.cuDeviceGet(C.byref(dev), 0) == 0

def call_driver_context():
    ctx = C.c_void_p()
    assert cu.cuCtxCreate_v2(C.byref(ctx), 0, dev) == 0
    p, m, o = C.c_uint64(), C.c_uint64(), C.c_uint64()
    for ptr, size in ((p, pos.nbytes), (m, mass.nbytes), (o, 40)):
        assert cu.cuMemAlloc_v2(C.byref(ptr), C.c_size_t(size)) == 0
    assert cu.cuMemcpyHtoD_v2(p, C.c_void_p(pos.ctypes.data), C.c_size_t(pos.nbytes)) == 0
    assert cu.cuMemcpyHtoD_v2(m, C.c_void_p(mass.ctypes.data), C.c_size_t(mass.nbytes)) == 0
    rc = lib.nbody_root_cube_noalloc(C.c_void_p(p.value), C.c_void_p(m.value), n, C.c_void_p(o.value), None)
    assert cu.cuCtxSynchronize() == 0
    out = np.zeros(5)
    assert cu.cuMemcpyDtoH_v2(C.c_void_p(out.ctypes.data), o, C.c_size_t(40)) == 0
    for ptr in (p, m, o):
        cu.cuMemFree_v2(ptr)
    assert cu.cuCtxDestroy_v2(ctx) == 0
    return rc, out

results = []
results.append(("before reset",) + call_runtime())
assert rt.cudaDeviceReset() == 0
results.append(("after reset",) + call_runtime())
results.append(("driver context 1",) + call_driver_context())
results.append(("driver context 2",) + call_driver_context())
bad = [(name, rc, out) for name, rc, out in results if rc != 0 or not np.array_equal(out, want)]
for name, rc, out in results:
    print(name, rc, out.tolist())
print("want", want.tolist())
sys.exit(1 if bad else 0)
"""


def test_root_cube_noalloc_across_reset_and_contexts(nb):
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
