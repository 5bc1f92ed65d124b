"""Drop-in: the reference's own unmodified main() (src/main.cpp:1359-1504),
compiled with the product's barnes_hut_cuda shim in place of its
src/cuda_helper.cpp + src/cuda_code.cu, runs a seeded simulation with
`cuda true` and must match the same program's CPU path (`cuda false`).

The program is run in a child process (it may exit() on errors) in a scratch
directory; its binary frame dumps (raw particle structs, src/main.cpp:730-743)
are matched particle by particle on their masses."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libnbref_gpu.so")
LIB_F32 = os.path.join(ROOT, "oracle", "_ref", "libnbref_gpu_f32.so")

RUNNER = r'''
import ctypes, sys
lib = ctypes.CDLL(sys.argv[1])
argv = (ctypes.c_char_p * 2)(b"nbodysim", sys.argv[2].encode())
sys.exit(lib.ref_main(2, argv))
'''


def run_main(tmp, cuda, gen_type, precision=None, frames=4, n=3000, lib=LIB, dtype=np.float64):
    d = tmp / ("gpu" if cuda else "cpu")
    (d / "data").mkdir(parents=True)
    cfg = d / "settings.cfg"
    cfg.write_text(f"use_seed true\nseed 3735928559\nnum_particles {n}\nnum_frames {frames}\n"
                   f"gen_type {gen_type}\nsize 512\ntheta 0.5\ndt 0.0333\ndump_binary true\n"
                   "keep_previous_binary true\ndump_text false\ndump_image false\ndisplay_progress false\n"
                   f"overwrite_data true\nthreads 1\ncuda {'true' if cuda else 'false'}\n")
    env = dict(os.environ)
    if precision:
        env["NBODY_B200_PRECISION"] = precision
    r = subprocess.run([sys.executable, "-c", RUNNER, lib, str(cfg)], cwd=d, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = []
    for f in range(frames):
        raw = np.fromfile(d / "data" / f"{f:04d}.dat", dtype=dtype).reshape(-1, 10).astype(np.float64)
        out.append(raw[np.argsort(raw[:, 9])])  # order by mass: unique per particle
    return out


@pytest.fixture(scope="module")
def dropin_lib(nb):
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libnbref_gpu.so not built (needs the reference tree at build time)")
    return LIB


@pytest.mark.parametrize("gen_type,precision,tol", [("cube", "fp64", 1e-12), ("sphere", None, 1e-6)])
def test_reference_main_with_gpu_shim_matches_cpu(dropin_lib, tmp_path, gen_type, precision, tol):
    cpu = run_main(tmp_path, False, gen_type)
    gpu = run_main(tmp_path, True, gen_type, precision)
    for f, (c, g) in enumerate(zip(cpu, gpu)):
        assert np.array_equal(c[:, 9], g[:, 9])
        scale = np.abs(c[:, 0:3]).max()
        err = np.abs(c[:, 0:3] - g[:, 0:3]).max() / scale
        assert err <= tol, (f, err)
        # accelerations of the last force pass (the field the shim overwrites)
        acc_c, acc_g = c[:, 6:9], g[:, 6:9]
        rel = np.linalg.norm(acc_c - acc_g, axis=1) / np.linalg.norm(acc_c, axis=1)
        assert np.percentile(rel, 99) <= (1e-12 if precision else 1e-5), (f, np.percentile(rel, 99))


@pytest.mark.parametrize("gen_type,precision", [("cube", None), ("cube", "fp64"), ("sphere", None)])
def test_float_build_main_with_gpu_shim(nb, tmp_path, gen_type, precision):
    """The reference's FLOAT build (what its makefile ships) with the shim. The
    shim passes sizeof(datatype) to the library, which then builds the float
    tree and takes every opening decision as the FLOAT build does; the frames
    agree with the FLOAT CPU path to float rounding of the summation order."""
    if not os.path.exists(LIB_F32):
        pytest.skip("oracle/_ref/libnbref_gpu_f32.so not built (needs the reference tree at build time)")
    cpu = run_main(tmp_path / "f32", False, gen_type, lib=LIB_F32, dtype=np.float32)
    gpu = run_main(tmp_path / "f32", True, gen_type, precision=precision, lib=LIB_F32, dtype=np.float32)
    for f, (c, g) in enumerate(zip(cpu, gpu)):
        assert np.array_equal(c[:, 9], g[:, 9])
        err = np.abs(c[:, 0:3] - g[:, 0:3]).max() / np.abs(c[:, 0:3]).max()
        assert err <= 1e-6, (f, err)
        rel = np.linalg.norm(c[:, 6:9] - g[:, 6:9], axis=1) / np.linalg.norm(c[:, 6:9], axis=1)
        assert np.percentile(rel, 99) <= 1e-5, (f, np.percentile(rel, 99))
