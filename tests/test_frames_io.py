"""Frame files: the reference's own main() writes binary and text frames (CPU
path, both the DOUBLE and the FLOAT build); the library reads them back,
rewrites them byte for byte, and finds the resume frame the way read_data does
(src/main.cpp:283-291, 730-759, 790-811)."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RUNNER = r'''
import ctypes, sys
lib = ctypes.CDLL(sys.argv[1])
argv = (ctypes.c_char_p * 2)(b"nbodysim", sys.argv[2].encode())
sys.exit(lib.ref_main(2, argv))
'''


def run_reference(lib, d, frames=3, n=400, gen_type="sphere"):
    (d / "data").mkdir(parents=True)
    cfg = d / "settings.cfg"
    cfg.write_text(f"use_seed true\nseed 12345\nnum_particles {n}\nnum_frames {frames}\n"
                   f"gen_type {gen_type}\nsize 512\ntheta 0.5\ndt 0.0333\ndump_binary true\n"
                   "keep_previous_binary true\ndump_text true\nkeep_previous_text true\ndump_image false\n"
                   "display_progress false\noverwrite_data true\nthreads 1\ncuda false\n")
    r = subprocess.run([sys.executable, "-c", RUNNER, lib, str(cfg)], cwd=d, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return d / "data"


@pytest.mark.parametrize("lib_name,dtype,nbytes", [("libnbref.so", np.float64, 8), ("libnbref_f32.so", np.float32, 4)])
def test_reference_frames_round_trip(nb, oracle_mod, tmp_path, lib_name, dtype, nbytes):
    lib = os.path.join(ROOT, "oracle", "_ref", lib_name)
    if not os.path.exists(lib):
        pytest.skip("reference harness not built (oracle/_ref)")
    data = run_reference(lib, tmp_path)
    for f in range(3):
        dat = str(data / f"{f:04d}.dat")
        assert nb.frame_path(str(data), f, True) == dat
        raw = np.fromfile(dat, dtype=dtype).reshape(-1, 10).astype(np.float64)
        pos, vel, acc, mass = nb.read_dat(dat, nbytes)
        assert np.array_equal(pos, raw[:, 0:3]) and np.array_equal(vel, raw[:, 3:6])
        assert np.array_equal(acc, raw[:, 6:9]) and np.array_equal(mass, raw[:, 9])
        out = tmp_path / f"re{f}.dat"
        nb.write_dat(str(out), pos, vel, mass, acc=acc, datatype_bytes=nbytes)
        assert out.read_bytes() == (data / f"{f:04d}.dat").read_bytes()
        txt = tmp_path / f"re{f}.txt"
        nb.write_txt(str(txt), pos, datatype_bytes=nbytes)
        assert txt.read_bytes() == (data / f"{f:04d}.txt").read_bytes()
    assert nb.find_resume_frame(str(data), 10) == 2
    assert nb.find_resume_frame(str(data), 1) == 1
    os.remove(data / "0002.dat")
    assert nb.find_resume_frame(str(data), 10) == 1


def test_frame_helpers(nb, tmp_path):
    assert nb.frame_path(None, 7, True) == "./data/0007.dat"
    assert nb.frame_path("d", 12345, False) == "d/12345.txt"
    assert nb.find_resume_frame(str(tmp_path), 5) == -1
    rng = np.random.default_rng(3)
    pos, vel, mass = rng.normal(size=(50, 3)), rng.normal(size=(50, 3)), rng.random(50)
    p = str(tmp_path / "0000.dat")
    nb.write_dat(p, pos, vel, mass)  # no accelerations: zeros
    q, v, a, m = nb.read_dat(p)
    assert np.array_equal(q, pos) and np.array_equal(v, vel) and not a.any() and np.array_equal(m, mass)
    nb.write_dat(p, pos, vel, mass, datatype_bytes=4)
    q, _, _, m = nb.read_dat(p, 4)
    assert np.array_equal(q, pos.astype(np.float32).astype(np.float64))
    with pytest.raises(nb.NBodyError):
        nb.write_dat(p, pos, vel, mass, datatype_bytes=2)
    with pytest.raises(nb.NBodyError):
        nb.read_dat(str(tmp_path / "missing.dat"))
    rgb = rng.integers(0, 256, size=(3, 4, 3), dtype=np.uint8)
    ppm = tmp_path / "i.ppm"
    nb.write_ppm(str(ppm), rgb)
    body = ppm.read_bytes()
    assert body.startswith(b"P6\n4 3\n255\n")
    assert body[len(b"P6\n4 3\n255\n"):] == rgb[::-1].tobytes()  # bitmap row 0 is the bottom row
