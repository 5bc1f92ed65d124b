"""GPU: the frame-loop program (``python -m nbodysim_b200.run``) against the
reference's own main() on the same settings file, its resume path, its images
and its overwrite rule."""
import os
import subprocess
import sys

import numpy as np
import pytest

from test_frames_io import ROOT, RUNNER

pytestmark = pytest.mark.gpu

CFG = ("use_seed true\nseed 12345\nnum_particles {n}\nnum_frames {frames}\ngen_type cube\nsize 64\ntheta 0.5\n"
       "dt 0.0333\ndump_binary true\nkeep_previous_binary true\ndump_text true\nkeep_previous_text true\n"
       "dump_image {image}\nimg_w 160\nimg_h 120\nprojection front\nbrightness 40\ndisplay_progress false\n"
       "overwrite_data {overwrite}\nthreads 1\ncuda false\nread_existing {resume}\nprecision fp64\n")


def write_cfg(d, n=1500, frames=3, image="false", overwrite="true", resume="false"):
    d.mkdir(parents=True, exist_ok=True)
    p = d / "settings.cfg"
    p.write_text(CFG.format(n=n, frames=frames, image=image, overwrite=overwrite, resume=resume))
    return p


def run_ours(d, cfg, check=True):
    env = dict(os.environ, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-m", "nbodysim_b200.run", str(cfg)], cwd=d, env=env, capture_output=True,
                       text=True, timeout=600)
    if check:
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r


def by_mass(rec):
    return rec[np.argsort(rec[:, 9])]


def test_frames_match_reference_main(nb, tmp_path):
    lib = os.path.join(ROOT, "oracle", "_ref", "libnbref.so")
    if not os.path.exists(lib):
        pytest.skip("reference harness not built (oracle/_ref)")
    ours, theirs = tmp_path / "ours", tmp_path / "ref"
    run_ours(ours, write_cfg(ours))
    cfg = write_cfg(theirs)
    (theirs / "data").mkdir()
    r = subprocess.run([sys.executable, "-c", RUNNER, lib, str(cfg)], cwd=theirs, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    for f in range(3):
        a = by_mass(np.fromfile(ours / "data" / f"{f:04d}.dat").reshape(-1, 10))
        b = by_mass(np.fromfile(theirs / "data" / f"{f:04d}.dat").reshape(-1, 10))
        assert np.array_equal(a[:, 9], b[:, 9])
        err = (np.abs(a[:, :6] - b[:, :6]).max(axis=0) / np.abs(b[:, :6]).max(axis=0)).max()
        assert err <= 1e-12, (f, err)
        assert len((ours / "data" / f"{f:04d}.txt").read_text().splitlines()) == 1500


def test_resume_continues_bit_for_bit(nb, tmp_path):
    straight, resumed = tmp_path / "straight", tmp_path / "resumed"
    run_ours(straight, write_cfg(straight, frames=4))
    run_ours(resumed, write_cfg(resumed, frames=2))
    r = run_ours(resumed, write_cfg(resumed, frames=4, resume="true"))
    assert "Resuming from 2" in r.stdout
    for f in (2, 3):
        assert (straight / "data" / f"{f:04d}.dat").read_bytes() == (resumed / "data" / f"{f:04d}.dat").read_bytes()


def test_images_and_overwrite_rule(nb, ref, tmp_path):
    d = tmp_path / "img"
    cfg = write_cfg(d, frames=2, image="true")
    run_ours(d, cfg)
    pos = np.fromfile(d / "data" / "0001.dat").reshape(-1, 10)[:, :3].copy()
    want = ref.write_image(pos, 160, 120, 0, 0, False, False, 1.0, 40.0)
    body = (d / "img" / "0001.ppm").read_bytes()
    head = b"P6\n160 120\n255\n"
    assert body.startswith(head)
    got = np.frombuffer(body[len(head):], np.uint8).reshape(120, 160, 3)[::-1]  # the PPM's top row is the bitmap's last
    assert np.array_equal(got, want)
    # overwrite disabled and the frame files exist: the program refuses, as the reference does
    r = run_ours(d, write_cfg(d, frames=2, image="true", overwrite="false"), check=False)
    assert r.returncode == 1 and "Overwrite disabled" in r.stderr
