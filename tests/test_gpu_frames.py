"""GPU: frame files from and into the resident state. The reference's own
main() (CPU path) writes frames 0-3; the engine resumes from frame 1 the way
read_data does and must reproduce frames 2 and 3 (FP64 form)."""
import os

import numpy as np
import pytest

from test_frames_io import ROOT, run_reference

pytestmark = pytest.mark.gpu


def by_mass(rec):
    return rec[np.argsort(rec[:, 9])]  # masses are unique per particle


def test_resume_from_reference_frames(nb, tmp_path):
    lib = os.path.join(ROOT, "oracle", "_ref", "libnbref.so")
    if not os.path.exists(lib):
        pytest.skip("reference harness not built (oracle/_ref)")
    data = run_reference(lib, tmp_path / "ref", frames=4, n=2000, gen_type="cube")
    frames = [np.fromfile(data / f"{f:04d}.dat").reshape(-1, 10) for f in range(4)]
    resume = tmp_path / "resume"
    resume.mkdir()
    (resume / "0001.dat").write_bytes((data / "0001.dat").read_bytes())
    with nb.Engine(precision=nb.PRECISION_FP64) as e:
        assert e.load_frame(str(resume), 10) == 2
        for f in (2, 3):
            e.step(1)
            e.save_frame(str(resume), f, binary=True, text=True)
            got = by_mass(np.fromfile(resume / f"{f:04d}.dat").reshape(-1, 10))
            want = by_mass(frames[f])
            assert np.array_equal(got[:, 9], want[:, 9])
            scale = np.abs(want[:, :9]).max(axis=0)
            err = (np.abs(got[:, :9] - want[:, :9]).max(axis=0) / scale).max()
            assert err <= 1e-12, (f, err)
            txt = (resume / f"{f:04d}.txt").read_text().splitlines()
            assert len(txt) == 2000 and txt[0].count(", ") == 2
    with nb.Engine() as e:
        assert e.load_frame(str(tmp_path / "ref" / "nothing_here"), 5) == 0


def test_save_load_round_trip(nb, tmp_path):
    pos, vel, mass = nb.generate(5000, gen_type=2)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        e.step(2)
        e.save_frame(str(tmp_path), 7)
        p, v, a = e.get_particles(acc=True)
    q, w, b, m = nb.read_dat(str(tmp_path / "0007.dat"))
    assert np.array_equal(q, p) and np.array_equal(w, v) and np.array_equal(b, a) and np.array_equal(m, mass)
    with nb.Engine() as e:
        assert e.load_frame(str(tmp_path), 9) == 8
        q2, w2 = e.get_particles()
    assert np.array_equal(q2, p) and np.array_equal(w2, v)
