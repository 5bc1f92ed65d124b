"""Host-side checks that need no GPU: the C-ABI library loads and exports every
entry point include/nbody_b200.h declares; the host generator is bit-identical
to the oracle; argument and device errors come back as status codes; the
settings parser mirrors the reference's keys."""
import ctypes as C

import numpy as np
import pytest


def test_library_exports_every_declared_symbol(nb):
    lib = nb.load_library()
    syms = nb.header_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(nb._SIGS), "ctypes signatures missing for some declared entry points"


def test_no_device_is_a_status_not_an_abort(nb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(nb.NBodyError) as e:
        nb.Engine()
    assert e.value.status == nb.ERR_NO_DEVICE


def test_status_strings(nb):
    lib = nb.load_library()
    for s in range(0, 9):
        assert lib.nbody_status_string(s)
    assert lib.nbody_status_string(99) == b"unknown status"


def test_invalid_params_rejected_before_device(nb):
    lib = nb.load_library()
    p = nb.default_params(theta=-1.0)
    h = C.c_void_p()
    assert lib.nbody_create(C.byref(p), C.byref(h)) == nb.ERR_INVALID
    p = nb.default_params(precision=7)
    assert lib.nbody_create(C.byref(p), C.byref(h)) == nb.ERR_INVALID
    assert lib.nbody_create(None, C.byref(h)) == nb.ERR_INVALID


def test_default_params_match_reference_defaults(nb):
    p = nb.default_params()
    assert (p.theta, p.dt, p.damping) == (0.5, 0.0333, 0)            # src/main.cpp:1327-1328,1343
    assert (p.min_adaptive_dt, p.max_pos_change, p.max_vel_change) == (0.00333, 3.0, 3.0)  # README.md:54-60


@pytest.mark.parametrize("gt", [0, 1, 2])
@pytest.mark.parametrize("md", [0, 1, 2])
def test_generator_bit_identical(nb, orc, oracle_mod, gt, md):
    p, v, m = nb.generate(2000, gen_type=gt, mass_dist=md, min_vel=1.0, max_vel=5.0, scale=(1.0, 0.5, 2.0))
    q = orc.generate(oracle_mod.GenParams(gen_type=gt, mass_dist=md, min_vel=1.0, max_vel=5.0,
                                          scale=(1.0, 0.5, 2.0)), 2000)
    for a, b in zip((p, v, m), q):
        assert np.array_equal(a, b)


def test_generator_golden(nb, golden):
    g = golden("generate.npz")
    for gt in (0, 1, 2):
        for md in (0, 1, 2):
            p, v, m = nb.generate(64, gen_type=gt, mass_dist=md, min_vel=1.0, max_vel=5.0)
            assert np.array_equal(p, g[f"gen_{gt}_{md}_pos"]) and np.array_equal(m, g[f"gen_{gt}_{md}_mass"])


def test_generator_rejects_bad_args(nb):
    with pytest.raises(nb.NBodyError):
        nb.generate(4, gen_type=5)
    with pytest.raises(nb.NBodyError):
        nb.generate(4, scale=(-1.0, 1.0, 1.0))


def test_settings_parser_reference_file_format(tmp_path):
    from nbodysim_b200.settings import read_settings
    f = tmp_path / "s.cfg"
    f.write_text("read_existing true\nnum_particles 50000\ntheta 0.3\ngen_type shell\nmass_dist exp\n"
                 "rotation_vector 0 1 0\nscale_z 0.2\ndamping true\nthreads 8\nbogus 1\nfalse\n"
                 "adaptive true\nmax_pos_change 2.5\nprecision fp64\nseed 3735928559\n")
    msgs = []
    s = read_settings(str(f), warn=msgs.append)
    assert s.read_existing and s.num_particles == 50000 and s.theta == 0.3
    assert s.gen_type == 2 and s.mass_dist == 1 and s.rotation_vector == (0.0, 1.0, 0.0)
    assert s.scale_z == 0.2 and s.damping and s.threads == 8 and s.adaptive and s.max_pos_change == 2.5
    assert s.precision == 1 and s.seed == 0xDEADBEEF
    assert any("Unrecognized variable bogus" in m for m in msgs)


def test_settings_defaults_match_reference():
    from nbodysim_b200.settings import set_default
    s = set_default()
    assert (s.num_particles, s.num_frames, s.size, s.theta, s.dt, s.seed) == (5000, 300, 512, 0.5, 0.0333, 0xDEADBEEF)
    assert (s.min_mass, s.max_mass, s.r_sphere, s.rotation_magnitude) == (5e10, 5e11, 100, 0.1)
    assert s.threads == 1 and not s.cuda and not s.collide
