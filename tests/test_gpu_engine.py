"""GPU: resident-state stepping, frame-loop parity, adaptive dt, diagnostics."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_frames_match_reference_fp64(nb, golden):
    g = golden("frames_cube256.npz")
    with nb.Engine(precision=nb.PRECISION_FP64) as e:
        e.set_particles(g["pos"], g["vel"], g["mass"])
        for f in range(5):
            e.step(1)
            p, v = e.get_particles()
            err = np.abs(p - g["frames"][f]).max() / np.abs(g["frames"][f]).max()
            assert err <= 1e-13, (f, err)


def test_frames_match_oracle_mixed(nb, orc):
    pos, vel, mass = nb.generate(2000)
    _, _, frames = orc.run_frames(pos, vel, mass, 10, keep_frames=True)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        for f in range(10):
            e.step(1)
        p, v = e.get_particles()
    err = np.linalg.norm(p - frames[-1], axis=1).max()
    assert err <= 1e-6 * np.abs(frames[-1]).max(), err


@pytest.mark.parametrize("adaptive", [0, 1])
def test_step_host_overlapped_upload_equals_resident(nb, adaptive):
    """From 65,536 particles nbody_step_host uploads the masses and velocities on
    a second stream during the force pass; the result must not change."""
    pos, vel, mass = nb.generate(70000, gen_type=1, min_vel=0.0, max_vel=2.0)
    with nb.Engine(adaptive=adaptive) as e:
        e.set_particles(pos, vel, mass)
        e.step(2)
        p1, v1 = e.get_particles()
        dt1 = e.stats()["last_dt"]
        p2, v2 = pos.copy(), vel.copy()
        e.step_host(p2, v2, mass, 1)
        e.step_host(p2, v2, mass, 1)
        dt2 = e.stats()["last_dt"]
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2) and dt1 == dt2


def test_step_host_overlapped_nonfinite_mass(nb):
    """A non-finite mass that arrives on the second stream is still reported, and
    the context stays usable."""
    pos, vel, mass = nb.generate(70000, gen_type=1)
    bad = mass.copy()
    bad[12345] = np.nan
    with nb.Engine() as e:
        p, v = pos.copy(), vel.copy()
        with pytest.raises(nb.NBodyError) as ex:
            e.step_host(p, v, bad, 1)
        assert ex.value.status == nb.ERR_NONFINITE
        p, v = pos.copy(), vel.copy()
        e.step_host(p, v, mass, 1)
        assert np.isfinite(p).all() and np.isfinite(v).all()


def test_step_host_equals_resident(nb):
    pos, vel, mass = nb.generate(3000, gen_type=1)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        e.step(3)
        p1, v1 = e.get_particles()
        p2, v2 = pos.copy(), vel.copy()
        e.step_host(p2, v2, mass, 3)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_single_step_is_reference_update(nb, orc):
    pos, vel, mass = nb.generate(4000, gen_type=1)
    with nb.Engine(precision=nb.PRECISION_FP64) as e:
        e.set_particles(pos, vel, mass)
        e.step(1)
        p, v = e.get_particles()
    acc, _ = orc.forces(pos, mass, 0.5)
    rp, rv = orc.update(pos, vel, acc, 0.0333)
    assert np.abs(p - rp).max() <= 1e-12 * np.abs(rp).max()
    assert np.abs(v - rv).max() <= 1e-10 * np.abs(rv).max()


def test_adaptive_dt_rule(nb):
    pos, vel, mass = nb.generate(5000, gen_type=2, size=1024)
    with nb.Engine(adaptive=1, max_pos_change=0.05, max_vel_change=3.0, min_adaptive_dt=1e-4) as e:
        acc = e.barnes_hut(pos, mass)
        e.set_particles(pos, vel, mass)
        e.step(1)
        dt = e.stats()["last_dt"]
    amax = np.linalg.norm(acc, axis=1).max()
    vmax = np.linalg.norm(vel, axis=1).max()
    expect = min(0.0333, 3.0 / amax, 0.05 / vmax)
    expect = min(max(expect, 1e-4), 0.0333)
    assert abs(dt - expect) <= 1e-6 * expect


def test_diagnostics(nb, orc):
    pos, vel, mass = nb.generate(3000, gen_type=1)
    with nb.Engine() as e, nb.Engine(precision=nb.PRECISION_FP64) as e64:
        e.set_particles(pos, vel, mass)
        e64.set_particles(pos, vel, mass)
        d = e.diagnostics()
        d64 = e64.diagnostics()
    ke = 0.5 * np.sum(mass * np.sum(vel * vel, 1))
    assert abs(d["kinetic"] - ke) <= 1e-12 * ke
    P = (mass[:, None] * vel).sum(0)
    L = (mass[:, None] * np.cross(pos, vel)).sum(0)
    assert np.allclose(d["momentum"], P, rtol=1e-10, atol=1e-10 * np.abs(mass[:, None] * vel).sum())
    assert np.allclose(d["angular_momentum"], L, rtol=1e-10)
    assert abs(d["mass"] - mass.sum()) <= 1e-12 * mass.sum()
    # potential: the MIXED form's diagnostics sum FP64 pair terms over the same lists as
    # the FP64 form, so the two agree to FP64 rounding; vs direct-sum FP64 within the BH truncation
    assert abs(d["potential"] - d64["potential"]) <= 1e-10 * abs(d64["potential"])
    G = 6.67384e-11
    r = np.linalg.norm(pos[:, None, :] - pos[None, :, :], axis=2)
    np.fill_diagonal(r, np.inf)
    pe = -0.5 * G * np.sum(mass[:, None] * mass[None, :] / r)
    assert abs(d64["potential"] - pe) <= 1e-2 * abs(pe)


def test_diagnostics_keep_mixed_accelerations(nb):
    """The FP64 potential pass of a MIXED context leaves its accelerations alone."""
    pos, vel, mass = nb.generate(5000, gen_type=2, size=1024.0)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        e.compute_forces()
        _, _, a0 = e.get_particles(acc=True)
        d = e.diagnostics()
        _, _, a1 = e.get_particles(acc=True)
        assert np.array_equal(a0, a1) and np.isfinite(d["potential"]) and d["potential"] < 0


def test_device_view(nb):
    pos, vel, mass = nb.generate(100)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        v = e.device_view()
        assert v.n == 100 and v.pos and v.vel and v.mass and v.acc and v.acc_is_double == 0


def test_state_errors(nb):
    with nb.Engine() as e:
        with pytest.raises(nb.NBodyError) as ex:
            e.step(1)
        assert ex.value.status == nb.ERR_STATE


def test_step_host_on_a_caller_stream(nb):
    """nbody_set_stream: the engine orders its work (and the overlapped velocity
    upload of nbody_step_host) after the caller's stream."""
    import ctypes
    import torch
    pos, vel, mass = nb.generate(70000, gen_type=2, size=1024.0)
    s = torch.cuda.Stream()
    with nb.Engine(adaptive=1) as e, nb.Engine(adaptive=1) as ref:
        assert e._lib.nbody_set_stream(e._h, ctypes.c_void_p(s.cuda_stream)) == nb.OK
        p1, v1 = pos.copy(), vel.copy()
        e.step_host(p1, v1, mass, 2)
        ref.set_particles(pos, vel, mass)
        ref.step(2)
        p2, v2 = ref.get_particles()
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("stream", [0, 2])  # the legacy default stream, the per-thread default stream
def test_steps_on_the_default_streams(nb, stream):
    """On the default streams the chained launches (and, on the per-thread
    stream, the captured graphs; the legacy stream is not captured) give the same
    steps as the engine's own stream."""
    import ctypes
    pos, vel, mass = nb.generate(30000, gen_type=2, size=1024.0, seed=3)
    with nb.Engine(adaptive=1) as e, nb.Engine(adaptive=1) as ref:
        assert e._lib.nbody_set_stream(e._h, ctypes.c_void_p(stream)) == nb.OK
        e.set_particles(pos, vel, mass)
        e.step(3)
        p1, v1 = e.get_particles()
        ref.set_particles(pos, vel, mass)
        ref.step(3)
        p2, v2 = ref.get_particles()
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


@pytest.mark.parametrize("precision", [0, 1])
def test_walk_stats_switch_keeps_results(nb, precision):
    """The walk's statistics come from their own kernel instance, switched on by
    nbody_set_walk_stats: forces and counts are the same with and without it."""
    pos, _, mass = nb.generate(20000, gen_type=2, size=1024.0, seed=11)
    with nb.Engine(precision=precision) as e:
        a0, c0 = e.barnes_hut(pos, mass, counts=True)
        s0 = e.stats()
        assert s0["walk_entries"] == 0 and s0["walk_tiles"] == 0 and s0["max_stack"] == 0
        e.set_walk_stats(True)
        a1, c1 = e.barnes_hut(pos, mass, counts=True)
        s1 = e.stats()
        assert s1["walk_entries"] > 0 and s1["walk_tiles"] > 0 and s1["walk_list"] > 0 and s1["max_stack"] > 0
        assert s1["interactions"] == s0["interactions"] == int(c0.sum())
    assert np.array_equal(a0, a1) and np.array_equal(c0, c1)
