"""GPU parity with the reference's FLOAT build (-DFLOAT, the build its makefile
ships): the library with nbody_params.datatype_bytes = 4, through the C ABI,
against the oracle's FLOAT path (oracle/bh_oracle.c *_f32, pinned bit for bit to
the FLOAT reference in tests/test_oracle_pins.py).

Bars: per-particle accepted-node counts EQUAL the FLOAT build's; accelerations
within p99 relative error 1e-5 of the FLOAT build's (P99_MIXED: FP32 pair
forces; the FP64 form's FP64 pair sums on the same float tree differ from the
float reference only by the reference's own float rounding, P99_FP64); the
root cube equal; the update rounded as the FLOAT build rounds it. The inputs
include a split-plane set on which over a thousand particles accept different
nodes in the FLOAT and DOUBLE builds, so the DOUBLE decisions would fail it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P99_MIXED = 1e-5
P99_FP64 = 1e-5


def rel(a, b):
    den = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(den > 0, den, 1.0)


@pytest.fixture(scope="module")
def engines(nb):
    e32 = nb.Engine(datatype_bytes=4)
    e64 = nb.Engine(datatype_bytes=4, precision=nb.PRECISION_FP64)
    yield e32, e64
    e32.close()
    e64.close()


@pytest.mark.parametrize("theta,damp", [(0.3, False), (0.5, False), (0.7, False), (0.5, True)])
def test_split_plane_set_counts_and_forces(nb, orc, golden, engines, theta, damp):
    g = golden("forces_float.npz")
    pos, mass = g["split_pos"], g["split_mass"]
    ref = g["split_acc_damped_0.5"] if damp else g[f"split_acc_{theta}"]
    _, rc = orc.forces(pos, mass, theta, damping=damp, single=True)
    _, rc64 = orc.forces(pos, mass, theta, damping=damp)
    assert (rc != rc64).sum() > 500  # the DOUBLE build's decisions differ here
    for e, bar in zip(engines, (P99_MIXED, P99_FP64)):
        acc, cnt = e.barnes_hut(pos, mass, damping=damp, theta=theta, counts=True)
        assert np.array_equal(cnt, rc), f"{np.count_nonzero(cnt != rc)} particles differ in accepted-node count"
        err = rel(acc, ref)
        assert np.percentile(err, 99) <= bar, (np.percentile(err, 99), err.max())
        st = e.stats()
        c, s = orc.root_cube(pos, single=True)
        assert np.array_equal(np.array(st["root_center"]), c) and st["root_side"] == s


CASES = [  # gen_type, n, theta, damping
    (0, 50000, 0.5, False), (1, 100000, 0.5, False), (2, 100000, 0.5, False),
    (2, 20000, 0.3, False), (0, 5000, 0.7, True), (1, 33, 0.5, False),
]


@pytest.mark.parametrize("gt,n,theta,damp", CASES)
def test_generated_counts_and_forces(nb, orc, engines, gt, n, theta, damp):
    pos, vel, mass = nb.generate(n, gen_type=gt, size=1024 if gt else 512)
    ra, rc = orc.forces(pos, mass, theta, damping=damp, single=True)
    for e, bar in zip(engines, (P99_MIXED, P99_FP64)):
        acc, cnt = e.barnes_hut(pos, mass, damping=damp, theta=theta, counts=True)
        assert np.array_equal(cnt, rc), f"{np.count_nonzero(cnt != rc)} particles differ in accepted-node count"
        err = rel(acc, ra)
        assert np.percentile(err, 99) <= bar, (np.percentile(err, 99), err.max())
        assert e.stats()["interactions"] == int(rc.sum())


def test_lattice_float_build(nb, orc, golden, engines):
    """Particles exactly on split planes: the strict '>' rule with float centres."""
    for k in (3, 4):
        g = golden(f"forces_lattice{k}.npz")
        for th in (0.5, 0.3):
            ra, rc = orc.forces(g["pos"], g["mass"], th, single=True)
            scale = np.linalg.norm(ra, axis=1).max()
            for e in engines:
                acc, cnt = e.barnes_hut(g["pos"], g["mass"], theta=th, counts=True)
                assert np.array_equal(cnt, rc)
                assert np.abs(acc - ra).max() <= 1e-5 * scale


def test_float_update_and_frames(nb, orc, golden):
    """The resident frame loop in the FLOAT build: float tree and decisions,
    update in float arithmetic (src/particle.cpp:66-74 with datatype float).
    Three frames against the FLOAT reference's own frame loop (golden), and the
    stored state stays float-valued."""
    g = golden("forces_float.npz")
    for prec in (nb.PRECISION_FP64, nb.PRECISION_MIXED):
        with nb.Engine(datatype_bytes=4, precision=prec) as e:
            e.set_particles(g["frames_pos"], g["frames_vel"], g["frames_mass"])
            for f in range(3):
                e.step(1)
                p, v = e.get_particles()
                assert np.array_equal(p, p.astype(np.float32).astype(np.float64))
                assert np.array_equal(v, v.astype(np.float32).astype(np.float64))
                err = np.abs(p - g["frames"][f]).max() / np.abs(g["frames"][f]).max()
                assert err <= 1e-6, (prec, f, err)


def test_float_build_ensemble_equals_single_systems(nb):
    """Independent systems get the FLOAT build's root cube and tree each."""
    counts = [700, 33, 2500]
    parts = [nb.generate(c, gen_type=s % 3, size=512.0, seed=11 + s) for s, c in enumerate(counts)]
    pos = np.concatenate([p[0] for p in parts]); vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    with nb.Engine(datatype_bytes=4, precision=nb.PRECISION_FP64) as e:
        e.set_systems(counts)
        e.set_particles(pos, vel, mass)
        e.step(2)
        pe, ve = e.get_particles()
    off = 0
    for p, v, m in parts:
        with nb.Engine(datatype_bytes=4, precision=nb.PRECISION_FP64) as e1:
            e1.set_particles(p, v, m)
            e1.step(2)
            p1, v1 = e1.get_particles()
        assert np.array_equal(pe[off:off + len(m)], p1)
        assert np.array_equal(ve[off:off + len(m)], v1)
        off += len(m)


def test_float_build_rejections(nb):
    for kw in (dict(datatype_bytes=5), dict(datatype_bytes=4, collide=1), dict(datatype_bytes=4, min_node_size=1.0)):
        with pytest.raises(nb.NBodyError) as ex:
            nb.Engine(**kw)
        assert ex.value.status == nb.ERR_INVALID
    pos, vel, mass = nb.generate(100)
    with nb.Engine(datatype_bytes=4) as e:
        with pytest.raises(nb.NBodyError) as ex:
            e.force_vjp(pos, mass, np.ones_like(pos))
        assert ex.value.status == nb.ERR_INVALID
        e.set_particles(pos, vel, mass)
        with pytest.raises(nb.NBodyError) as ex:
            e.forward_checkpointed(4)
        assert ex.value.status == nb.ERR_INVALID
        e.step(1)  # the context stays usable
