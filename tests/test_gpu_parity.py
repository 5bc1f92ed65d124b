"""GPU parity: the CUDA path through the C ABI against the oracle (the
reference's CPU path restated bit for bit, oracle/bh_oracle.c).

Bars: per-particle accepted-node counts are EQUAL (every opening decision is
the reference's); accelerations within p99 relative error 1e-5 for the MIXED
form (FP32 pair forces) and 1e-12 max for the FP64 form."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P99_MIXED = 1e-5
MAX_FP64 = 1e-12


@pytest.fixture(scope="module")
def eng(nb):
    e = nb.Engine()
    yield e
    e.close()


@pytest.fixture(scope="module")
def eng64(nb):
    e = nb.Engine(precision=nb.PRECISION_FP64)
    yield e
    e.close()


def rel(a, b):
    den = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(den > 0, den, 1.0)


CASES = [  # gen_type, n, theta, damping
    (0, 5000, 0.5, False), (0, 5000, 0.3, False), (0, 5000, 0.7, False), (0, 5000, 0.5, True),
    (1, 20000, 0.5, False), (2, 20000, 0.5, False), (2, 20000, 0.3, False), (1, 4099, 0.7, True),
]


@pytest.mark.parametrize("gt,n,theta,damp", CASES)
def test_mixed_forces_and_counts(nb, eng, orc, gt, n, theta, damp):
    pos, vel, mass = nb.generate(n, gen_type=gt, size=1024 if gt else 512)
    acc, cnt = eng.barnes_hut(pos, mass, damping=damp, theta=theta, counts=True)
    ra, rc = orc.forces(pos, mass, theta, damping=damp)
    assert np.array_equal(cnt, rc), f"{np.count_nonzero(cnt != rc)} particles differ in accepted-node count"
    e = rel(acc, ra)
    assert np.percentile(e, 99) <= P99_MIXED, (np.percentile(e, 99), e.max())
    assert eng.stats()["interactions"] == int(rc.sum())


@pytest.mark.parametrize("gt,n,theta,damp", CASES[:6])
def test_fp64_forces_and_counts(nb, eng64, orc, gt, n, theta, damp):
    pos, vel, mass = nb.generate(n, gen_type=gt, size=1024 if gt else 512)
    acc, cnt = eng64.barnes_hut(pos, mass, damping=damp, theta=theta, counts=True)
    ra, rc = orc.forces(pos, mass, theta, damping=damp)
    assert np.array_equal(cnt, rc)
    assert rel(acc, ra).max() <= MAX_FP64


@pytest.mark.parametrize("name", ["cube512", "sphere512", "shell512"])
def test_against_golden(nb, eng, golden, name):
    g = golden(f"forces_{name}.npz")
    key = "acc_0.5" if name == "cube512" else "acc_0_5"
    acc = eng.barnes_hut(g["pos"], g["mass"], theta=0.5)
    assert np.percentile(rel(acc, g[key]), 99) <= P99_MIXED


@pytest.mark.parametrize("k", [3, 4])
def test_lattice_split_plane_ties(nb, eng, eng64, orc, golden, k):
    """Particles exactly on split planes: the strict '>' octant rule and tie decisions.
    Symmetric lattices have particles whose net force is zero up to rounding, so
    errors are measured against the largest acceleration in the lattice."""
    g = golden(f"forces_lattice{k}.npz")
    for th, key in ((0.5, "acc_0_5"), (0.3, "acc_0_3")):
        ref = g[key]
        scale = np.linalg.norm(ref, axis=1).max()
        _, rc = orc.forces(g["pos"], g["mass"], th)
        a64, c64 = eng64.barnes_hut(g["pos"], g["mass"], theta=th, counts=True)
        assert np.array_equal(c64, rc)
        assert np.abs(a64 - ref).max() <= MAX_FP64 * scale
        a, c = eng.barnes_hut(g["pos"], g["mass"], theta=th, counts=True)
        assert np.array_equal(c, rc)
        assert np.abs(a - ref).max() <= 1e-6 * scale


def test_edge_sizes(nb, eng, orc):
    assert eng.barnes_hut(np.zeros((0, 3)), np.zeros(0)).shape == (0, 3)
    a = eng.barnes_hut(np.array([[1.0, 2.0, 3.0]]), np.array([5e10]))
    assert np.array_equal(a, np.zeros((1, 3)))
    for n in (2, 3, 31, 32, 33, 65, 1000):
        pos, _, mass = nb.generate(n, seed=n)
        acc, cnt = eng.barnes_hut(pos, mass, counts=True)
        ra, rc = orc.forces(pos, mass, 0.5)
        assert np.array_equal(cnt, rc)
        assert rel(acc, ra).max() <= 1e-5


def test_close_pairs_need_deep_keys(nb, eng, eng64, orc):
    """Pairs closer than 2^-21 of the root side exercise the 42/63-level keys."""
    pos, _, mass = nb.generate(3000, seed=7)
    pos[1] = pos[0] + np.array([3e-9, -2e-9, 1e-9])
    pos[2] = pos[0] + np.array([1e-12, 0.0, 0.0])
    pos[5] = pos[4] + np.array([0.0, 5e-8, 0.0])
    acc, cnt = eng64.barnes_hut(pos, mass, counts=True)
    ra, rc = orc.forces(pos, mass, 0.5)
    assert np.array_equal(cnt, rc)
    assert rel(acc, ra).max() <= 1e-9
    acc, cnt = eng.barnes_hut(pos, mass, counts=True)
    assert np.array_equal(cnt, rc)


def test_escaped_particles_need_two_key_words(nb, eng, eng64, orc):
    """Far escapees blow the root cube up by ~1e7: the bulk then shares its first
    21 octree levels, and separating it needs the second key word."""
    pos, _, mass = nb.generate(6000, seed=11)
    pos[0] = [3.0e9, -1.0e9, 2.0e9]
    pos[1] = [-2.5e9, 2.0e9, -3.0e9]
    ra, rc = orc.forces(pos, mass, 0.5)
    acc, cnt = eng64.barnes_hut(pos, mass, counts=True)
    assert np.array_equal(cnt, rc)
    assert rel(acc, ra).max() <= 1e-9
    acc, cnt = eng.barnes_hut(pos, mass, counts=True)
    assert np.array_equal(cnt, rc)
    assert np.percentile(rel(acc, ra), 99) <= P99_MIXED
    assert eng.stats()["tree_depth"] > 21


def test_coincident_particles_rejected(nb, eng):
    pos, _, mass = nb.generate(100)
    pos[7] = pos[3]
    with pytest.raises(nb.NBodyError) as e:
        eng.barnes_hut(pos, mass)
    assert e.value.status == nb.ERR_COINCIDENT
    pos, _, mass = nb.generate(100)   # the context stays usable
    eng.barnes_hut(pos, mass)


def test_nonfinite_rejected(nb, eng):
    pos, _, mass = nb.generate(100)
    pos[10, 1] = np.nan
    with pytest.raises(nb.NBodyError) as e:
        eng.barnes_hut(pos, mass)
    assert e.value.status == nb.ERR_NONFINITE
    mass[3] = np.inf
    pos[10, 1] = 0.0
    with pytest.raises(nb.NBodyError) as e:
        eng.barnes_hut(pos, mass)
    assert e.value.status == nb.ERR_NONFINITE


def test_direct_sum_error_reported(nb, eng, orc):
    """Every result also gets its error against the FP64 direct sum (reported, BH-truncation sized)."""
    pos, _, mass = nb.generate(20000, gen_type=1)
    acc = eng.barnes_hut(pos, mass, theta=0.5)
    idx = np.random.default_rng(0xDEADBEEF).choice(20000, 512, replace=False)
    d = orc.direct(pos, mass, targets=idx)
    e = rel(acc[idx], d)
    assert np.percentile(e, 99) < 5e-2
    ra, _ = orc.forces(pos, mass, 0.5)
    assert abs(np.percentile(rel(ra[idx], d), 99) - np.percentile(e, 99)) < 1e-5


@pytest.mark.parametrize("damp", [False, True])
def test_direct_sum_kernel_matches_oracle(nb, orc, damp):
    """nbody_direct_forces (FP64, compensated) against the oracle's compensated direct sum."""
    pos, vel, mass = nb.generate(6000, gen_type=1)
    targets = np.random.default_rng(2).choice(6000, 300, replace=False).astype(np.uint32)
    want = orc.direct(pos, mass, targets=targets, damping=damp)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        got = e.direct_forces(targets, damping=damp)
        first = e.direct_forces(None)[:5]
    scale = np.linalg.norm(want, axis=1)
    assert (np.linalg.norm(got - want, axis=1) / scale).max() <= 1e-13
    assert np.allclose(first, orc.direct(pos, mass, targets=np.arange(5, dtype=np.uint32)), rtol=1e-13, atol=0)
