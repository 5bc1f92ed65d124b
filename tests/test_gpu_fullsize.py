"""Parity at the headline size: the shell of N = 1,048,576 particles (r 100,
rotation 0.1, size 1024), on its seeded initial state and after 20 adaptive
steps, when escaped particles have stretched the root cube by orders of
magnitude and the second key word decides most of the tree.

- The oracle walks a seeded sample of 2048 particles through the full tree: the
  accepted-node counts of the sample are EQUAL, accelerations within p99 1e-5
  (MIXED) and 1e-12 max (FP64 form).
- Over all N particles: the MIXED and FP64 forms accept the same nodes for every
  particle (both make the reference's decisions), the counts add up to the
  interaction statistic, and MIXED stays within p99 1e-5 of the FP64 form.
- With damping on the sample; the reference's FLOAT build on the sample; and
  the sphere of 100,000 particles, every particle against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 1 << 20
P99_MIXED = 1e-5
MAX_FP64 = 1e-12


def rel(a, b):
    den = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(den > 0, den, 1.0)


@pytest.fixture(scope="module")
def states(nb):
    pos, vel, mass = nb.generate(N, gen_type=nb.SHELL, size=1024.0, r_sphere=100.0, rotation_magnitude=0.1)
    with nb.Engine(adaptive=1, min_adaptive_dt=0.00333, max_pos_change=3.0, max_vel_change=3.0) as e:
        e.set_particles(pos, vel, mass)
        e.step(20)
        pos20, _ = e.get_particles()
    return {"initial": (pos, mass), "evolved": (pos20, mass)}


@pytest.fixture(scope="module")
def sample():
    return np.sort(np.random.default_rng(0xDEADBEEF).choice(N, 2048, replace=False)).astype(np.uint32)


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


@pytest.mark.parametrize("state,theta", [("initial", 0.3), ("initial", 0.5), ("initial", 0.7), ("evolved", 0.5)])
def test_sample_against_oracle(states, sample, eng, eng64, orc, state, theta):
    pos, mass = states[state]
    acc, cnt = eng.barnes_hut(pos, mass, theta=theta, counts=True)
    ra, rc = orc.forces(pos, mass, theta, sample=sample)
    assert np.array_equal(cnt[sample], rc), f"{np.count_nonzero(cnt[sample] != rc)} sampled particles differ"
    e = rel(acc[sample], ra)
    assert np.percentile(e, 99) <= P99_MIXED, (np.percentile(e, 99), e.max())
    if theta == 0.5:
        a64, c64 = eng64.barnes_hut(pos, mass, theta=theta, counts=True)
        assert np.array_equal(c64[sample], rc)
        assert rel(a64[sample], ra).max() <= MAX_FP64


@pytest.mark.parametrize("state", ["initial", "evolved"])
def test_forms_agree_on_every_particle(states, eng, eng64, state):
    pos, mass = states[state]
    acc, cnt = eng.barnes_hut(pos, mass, theta=0.5, counts=True)
    inter = eng.stats()["interactions"]
    a64, c64 = eng64.barnes_hut(pos, mass, theta=0.5, counts=True)
    assert np.array_equal(cnt, c64), f"{np.count_nonzero(cnt != c64)} particles differ in accepted-node count"
    assert inter == int(cnt.sum(dtype=np.uint64)) == eng64.stats()["interactions"]
    assert np.isfinite(acc).all()
    assert np.percentile(rel(acc, a64), 99) <= P99_MIXED


def test_damped_sample_against_oracle(states, sample, eng, orc):
    pos, mass = states["initial"]
    acc, cnt = eng.barnes_hut(pos, mass, damping=True, theta=0.5, counts=True)
    ra, rc = orc.forces(pos, mass, 0.5, damping=True, sample=sample)
    assert np.array_equal(cnt[sample], rc)
    assert np.percentile(rel(acc[sample], ra), 99) <= P99_MIXED


@pytest.mark.parametrize("state", ["initial", "evolved"])
def test_float_build_sample_against_oracle(nb, states, sample, orc, state):
    """The reference's FLOAT build (datatype_bytes = 4) at the headline size: the
    oracle's FLOAT path walks the seeded sample through its float tree; the
    accepted-node counts are equal and the MIXED forces within p99 1e-5."""
    pos, mass = states[state]
    with nb.Engine(datatype_bytes=4) as e:
        acc, cnt = e.barnes_hut(pos, mass, theta=0.5, counts=True)
    ra, rc = orc.forces(pos, mass, 0.5, sample=sample, single=True)
    assert np.array_equal(cnt[sample], rc), f"{np.count_nonzero(cnt[sample] != rc)} sampled particles differ"
    assert np.percentile(rel(acc[sample], ra), 99) <= P99_MIXED


def test_sphere_100k_every_particle(nb, eng, orc):
    """The sphere of 100,000 particles (r 100, rotation 0.1): every particle against the oracle."""
    pos, _, mass = nb.generate(100_000, gen_type=nb.SPHERE, size=1024.0, r_sphere=100.0, rotation_magnitude=0.1)
    acc, cnt = eng.barnes_hut(pos, mass, theta=0.5, counts=True)
    ra, rc = orc.forces(pos, mass, 0.5)
    assert np.array_equal(cnt, rc), f"{np.count_nonzero(cnt != rc)} particles differ"
    assert np.percentile(rel(acc, ra), 99) <= P99_MIXED


@pytest.mark.parametrize("state", ["initial", "evolved"])
def test_planned_sort_with_runs_equals_full_sort(nb, states, state):
    """The planned sort at the headline size: a fresh context sorts both key words
    in full; the next pass sorts the plan's passes (4 on the initial shell, where
    the deepest split needs 6), fewer than the deepest split needs, and thousands
    of runs of tied neighbours in place. Forces and counts are bit-identical."""
    pos, mass = states[state]
    with nb.Engine() as e:
        acc_full, cnt_full = e.barnes_hut(pos, mass, counts=True)
        st = e.stats()
        assert st["sort_passes"] == 16
        plan = st["sort_next_passes"]
        acc, cnt = e.barnes_hut(pos, mass, counts=True)
        st = e.stats()
    deepest = (st["sort_split_bits"] + 7) // 8 if st["sort_split_bits"] <= 63 else \
        8 + (st["sort_split_bits"] - 63 + 7) // 8
    assert st["sort_passes"] == plan < deepest
    assert st["sort_tie_runs"] > 1000
    assert np.array_equal(cnt, cnt_full) and np.array_equal(acc, acc_full)
