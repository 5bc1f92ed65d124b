"""GPU merging against the reference's own frame with collisions and/or
apply_minimum_size (src/main.cpp:386-396, 423-550, 1001-1060): golden
fixtures from tests/golden/make_golden.py, and the reference live where
oracle/_ref is built. Particle order differs (the reference keeps an
unordered_set), so both sides are ordered by mass before comparing."""
import numpy as np
import pytest

from golden.make_golden import MERGE_CASES

pytestmark = pytest.mark.gpu


def run_gpu(nb, pos, vel, mass, precision, collide, rng, ms, steps=1, **kw):
    with nb.Engine(precision=precision, collide=int(collide), collision_range=rng, min_node_size=ms, **kw) as e:
        e.set_particles(pos, vel, mass)
        e.step(steps)
        p, v = e.get_particles()
        m = e.get_masses()
        st = e.stats()
    o = np.argsort(m, kind="stable")
    return p[o], v[o], m[o], st


def compare(got, want, tol):
    p, v, m = got
    wp, wv, wm = want
    assert len(m) == len(wm)
    assert np.allclose(m, wm, rtol=1e-14, atol=0), np.abs(m - wm).max()
    for a, b in ((p, wp), (v, wv)):
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
        assert err <= tol, err


@pytest.mark.parametrize("case", MERGE_CASES, ids=[c[0] for c in MERGE_CASES])
def test_merging_matches_reference_fixture(nb, golden, case):
    name, collide, rng, ms = case
    g = golden("merge_cube400.npz")
    want = (g[f"{name}_pos"], g[f"{name}_vel"], g[f"{name}_mass"])
    p, v, m, st = run_gpu(nb, g["pos"], g["vel"], g["mass"], nb.PRECISION_FP64, collide, rng, ms)
    compare((p, v, m), want, 1e-12)
    assert st["merged_min_size"] + st["merged_collisions"] == 400 - len(m)
    # MIXED: the merge decisions are the same (they run in FP64); forces to FP32 accuracy
    p, v, m, _ = run_gpu(nb, g["pos"], g["vel"], g["mass"], nb.PRECISION_MIXED, collide, rng, ms)
    compare((p, v, m), want, 1e-5)


@pytest.mark.parametrize("gen_type,size,collide,rng,ms", [
    (0, 50.0, True, 0.3, 0.0), (0, 50.0, True, 1.0, 0.0), (1, 400.0, True, 2.0, 0.0),
    (0, 50.0, False, 0.01, 3.0), (2, 300.0, False, 0.01, 2.0), (0, 50.0, True, 0.5, 2.5),
])
def test_merging_matches_reference_live(nb, ref, gen_type, size, collide, rng, ms):
    pos, vel, mass = nb.generate(3000, gen_type=gen_type, size=size)
    wp, wv, _, wm = ref.frame_merging(pos, vel, mass, collide=collide, collision_range=rng, min_size=ms)
    o = np.argsort(wm, kind="stable")
    assert len(wm) < 3000  # the case merges something
    p, v, m, _ = run_gpu(nb, pos, vel, mass, nb.PRECISION_FP64, collide, rng, ms)
    compare((p, v, m), (wp[o], wv[o], wm[o]), 1e-12)


def test_min_size_everything_and_repeated_steps(nb, ref):
    pos, vel, mass = nb.generate(500, gen_type=0, size=10.0)
    # every cell is below min_size: the whole system folds into one particle (serial apply_minimum_size)
    wp, wv, _, wm = ref.frame_merging(pos, vel, mass, min_size=1e9)
    p, v, m, st = run_gpu(nb, pos, vel, mass, nb.PRECISION_FP64, False, 0.01, 1e9)
    assert len(m) == 1 == len(wm) and m[0] == wm[0]
    assert np.array_equal(p, wp) and np.array_equal(v, wv)
    # several steps with collisions: mass is conserved, the count never grows
    pos, vel, mass = nb.generate(4000, gen_type=0, size=40.0)
    with nb.Engine(collide=1, collision_range=0.8, adaptive=1) as e:
        e.set_particles(pos, vel, mass)
        n_prev = 4000
        for _ in range(4):
            e.step(1)
            assert e.n <= n_prev
            n_prev = e.n
            st = e.stats()
            assert st["merged_collisions"] == 0 or st["collision_pairs"] > 0
            assert np.isfinite(st["last_dt"]) and st["last_dt"] > 0
        m = e.get_masses()
        p, v = e.get_particles()
    assert n_prev < 4000
    assert abs(m.sum() - mass.sum()) <= 1e-12 * mass.sum()
    assert np.isfinite(p).all() and np.isfinite(v).all()


def test_merging_rejected_where_n_is_fixed(nb):
    pos, vel, mass = nb.generate(300)
    with nb.Engine(collide=1) as e:
        with pytest.raises(nb.NBodyError):
            e.step_host(pos.copy(), vel.copy(), mass, 1)
        e.set_particles(pos, vel, mass)
        with pytest.raises(nb.NBodyError):
            e.forward_checkpointed(4)
        e.set_systems([100, 200])
        with pytest.raises(nb.NBodyError):
            e.step(1)
    with nb.Engine(min_node_size=1.0) as e:
        e.set_particles(pos, vel, mass)
        e.compute_forces()  # forces only: nothing merges
        assert e.device_view().n == 300


@pytest.mark.parametrize("gen_type,size,collide,rng,ms", [(0, 200.0, True, 1.0, 0.0), (1, 400.0, True, 0.5, 1.0)])
def test_merging_matches_reference_at_60k(nb, ref, gen_type, size, collide, rng, ms):
    """60,000 particles: hundreds of merges in one frame (pairs, chains and, in
    the second case, minimum-size folds too), against the reference's frame."""
    pos, vel, mass = nb.generate(60000, gen_type=gen_type, size=size)
    wp, wv, _, wm = ref.frame_merging(pos, vel, mass, collide=collide, collision_range=rng, min_size=ms)
    o = np.argsort(wm, kind="stable")
    assert len(wm) < 60000 - 100
    p, v, m, _ = run_gpu(nb, pos, vel, mass, nb.PRECISION_FP64, collide, rng, ms)
    compare((p, v, m), (wp[o], wv[o], wm[o]), 1e-12)
