"""GPU: independent systems in one engine (nbody_set_systems), CUDA-graph replay.

Each system of an ensemble must get exactly what it gets when run alone: the same
root cube, octree, 32-particle groups and arithmetic, so results are bitwise equal."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_systems(nb, counts, seed=0):
    parts = []
    for s, n in enumerate(counts):
        parts.append(nb.generate(int(n), gen_type=s % 3, size=1024.0 if s % 3 else 512.0, seed=seed + 7919 * s))
    pos = np.concatenate([p[0] for p in parts])
    vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    return parts, pos, vel, mass


@pytest.mark.parametrize("precision", [0, 1])
def test_ensemble_forces_equal_per_system(nb, precision):
    counts = [1, 2, 33, 1000, 4096, 31, 2500]
    parts, pos, vel, mass = make_systems(nb, counts)
    with nb.Engine(precision=precision) as e:
        e.set_systems(counts)
        e.set_particles(pos, vel, mass)
        e.compute_forces()
        _, _, acc = e.get_particles(acc=True)
        total = e.stats()["interactions"]
        off = 0
        inter = 0
        for (p, v, m) in parts:
            a, cnt = e.barnes_hut(p, m, counts=True)
            assert np.array_equal(acc[off:off + len(m)], a), off
            inter += int(cnt.sum())
            off += len(m)
    assert total == inter


def test_ensemble_steps_equal_per_system(nb):
    counts = [700, 1500, 64, 3000]
    parts, pos, vel, mass = make_systems(nb, counts, seed=3)
    with nb.Engine(precision=nb.PRECISION_FP64) as e:
        e.set_systems(counts)
        e.set_particles(pos, vel, mass)
        e.step(3)
        pe, ve = e.get_particles()
    off = 0
    for (p, v, m) in parts:
        with nb.Engine(precision=nb.PRECISION_FP64) as e1:
            e1.set_particles(p, v, m)
            e1.step(3)
            p1, v1 = e1.get_particles()
        assert np.array_equal(pe[off:off + len(m)], p1)
        assert np.array_equal(ve[off:off + len(m)], v1)
        off += len(m)


def test_graph_replay_equals_direct_launches(nb):
    pos, vel, mass = nb.generate(20000, gen_type=1)
    out = []
    for graphs in (True, False):
        with nb.Engine() as e:
            e.set_graphs(graphs)
            e.set_particles(pos, vel, mass)
            e.step(5)
            out.append(e.get_particles())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_graph_replay_through_adjoint(nb):
    pos, vel, mass = nb.generate(3000, gen_type=1, seed=2)
    target = pos + 1.0
    res = []
    for graphs in (True, False):
        with nb.Engine(precision=nb.PRECISION_FP64) as e:
            e.set_graphs(graphs)
            e.set_particles(pos, vel, mass)
            e.forward_checkpointed(10, 4)
            xK, _ = e.get_particles()
            res.append(e.backward(2.0 * (xK - target) / len(mass)))
    for a, b in zip(*res):
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max()


def test_set_systems_validation(nb):
    with nb.Engine() as e:
        with pytest.raises(nb.NBodyError):
            e.set_systems([10, 0, 5])
        e.set_systems([10, 5])
        pos, vel, mass = nb.generate(16)
        with pytest.raises(nb.NBodyError):
            e.set_particles(pos, vel, mass)  # 16 != 15
        e.set_systems([16])
        e.set_particles(pos, vel, mass)
        e.step(1)


def test_autotune_picks_a_valid_shape_and_keeps_results(nb):
    pos, vel, mass = nb.generate(30000, gen_type=2, size=1024.0)
    with nb.Engine() as e:
        e.set_particles(pos, vel, mass)
        e.compute_forces()
        _, _, a0 = e.get_particles(acc=True)
        shape = e.autotune()
        assert shape["warps_per_block"] in (1, 2, 4) and shape["blocks"] > 0
        e.compute_forces()
        _, _, a1 = e.get_particles(acc=True)
    # the block shape changes which warp runs which group, never a group's arithmetic
    assert np.array_equal(a0, a1)
    with nb.Engine(autotune=1) as e:
        e.set_particles(pos, vel, mass)
        e.step(2)
        assert e.stats()["walk_warps_per_block"] in (1, 2, 4)


def test_ensemble_at_full_scale(nb, orc):
    """512 systems, N per system log-uniform in [1024, 65536] (~9M particles), gen
    type cycling cube/sphere/shell: one force pass over the ensemble. Six systems
    (the smallest, the largest and four seeded picks) must equal their own runs bit
    for bit, and two of them the oracle's accepted-node counts."""
    rng = np.random.default_rng(0xDEADBEEF)
    counts = np.exp(rng.uniform(np.log(1024), np.log(65536), 512)).astype(np.uint32)
    parts = [nb.generate(int(c), gen_type=s % 3, size=512.0 if s % 3 == 0 else 1024.0, seed=0xDEADBEEF + s)
             for s, c in enumerate(counts)]
    pos = np.concatenate([p[0] for p in parts]); vel = np.concatenate([p[1] for p in parts])
    mass = np.concatenate([p[2] for p in parts])
    offs = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    picks = sorted({int(np.argmin(counts)), int(np.argmax(counts)), *map(int, rng.choice(512, 4, replace=False))})
    with nb.Engine() as e:
        e.set_systems(counts)
        e.set_particles(pos, vel, mass)
        e.compute_forces()
        _, _, acc = e.get_particles(acc=True)
        for k, s in enumerate(picks):
            p, _, m = parts[s]
            a, cnt = e.barnes_hut(p, m, counts=True)
            assert np.array_equal(acc[offs[s]:offs[s + 1]], a), s
            if k < 2:
                _, rc = orc.forces(p, m, 0.5)
                assert np.array_equal(cnt, rc), s


def test_ensemble_through_step_host(nb):
    """nbody_step_host on an ensemble large enough for the overlapped uploads
    (masses and velocities on a second stream; the per-system root cubes wait
    for the masses): the same as the resident steps, bit for bit."""
    counts = [30000, 25000, 20000]
    parts, pos, vel, mass = make_systems(nb, counts, seed=11)
    with nb.Engine() as e:
        e.set_systems(counts)
        e.set_particles(pos, vel, mass)
        e.step(2)
        p1, v1 = e.get_particles()
    with nb.Engine() as e:
        e.set_systems(counts)
        p2, v2 = pos.copy(), vel.copy()
        e.step_host(p2, v2, mass, 1)
        e.step_host(p2, v2, mass, 1)
    assert np.array_equal(p1, p2) and np.array_equal(v1, v2)
