"""GPU: every sort plan of the octree build gives the same octree.

A fresh context sorts both key words in full (16 passes of 8 bits). Later builds
sort only top key bits: the first word's (octree levels 1-21), or all of it and
the second word's (levels 22-42). The plan is the fewest passes that leave at
most max(64, n / 16) pairs of the last build's neighbours tied. Runs of
neighbours left equal over the planned bits are sorted in place by their full
keys (runs of at most 64); a longer run makes the full sort run on the device,
after which the plans cover the deepest split (the key bits that separate every
pair of neighbours) for 8 calls. Calls of several steps always cover the
deepest split. Whatever the plan, accepted-node counts must equal the oracle's
and the forces must not change."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def clustered_with_outliers(nb, n=5000):
    """A tight cluster and two far particles: the root cube is ~2e7 wide, so the
    first 21 levels (cells of ~10) do not separate the cluster's particles."""
    pos, vel, mass = nb.generate(n, gen_type=1, r_sphere=1.0, size=4.0, seed=21)
    pos[0] = [1e7, 3.0, -2.0]
    pos[1] = [-1e7, -5.0, 7.0]
    return pos, mass


def planned_passes(split_bits):
    """Passes of the plan that covers `split_bits`."""
    bits = split_bits
    if bits <= 63:
        return (bits + 7) // 8
    return 8 + (bits - 63 + 7) // 8 if bits <= 126 else 16


@pytest.mark.parametrize("precision", [0, 1])
def test_sort_plans_agree(nb, orc, precision):
    spread, _, ms = nb.generate(20000, gen_type=2, size=1024.0, seed=5)
    tied, mt = clustered_with_outliers(nb)
    _, rc_tied = orc.forces(tied, mt, 0.5)
    _, rc_spread = orc.forces(spread, ms, 0.5)
    with nb.Engine(precision=precision) as fresh:
        a_tied_full, c_tied_full = fresh.barnes_hut(tied, mt, counts=True)  # a fresh context sorts both words
        st = fresh.stats()
        assert st["sort_passes"] == 16 and st["sort_split_bits"] > 63
    assert np.array_equal(c_tied_full, rc_tied)
    with nb.Engine(precision=precision) as e:
        a_s, c_s = e.barnes_hut(spread, ms, counts=True)
        assert np.array_equal(c_s, rc_spread)
        st = e.stats()
        assert st["sort_passes"] == 16
        split = st["sort_split_bits"]
        assert 3 <= split <= 63 - 8
        # the second call sorts fewer top bits of the first word than the deepest
        # split needs, and sorts the runs they leave in place
        plan = st["sort_next_passes"]
        a_s1, c_s1 = e.barnes_hut(spread, ms, counts=True)
        st = e.stats()
        assert st["sort_passes"] == plan < planned_passes(split) < 8 and st["sort_tie_runs"] > 0
        assert st["sort_next_passes"] == plan
        assert np.array_equal(c_s1, rc_spread) and np.array_equal(a_s1, a_s)
        # planned for the spread state, but this one needs the second word and the
        # cluster is one run of thousands: the device runs the full sort after the planned one
        a_t, c_t = e.barnes_hut(tied, mt, counts=True)
        st = e.stats()
        assert st["sort_passes"] == plan + 16
        assert np.array_equal(c_t, rc_tied)
        assert np.array_equal(a_t, a_tied_full)
        # now, for a few calls, the deepest split: all of the first word and the top bits of the second
        split_t = st["sort_split_bits"]
        assert st["sort_next_passes"] == planned_passes(split_t)
        a_t2, c_t2 = e.barnes_hut(tied, mt, counts=True)
        assert 8 < e.stats()["sort_passes"] == planned_passes(split_t) < 16
        assert np.array_equal(c_t2, rc_tied) and np.array_equal(a_t2, a_tied_full)
        # back to the spread state: the larger plan covers it, then the plan shrinks
        a_s2, c_s2 = e.barnes_hut(spread, ms, counts=True)
        assert e.stats()["sort_passes"] == planned_passes(split_t)
        assert np.array_equal(c_s2, rc_spread) and np.array_equal(a_s2, a_s)
        a_s3, _ = e.barnes_hut(spread, ms, counts=True)
        assert e.stats()["sort_passes"] == planned_passes(split)
        assert np.array_equal(a_s3, a_s)
        # once those calls are over, the fewer passes again
        for _ in range(5):
            a_s4, c_s4 = e.barnes_hut(spread, ms, counts=True)
        assert e.stats()["sort_next_passes"] == plan
        a_s4, c_s4 = e.barnes_hut(spread, ms, counts=True)
        assert e.stats()["sort_passes"] == plan
        assert np.array_equal(a_s4, a_s) and np.array_equal(c_s4, rc_spread)


@pytest.mark.parametrize("single,offset", [(False, 1e-4), (False, 1e-7), (True, 1e-4)])
def test_short_plan_runs_sorted_in_place(nb, orc, single, offset):
    """A state whose deepest split lies below the plan's bits: the close pair is a
    run of equal neighbours, sorted in place by its full keys (by the first word
    at 1e-4, where the second word is not needed; by the second word, computed for
    the run, at 1e-7). FP64 and FLOAT builds."""
    pos, _, mass = nb.generate(20000, gen_type=2, size=1024.0, seed=7)
    deeper = pos.copy()
    deeper[1] = deeper[0] + np.array([1.0, -2.0, 1.0]) * offset  # a pair much closer than any other
    dt = 4 if single else 8
    _, rc = orc.forces(deeper, mass, 0.5, single=single)
    with nb.Engine(datatype_bytes=dt) as e:
        e.barnes_hut(pos, mass)
        e.barnes_hut(pos, mass)
        st = e.stats()
        split, plan = st["sort_split_bits"], st["sort_next_passes"]
        acc, cnt = e.barnes_hut(deeper, mass, counts=True)
        st = e.stats()
        assert st["sort_split_bits"] > split
        assert st["sort_passes"] == plan < 8  # no full sort
        assert st["sort_tie_runs"] >= 1
        assert np.array_equal(cnt, rc)
        acc2, cnt2 = e.barnes_hut(deeper, mass, counts=True)  # one more tied pair: still no full sort
        assert e.stats()["sort_passes"] == st["sort_next_passes"] < 8
    with nb.Engine(datatype_bytes=dt) as fresh:
        acc_full, cnt_full = fresh.barnes_hut(deeper, mass, counts=True)
    for a, c in ((acc, cnt), (acc2, cnt2)):
        assert np.array_equal(a, acc_full) and np.array_equal(c, cnt_full)


def test_graph_replay_across_plans(nb):
    """Steps replayed from captured graphs keep their results when the state
    moves between sort plans (each plan is its own captured graph)."""
    spread, vel, ms = nb.generate(20000, gen_type=2, size=1024.0, seed=5)
    out = []
    for graphs in (True, False):
        with nb.Engine(precision=nb.PRECISION_FP64) as e:
            e.set_graphs(graphs)
            e.set_particles(spread, vel, ms)
            e.step(3)
            tied, mt = clustered_with_outliers(nb)
            e.set_particles(tied, np.zeros_like(tied), mt)
            e.step(2)
            e.set_particles(spread, vel, ms)
            e.step(3)
            out.append(e.get_particles())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_short_plan_runs_in_the_second_word(nb, orc):
    """A plan that sorts all of the first word and the top bits of the second: a
    pair closer than its bits resolve is a run sorted in place by the gathered
    second words."""
    tied, mt = clustered_with_outliers(nb)
    deeper = tied.copy()
    deeper[3] = deeper[2] + np.array([1.0, 1.0, -1.0]) * 1e-5  # ~40 levels below a 2e7 root: within the second word
    _, rc = orc.forces(deeper, mt, 0.5)
    with nb.Engine() as e:
        e.barnes_hut(tied, mt)
        e.barnes_hut(tied, mt)
        st = e.stats()
        split, plan = st["sort_split_bits"], st["sort_next_passes"]
        assert 8 < plan <= planned_passes(split) < 16
        acc, cnt = e.barnes_hut(deeper, mt, counts=True)
        st = e.stats()
        assert split < st["sort_split_bits"] <= 126 and st["sort_tie_runs"] >= 1
        assert st["sort_passes"] == plan
        assert np.array_equal(cnt, rc)
    with nb.Engine() as fresh:
        acc_full, cnt_full = fresh.barnes_hut(deeper, mt, counts=True)
    assert np.array_equal(acc, acc_full) and np.array_equal(cnt, cnt_full)


def test_calls_of_several_steps_plan_the_deepest_split(nb, orc):
    """A call of several steps replays one captured step while the state drifts,
    so it sorts the passes that cover the last build's deepest split; a single
    step or force pass sorts the fewer passes of sort_next_passes."""
    pos, vel, mass = nb.generate(20000, gen_type=2, size=1024.0, seed=5)
    with nb.Engine(precision=nb.PRECISION_FP64) as e:
        e.barnes_hut(pos, mass)
        st = e.stats()
        split, plan = st["sort_split_bits"], st["sort_next_passes"]
        assert plan < planned_passes(split)
        e.set_particles(pos, vel, mass)
        e.step(2)
        st = e.stats()
        assert st["sort_passes"] == planned_passes(split)
        after_two, nxt = e.get_particles(), st["sort_next_passes"]
        e.step(1)
        assert e.stats()["sort_passes"] == nxt
    with nb.Engine(precision=nb.PRECISION_FP64) as ref:  # the same steps on the full sort's trees
        ref.set_graphs(False)
        ref.set_particles(pos, vel, mass)
        ref.step(1)
        ref.step(1)
        p2, v2 = ref.get_particles()
    assert np.array_equal(after_two[0], p2) and np.array_equal(after_two[1], v2)
