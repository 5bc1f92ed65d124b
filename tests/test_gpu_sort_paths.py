"""GPU: the two ways the octree build sorts its keys give the same octree.

A build sorts by the first key word (octree levels 1-21) alone when the last
build found no two particles sharing it, and falls back on the device to the
full two-word sort when the new state has such ties. Whatever the prediction,
accepted-node counts must equal the oracle's and the forces must not change."""
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


@pytest.mark.parametrize("precision", [0, 1])
def test_first_word_sort_and_fallback_agree(nb, orc, precision):
    spread, _, ms = nb.generate(20000, gen_type=2, size=1024.0, seed=5)  # no shared first words
    tied, mt = clustered_with_outliers(nb)
    _, rc_tied = orc.forces(tied, mt, 0.5)
    _, rc_spread = orc.forces(spread, ms, 0.5)
    with nb.Engine(precision=precision) as fresh:
        a_tied_full, c_tied_full = fresh.barnes_hut(tied, mt, counts=True)  # a fresh context sorts both words
    assert np.array_equal(c_tied_full, rc_tied)
    with nb.Engine(precision=precision) as e:
        for _ in range(2):  # the second call sorts by the first word only
            a_s, c_s = e.barnes_hut(spread, ms, counts=True)
            assert np.array_equal(c_s, rc_spread)
        # predicted "no ties", but this state has them: the device falls back to the full sort
        a_t, c_t = e.barnes_hut(tied, mt, counts=True)
        assert np.array_equal(c_t, rc_tied)
        assert np.array_equal(a_t, a_tied_full)
        # and now the full sort is predicted; back to the spread state (no ties) once more
        a_t2, _ = e.barnes_hut(tied, mt, counts=True)
        assert np.array_equal(a_t2, a_tied_full)
        a_s2, c_s2 = e.barnes_hut(spread, ms, counts=True)
        assert np.array_equal(c_s2, rc_spread) and np.array_equal(a_s2, a_s)


def test_graph_replay_across_the_switch(nb):
    """Steps replayed from captured graphs keep their results when the state
    moves between the two sort paths (each path is its own captured graph)."""
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
            out.append(e.get_particles())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
