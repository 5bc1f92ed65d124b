"""The oracle (oracle/bh_oracle.c) pinned bit for bit to the reference's own code:
against the committed golden fixtures (made by tests/golden/make_golden.py from
the reference) and, where oracle/_ref was built, against the reference live."""
import numpy as np
import pytest


def test_generator_matches_golden(orc, oracle_mod, golden):
    g = golden("generate.npz")
    for gt in (0, 1, 2):
        for md in (0, 1, 2):
            p, v, m = orc.generate(oracle_mod.GenParams(gen_type=gt, mass_dist=md, min_vel=1.0, max_vel=5.0), 64)
            assert np.array_equal(p, g[f"gen_{gt}_{md}_pos"])
            assert np.array_equal(v, g[f"gen_{gt}_{md}_vel"])
            assert np.array_equal(m, g[f"gen_{gt}_{md}_mass"])


@pytest.mark.parametrize("theta", [0.3, 0.5, 0.7])
def test_forces_cube_golden(orc, golden, theta):
    g = golden("forces_cube512.npz")
    acc, _ = orc.forces(g["pos"], g["mass"], theta)
    assert np.array_equal(acc, g[f"acc_{theta}"])


def test_forces_damped_golden(orc, golden):
    g = golden("forces_cube512.npz")
    acc, _ = orc.forces(g["pos"], g["mass"], 0.5, damping=True)
    assert np.array_equal(acc, g["acc_damped_0.5"])


@pytest.mark.parametrize("name", ["sphere512", "shell512"])
def test_forces_sphere_shell_golden(orc, golden, name):
    g = golden(f"forces_{name}.npz")
    acc, _ = orc.forces(g["pos"], g["mass"], 0.5)
    assert np.array_equal(acc, g["acc_0_5"])


@pytest.mark.parametrize("k", [3, 4])
def test_forces_lattice_golden(orc, golden, k):
    """Lattice with particles exactly on split planes: the strict '>' octant rule."""
    g = golden(f"forces_lattice{k}.npz")
    for th, key in ((0.5, "acc_0_5"), (0.3, "acc_0_3")):
        acc, _ = orc.forces(g["pos"], g["mass"], th)
        assert np.array_equal(acc, g[key])


def test_frames_golden(orc, golden):
    g = golden("frames_cube256.npz")
    _, _, frames = orc.run_frames(g["pos"], g["vel"], g["mass"], 5, keep_frames=True)
    assert np.array_equal(frames, g["frames"])


def test_tree_records_golden(orc, golden):
    g = golden("tree_cube512.npz")
    t = orc.tree_nodes(g["pos"], g["mass"])
    for k in ("level", "count", "min_index", "mass", "com", "side"):
        assert np.array_equal(t[k], g["node_" + k]), k
    assert t["depth"] == int(g["node_depth"])


def test_root_cube_tie_rule(orc):
    # equal x and y extents larger than z: the reference falls through to z (src/main.cpp:909-920)
    pos = np.array([[0, 0, 0], [4, 4, 1]], float)
    c, s = orc.root_cube(pos)
    assert np.allclose(c, [2, 2, 0.5]) and s == 3.0


def test_direct_sum_two_body(orc):
    pos = np.array([[0.0, 0, 0], [2.0, 0, 0]])
    mass = np.array([1e10, 3e10])
    a = orc.direct(pos, mass)
    G = 6.67384e-11
    assert np.allclose(a[0], [G * 3e10 / 4, 0, 0], rtol=1e-15)
    assert np.allclose(a[1], [-G * 1e10 / 4, 0, 0], rtol=1e-15)


@pytest.mark.parametrize("gt,n,theta,damp", [(0, 3000, 0.5, False), (1, 3000, 0.3, False),
                                             (2, 3000, 0.7, True), (0, 2000, 0.5, True)])
def test_oracle_equals_reference_live(orc, ref, oracle_mod, gt, n, theta, damp):
    g = oracle_mod.GenParams(gen_type=gt, size=1024 if gt else 512)
    p, v, m = ref.generate(g, n)
    q = orc.generate(g, n)
    assert all(np.array_equal(a, b) for a, b in zip((p, v, m), q))
    a_ref, _ = ref.forces(p, m, theta, damping=damp)
    a_or, _ = orc.forces(p, m, theta, damping=damp)
    assert np.array_equal(a_ref, a_or)


@pytest.mark.parametrize("gt", [0, 1, 2])
def test_threaded_reference_equals_serial_build(ref, oracle_mod, gt):
    """With threads > 1 the reference builds its tree with gen_root_threaded
    (src/main.cpp:837-886): all 8 root children pre-allocated, each filled by
    its own thread through the closed inside() test (src/octree.cpp:320-336).
    On the seeded cube, sphere and shell that build gives the serial build's
    accelerations bit for bit, so the multi-threaded reference timings walk
    the same tree this library follows."""
    g = oracle_mod.GenParams(gen_type=gt, size=1024.0, r_sphere=100.0, rotation_magnitude=0.1)
    p, _, m = ref.generate(g, 20000)
    for theta in (0.5, 2.0):
        a1, _ = ref.forces(p, m, theta, threads=1)
        a8, _ = ref.forces(p, m, theta, threads=8)
        assert np.array_equal(a1, a8)


def test_threaded_reference_inserts_split_plane_particles_twice(ref):
    """The one place the two builds part: a particle exactly on a root split
    plane passes inside() for both neighbouring root children, so the threaded
    build holds it twice and every other particle feels it twice."""
    p = np.array([[-10.0, -3.0, 2.0], [0.0, 1.0, -1.0], [10.0, 4.0, -5.0], [5.0, -6.0, 7.0]])
    m = np.array([1e10, 2e10, 3e10, 4e10])  # root centre x = 0: particle 1 lies on the x split plane
    a1, _ = ref.forces(p, m, 0.5, threads=1)
    a8, _ = ref.forces(p, m, 0.5, threads=8)
    # it skips both of its own leaves (the sum order differs, so to rounding)
    assert np.allclose(a1[1], a8[1], rtol=1e-14, atol=0)
    G = 6.67384e-11
    for i in (0, 2, 3):  # the others take it twice
        d = p[1] - p[i]
        extra = G * m[1] * d / np.linalg.norm(d) ** 3
        assert np.allclose(a8[i] - a1[i], extra, rtol=1e-9, atol=0)


def test_oracle_frames_equal_reference_live(orc, ref, oracle_mod):
    p, v, m = ref.generate(oracle_mod.GenParams(gen_type=1), 800)
    _, _, f1 = ref.run_frames(p, v, m, 4, keep_frames=True)
    _, _, f2 = orc.run_frames(p, v, m, 4, keep_frames=True)
    assert np.array_equal(f1, f2)


def test_reference_image_hand_cases(ref):
    """write_image (src/main.cpp:556-678) on single particles, worked by hand."""
    import numpy as np
    # front: x = px + w/2 = 5, y = pz + h/2 = 1
    im = ref.write_image(np.array([[1.0, 0.0, -2.0]]), 8, 6, 0, 0, False, False, 1.0, 255.0)
    assert im[1, 5].tolist() == [255, 255, 255] and im.sum() == 3 * 255
    # iso at the origin: x = w/2 = 4, y = h/2 = 3, flipped to h-1-3 = 2; heat 300 -> (R, G, B) = (44, 211, 0)
    im = ref.write_image(np.array([[0.0, 0.0, 0.0]]), 8, 6, 3, 1, False, False, 1.0, 300.0)
    assert im[2, 4].tolist() == [44, 211, 0]
    assert (im[:, :, 2] == 255).sum() == 8 * 6 - 1  # every other pixel is heat 0: blue
    # y between h-1 and w-1 is clamped onto the top row (the bound uses the width)
    im = ref.write_image(np.array([[0.0, 0.0, 4.0]]), 12, 6, 0, 0, False, False, 1.0, 10.0)
    assert im[5, 6].tolist() == [10, 10, 10]


def test_reference_merging_hand_cases(ref):
    """The reference's merging steps on hand-worked layouts (one frame, dt 0.0333)."""
    import numpy as np
    dt = 0.0333
    # A=(0,0,0), B=(0.1,0,0), C=(10,0,0): root side 12, A and B share cells down to
    # level 6 (side 0.1875) and split at level 7 (side 0.09375)
    pos = np.array([[0.0, 0, 0], [0.1, 0, 0], [10.0, 0, 0]])
    vel = np.array([[1.0, 0, 0], [0.0, 2.0, 0], [0.0, 0, 0]])
    mass = np.array([3e9, 1e9, 5e9])
    _, _, _, m = ref.frame_merging(pos, vel, mass, min_size=0.1)
    assert len(m) == 3
    p, v, a, m = ref.frame_merging(pos, vel, mass, min_size=0.2)
    assert sorted(m.tolist()) == [4e9, 5e9]
    k = int(np.argmin(m))
    vm = (vel[0] * 3e9 + vel[1] * 1e9) / 4e9  # collide(): mass-weighted averages
    pm = (pos[0] * 3e9 + pos[1] * 1e9) / 4e9
    # the merged particle feels C's pull before the update; its velocity moves by a * dt
    assert np.allclose(v[k], vm + a[k] * dt, rtol=0, atol=1e-15)
    assert np.allclose(p[k], pm + v[k] * dt, rtol=0, atol=1e-15)
    # collisions: A and B within range 0.2 merge after the forces; the new particle has a = 0
    p, v, a, m = ref.frame_merging(pos, vel, mass, collide=True, collision_range=0.2)
    k = int(np.argmin(m))
    assert len(m) == 2 and m[k] == 4e9 and not a[k].any()
    assert np.array_equal(v[k], vm) and np.array_equal(p[k], pm + vm * dt)
    _, _, _, m = ref.frame_merging(pos, vel, mass, collide=True, collision_range=0.05)
    assert len(m) == 3


# ---- the reference's FLOAT build (-DFLOAT, the build its makefile ships) ----

def test_float_build_forces_golden(orc, golden):
    """Split-plane set (particles on the FLOAT build's root centre, which lies an
    ulp from the DOUBLE build's) and the default cube: the oracle's FLOAT path
    equals the FLOAT reference bit for bit, and its accepted nodes differ from
    the DOUBLE build's for over a thousand particles."""
    g = golden("forces_float.npz")
    pos, mass = g["split_pos"], g["split_mass"]
    for th in (0.3, 0.5, 0.7):
        acc, cnt = orc.forces(pos, mass, th, single=True)
        assert np.array_equal(acc, g[f"split_acc_{th}"]), th
    acc, cnt32 = orc.forces(pos, mass, 0.5, damping=True, single=True)
    assert np.array_equal(acc, g["split_acc_damped_0.5"])
    _, cnt64 = orc.forces(pos, mass, 0.5)
    _, cnt32 = orc.forces(pos, mass, 0.5, single=True)
    assert (cnt32 != cnt64).sum() > 500
    acc, _ = orc.forces(g["cube_pos"], g["cube_mass"], 0.5, single=True)
    assert np.array_equal(acc, g["cube_acc_0_5"])


def test_float_build_tree_and_frames_golden(orc, golden):
    g = golden("forces_float.npz")
    t = orc.tree_nodes(g["split_pos"], g["split_mass"], single=True)
    for k in ("level", "count", "min_index", "mass", "com", "side"):
        assert np.array_equal(t[k], g["split_node_" + k]), k
    _, _, frames = orc.run_frames(g["frames_pos"], g["frames_vel"], g["frames_mass"], 3, keep_frames=True,
                                  single=True)
    assert np.array_equal(frames, g["frames"])


def test_float_build_root_cube(orc, golden):
    """FLOAT root cube: float(lo + hi) / 2 and float(extent + 2) (src/main.cpp:898-920)."""
    g = golden("forces_float.npz")
    c, s = orc.root_cube(g["split_pos"], single=True)
    p32 = g["split_pos"].astype(np.float32)
    lo, hi = p32.min(0), p32.max(0)
    assert np.array_equal(c, ((lo + hi).astype(np.float64) / 2.0).astype(np.float32).astype(np.float64))
    ext = hi - lo
    assert s == float(np.float32(float(ext.max()) + 2.0))
    c64, _ = orc.root_cube(g["split_pos"])
    assert not np.array_equal(c, c64)


@pytest.mark.parametrize("gt,n,theta,damp", [(0, 3000, 0.5, False), (1, 4000, 0.3, True), (2, 4000, 0.7, False)])
def test_float_oracle_equals_float_reference_live(orc, oracle_mod, gt, n, theta, damp):
    import os
    if not os.path.exists(oracle_mod.REF_LIB_F32):
        pytest.skip("FLOAT reference harness not built (oracle/_ref)")
    R = oracle_mod.Reference(oracle_mod.REF_LIB_F32)
    p, v, m = R.generate(oracle_mod.GenParams(gen_type=gt, size=1024 if gt else 512), n)
    a_ref, _ = R.forces(p, m, theta, damping=damp)
    a_or, _ = orc.forces(p, m, theta, damping=damp, single=True)
    assert np.array_equal(a_ref, a_or)
    t_ref = R.tree_nodes(p, m)
    t_or = orc.tree_nodes(p, m, single=True)
    for k in ("level", "count", "min_index", "mass", "com", "side"):
        assert np.array_equal(t_ref[k], t_or[k]), k
