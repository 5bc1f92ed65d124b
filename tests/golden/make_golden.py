"""Generates the golden fixtures in this folder from the reference's own code.

Runs only where the reference tree is present and ``make -C oracle ref`` has
built ``oracle/_ref/libnbref.so`` and ``libnbref_f32.so`` (fosted3/nbodysim's
src/main.cpp, octree.cpp, particle.cpp, vector.cpp compiled unmodified, DOUBLE
and FLOAT builds). The outputs are small ``.npz`` files that pin the oracle
(``oracle/bh_oracle.c``) where the reference is absent. Usage:
``python tests/golden/make_golden.py`` (all), or with ``merging`` or ``float``
for one fixture only.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402


def lattice(k: int, step: float = 1.0):
    """k^3 lattice centred on the origin; odd k puts particles on every split plane."""
    r = (np.arange(k) - (k - 1) / 2.0) * step
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    return np.ascontiguousarray(g), np.full(len(g), 1e10)


def split_plane_set(seed: int = 0, n: int = 2000):
    """Float positions in an asymmetric box, so that the sum of the extrema on
    some axis needs more bits than a float holds: the FLOAT build's root centre
    (float(lo + hi) / 2) then lies an ulp above the DOUBLE build's, and 24
    particles placed exactly on it fall into the upper root octant in the DOUBLE
    build and the lower one in the FLOAT build. Over a thousand particles then
    accept different nodes in the two builds."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.2, 99.0, (n, 3)).astype(np.float32)
    pos[0] = np.float32([0.1, 0.15, 0.13])
    pos[1] = np.float32([100.0, 99.7, 99.9])
    lo, hi = pos.min(0), pos.max(0)
    cd = (lo.astype(np.float64) + hi.astype(np.float64)) / 2.0
    cf = ((lo + hi).astype(np.float64) / 2.0).astype(np.float32)
    extra = []
    for k in range(3):
        if float(cf[k]) > cd[k]:
            for _ in range(24):
                p = rng.uniform(5.0, 95.0, 3).astype(np.float32)
                p[k] = cf[k]
                extra.append(p)
    if extra:
        pos = np.concatenate([pos, np.array(extra, np.float32)])
    mass = rng.uniform(5e10, 5e11, len(pos)).astype(np.float32)
    return np.ascontiguousarray(pos, np.float64), mass.astype(np.float64)


def float_build() -> None:
    """The FLOAT build (-DFLOAT, the reference makefile's build): forces on the
    split-plane set and on the default cube, tree records, three frames."""
    R = O.Reference(O.REF_LIB_F32)
    assert R.datatype_bytes == 4
    pos, mass = split_plane_set(0)
    out = dict(split_pos=pos, split_mass=mass)
    for th in (0.3, 0.5, 0.7):
        out[f"split_acc_{th}"] = R.forces(pos, mass, th)[0]
    out["split_acc_damped_0.5"] = R.forces(pos, mass, 0.5, damping=True)[0]
    t = R.tree_nodes(pos, mass)
    out.update({"split_node_" + k: np.asarray(v) for k, v in t.items()})
    cpos, cvel, cmass = R.generate(O.GenParams(), 512)
    out.update(cube_pos=cpos, cube_mass=cmass, cube_acc_0_5=R.forces(cpos, cmass, 0.5)[0])
    fpos, fvel, fmass = R.generate(O.GenParams(min_vel=0.5, max_vel=2.0), 256)
    _, _, frames = R.run_frames(fpos, fvel, fmass, 3, keep_frames=True)
    out.update(frames_pos=fpos, frames_vel=fvel, frames_mass=fmass, frames=frames)
    np.savez_compressed(os.path.join(HERE, "forces_float.npz"), **out)


MERGE_CASES = (  # name, collide, collision_range, min_size
    ("collide_0.6", True, 0.6, 0.0),
    ("collide_1.0", True, 1.0, 0.0),
    ("minsize_1.0", False, 0.01, 1.0),
    ("minsize_2.0", False, 0.01, 2.0),
    ("both", True, 0.6, 2.0),
)


def merging(R) -> None:
    """One frame with collisions / apply_minimum_size, cube N = 400 in a 20-wide box."""
    pos, vel, mass = R.generate(O.GenParams(size=20.0), 400)
    out = dict(pos=pos, vel=vel, mass=mass)
    for name, collide, rng, ms in MERGE_CASES:
        p, v, a, m = R.frame_merging(pos, vel, mass, collide=collide, collision_range=rng, min_size=ms)
        order = np.argsort(m, kind="stable")  # the set's iteration order is arbitrary
        out[f"{name}_pos"], out[f"{name}_vel"], out[f"{name}_mass"] = p[order], v[order], m[order]
    np.savez_compressed(os.path.join(HERE, "merge_cube400.npz"), **out)


def main() -> None:
    R = O.Reference()
    assert R.datatype_bytes == 8
    if sys.argv[1:] == ["merging"]:
        merging(R)
        return
    if sys.argv[1:] == ["float"]:
        float_build()
        return
    merging(R)
    float_build()
    out = {}
    # seeded initial conditions: 64 particles per gen type x mass distribution
    for gt in (O.CUBE, O.SPHERE, O.SHELL):
        for md in (O.LINEAR, O.EXP, O.NORMAL):
            g = O.GenParams(gen_type=gt, mass_dist=md, min_vel=1.0, max_vel=5.0)
            p, v, m = R.generate(g, 64)
            out[f"gen_{gt}_{md}_pos"] = p
            out[f"gen_{gt}_{md}_vel"] = v
            out[f"gen_{gt}_{md}_mass"] = m
    np.savez_compressed(os.path.join(HERE, "generate.npz"), **out)

    # forces on the default cube (config 1's generator), N = 512
    pos, vel, mass = R.generate(O.GenParams(), 512)
    out = dict(pos=pos, mass=mass)
    for th in (0.3, 0.5, 0.7):
        out[f"acc_{th}"] = R.forces(pos, mass, th)[0]
    out["acc_damped_0.5"] = R.forces(pos, mass, 0.5, damping=True)[0]
    np.savez_compressed(os.path.join(HERE, "forces_cube512.npz"), **out)

    # sphere and shell, N = 512
    for name, gt in (("sphere", O.SPHERE), ("shell", O.SHELL)):
        pos, vel, mass = R.generate(O.GenParams(gen_type=gt, size=1024), 512)
        np.savez_compressed(os.path.join(HERE, f"forces_{name}512.npz"), pos=pos, mass=mass,
                            acc_0_5=R.forces(pos, mass, 0.5)[0])

    # lattices: 3^3 (particles on the split planes: strict '>' decides), 4^3
    for k in (3, 4):
        pos, mass = lattice(k)
        np.savez_compressed(os.path.join(HERE, f"forces_lattice{k}.npz"), pos=pos, mass=mass,
                            acc_0_5=R.forces(pos, mass, 0.5)[0], acc_0_3=R.forces(pos, mass, 0.3)[0])

    # five frames of the reference frame loop, cube N = 256
    pos, vel, mass = R.generate(O.GenParams(), 256)
    _, _, frames = R.run_frames(pos, vel, mass, 5, keep_frames=True)
    np.savez_compressed(os.path.join(HERE, "frames_cube256.npz"), pos=pos, vel=vel, mass=mass, frames=frames)

    # tree records (branching nodes), cube N = 512
    pos, vel, mass = R.generate(O.GenParams(), 512)
    t = R.tree_nodes(pos, mass)
    np.savez_compressed(os.path.join(HERE, "tree_cube512.npz"), pos=pos, mass=mass,
                        **{"node_" + k: np.asarray(v) for k, v in t.items()})
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
