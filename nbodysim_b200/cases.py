"""Fixed workloads for profiling one kernel under ncu (device code is this package's).

    python -m nbodysim_b200.cases walk --gen shell --n 1048576 --evolve 30 --save /tmp/shell30.npz
    python -m nbodysim_b200.cases walk --load /tmp/shell30.npz --passes 2

The first form generates the seeded reference initial conditions, advances them
`--evolve` steps with adaptive dt (the bench's regime), optionally saves the
state, then runs `--passes` force passes (`nbody_barnes_hut`). The second
starts from a saved state. Each force pass launches the walk kernel once, so
`ncu -k regex:k_walk -s <passes-1> -c 1` captures the last pass of a loaded state.
`adjoint` runs the adjoint workload (sphere, fixed dt, checkpointed forward + backward).
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import CUBE, SHELL, SPHERE, Engine, generate

GEN = {"cube": CUBE, "sphere": SPHERE, "shell": SHELL}


def walk_case(args) -> None:
    if args.load:
        z = np.load(args.load)
        pos, vel, mass = z["pos"], z["vel"], z["mass"]
    else:
        pos, vel, mass = generate(args.n, gen_type=GEN[args.gen], size=args.size)
        if args.evolve:
            with Engine(adaptive=1) as e:
                e.set_particles(pos, vel, mass)
                e.step(args.evolve)
                pos, vel = e.get_particles()
        if args.save:
            np.savez(args.save, pos=pos, vel=vel, mass=mass)
    with Engine(precision=1 if args.fp64 else 0) as e:
        e.set_walk_stats(not args.no_walk_stats)
        for _ in range(args.passes):
            e.barnes_hut(pos, mass, theta=args.theta)
        s = e.stats()
    print({k: s[k] for k in ("interactions", "walk_list", "walk_near", "walk_tiles", "walk_decisions",
                             "tree_nodes", "tree_depth", "sort_passes", "sort_split_bits", "sort_tie_runs")})


def adjoint_case(args) -> None:
    pos, vel, mass = generate(args.n, gen_type=SPHERE, size=512.0)
    with Engine(adaptive=0, precision=1 if args.fp64 else 0) as e:
        e.set_particles(pos, vel, mass)
        t0 = time.perf_counter()
        e.forward_checkpointed(args.steps, args.every)
        p, v = e.get_particles()
        t1 = time.perf_counter()
        e.backward(p - pos, None)
        t2 = time.perf_counter()
    print({"forward_s": t1 - t0, "backward_s": t2 - t1})


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="case", required=True)
    w = sub.add_parser("walk")
    w.add_argument("--gen", default="shell", choices=sorted(GEN))
    w.add_argument("--n", type=int, default=1 << 20)
    w.add_argument("--size", type=float, default=1024.0)
    w.add_argument("--evolve", type=int, default=0)
    w.add_argument("--save", default="")
    w.add_argument("--load", default="")
    w.add_argument("--passes", type=int, default=2)
    w.add_argument("--theta", type=float, default=0.5)
    w.add_argument("--fp64", action="store_true")
    w.add_argument("--no-walk-stats", action="store_true",
                   help="run the walk the bench runs (no statistics instance; the printed walk_* are then 0)")
    a = sub.add_parser("adjoint")
    a.add_argument("--n", type=int, default=65536)
    a.add_argument("--steps", type=int, default=256)
    a.add_argument("--every", type=int, default=16)
    a.add_argument("--fp64", action="store_true")
    args = ap.parse_args()
    {"walk": walk_case, "adjoint": adjoint_case}[args.case](args)


if __name__ == "__main__":
    main()
