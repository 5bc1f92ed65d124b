"""The reference's program on the resident GPU state.

    python -m nbodysim_b200.run [settings file]

Follows ``main`` (src/main.cpp:1359-1504): read the settings file (default
``settings.cfg``), resume from the newest ``./data/NNNN.dat`` when
``read_existing`` is set (``read_data``, src/main.cpp:790-811) or generate the
seeded initial conditions, then run ``num_frames`` frames. A frame is one
``nbody_step`` (octree, minimum-size merge, mass/COM, walk and forces,
collision merge, update; src/main.cpp:1420-1478) followed by the dump of
src/main.cpp:680-766: the binary and text frame files with the reference's
overwrite and keep-previous rules, and the image. Between dumps the particles
stay in GPU memory.

Differences, by necessity: the image is written as ``./img/NNNN.ppm`` (the same
bitmap as the reference's PNG; FreeImage is not a dependency of this library),
``cuda`` and ``threads`` are ignored (the frame always runs on the GPU), and
``--datatype-bytes 4`` writes the FLOAT build's records.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

from . import Engine, frame_path, gen_params_from_settings, generate, params_from_settings, write_ppm
from .settings import read_settings


def _image_path(img_dir: str, frame: int) -> str:
    return os.path.join(img_dir, f"{frame:04d}.ppm")  # gen_image, src/main.cpp:293-300


def _clear(path: str, overwrite: bool) -> None:
    """The overwrite check of dump (src/main.cpp:704-721)."""
    if os.path.exists(path):
        if not overwrite:
            print(f"Overwrite disabled, cannot overwrite {path}. Aborting.", file=sys.stderr)
            sys.exit(1)
        os.remove(path)


def dump(eng: Engine, s, frame: int, data_dir: str, img_dir: str, nbytes: int) -> None:
    """One frame's files, as dump (src/main.cpp:680-766) writes them."""
    bfile, tfile = frame_path(data_dir, frame, True), frame_path(data_dir, frame, False)
    ifile = _image_path(img_dir, frame)
    for path in (bfile, tfile, ifile):
        _clear(path, s.overwrite_data)
    if not s.keep_previous_binary and frame > 0:
        prev = frame_path(data_dir, frame - 1, True)
        if os.path.exists(prev):
            os.remove(prev)
    if not s.keep_previous_text and frame > 0:
        prev = frame_path(data_dir, frame - 1, False)
        if os.path.exists(prev):
            os.remove(prev)
    if s.dump_binary or s.dump_text:
        eng.save_frame(data_dir, frame, binary=s.dump_binary, text=s.dump_text, datatype_bytes=nbytes)
    if s.dump_image:
        rgb = eng.render(width=s.img_w, height=s.img_h, projection=s.projection, color=s.color,
                         adaptive=int(s.adaptive_brightness), nonlinear=int(s.nonlinear_brightness), scale=s.scale,
                         brightness=s.brightness)
        write_ppm(ifile, rgb)


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("settings", nargs="?", default="settings.cfg")
    ap.add_argument("--data-dir", default="./data")
    ap.add_argument("--img-dir", default="./img")
    ap.add_argument("--datatype-bytes", type=int, default=8, choices=(8, 4))
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    s = read_settings(args.settings)
    seed = s.seed if s.use_seed else int(time.time())
    eng = Engine(params_from_settings(s, precision=s.precision, device=args.device))
    start = 0
    if s.read_existing:
        start = eng.load_frame(args.data_dir, s.num_frames, args.datatype_bytes)
        print("No data to resume from." if start == 0 else f"Resuming from {start}")
    if not s.read_existing or start == 0:
        print(f"Seed: {seed}")
        print("Generating particles...")
        g = gen_params_from_settings(s)
        g.seed = seed
        pos, vel, mass = generate(s.num_particles, g)
        eng.set_particles(pos, vel, mass)
    if s.dump_image:
        os.makedirs(args.img_dir, exist_ok=True)
    if s.dump_binary or s.dump_text:
        os.makedirs(args.data_dir, exist_ok=True)
    frame = start
    print(f"Frame {frame}/{s.num_frames}", flush=True)
    while frame < s.num_frames:
        eng.step(1)
        if s.verbose:
            st = eng.stats()
            print(f"Number of particles: {eng.n}; interactions {st['interactions']}; dt {st['last_dt']}")
        if s.dump_binary or s.dump_text or s.dump_image:
            dump(eng, s, frame, args.data_dir, args.img_dir, args.datatype_bytes)
        frame += 1
        print(f"Frame {frame}/{s.num_frames}", flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
