"""The reference's configuration keys, defaults and file parser.

Mirrors ``struct settings`` (src/main.cpp:115-160), ``set_default``
(src/main.cpp:1312-1357) and ``read_settings`` (src/main.cpp:1123-1310): a
whitespace-separated stream of ``key value`` tokens; booleans are true only
for the literal ``true``; enum keys take their names (cube/sphere/shell,
linear/exp/normal, front/side/top/iso, bw/heat); bare ``true``/``false``
tokens are skipped; unknown keys are reported as "Unrecognized variable".

Extensions (documented in the reference's README.md:54-60 but not parsed by
its code): ``adaptive``, ``min_adaptive_dt``, ``max_pos_change``,
``max_vel_change``; and this engine's ``precision`` (``mixed`` or ``fp64``).
"""
from __future__ import annotations

import sys
from dataclasses import dataclass, field, fields

_ENUMS = {
    "gen_type": {"cube": 0, "sphere": 1, "shell": 2},
    "mass_dist": {"linear": 0, "exp": 1, "normal": 2},
    "vel_dist": {"linear": 0, "exp": 1, "normal": 2},
    "projection": {"front": 0, "side": 1, "top": 2, "iso": 3},
    "color": {"bw": 0, "heat": 1},
    "precision": {"mixed": 0, "fp64": 1},
}


@dataclass
class Settings:
    read_existing: bool = False
    use_seed: bool = False
    display_progress: bool = True
    dump_binary: bool = True
    dump_text: bool = True
    dump_image: bool = True
    overwrite_data: bool = False
    keep_previous_binary: bool = False
    keep_previous_text: bool = True
    verbose: bool = False
    damping: bool = False
    adaptive_brightness: bool = False
    nonlinear_brightness: bool = False
    collide: bool = False
    cuda: bool = False
    num_particles: int = 5000
    num_frames: int = 300
    threads: int = 1
    img_w: int = 1920
    img_h: int = 1080
    projection: int = 3
    size: float = 512.0
    theta: float = 0.5
    dt: float = 0.0333
    seed: int = 0xDEADBEEF
    min_mass: float = 5e10
    max_mass: float = 5e11
    min_vel: float = 0.0
    max_vel: float = 0.0
    r_sphere: float = 100.0
    rotation_magnitude: float = 0.1
    scale_x: float = 1.0
    scale_y: float = 1.0
    scale_z: float = 1.0
    brightness: float = 255.0
    scale: float = 1.0
    collision_range: float = 0.01
    rotation_vector: tuple = field(default=(0.0, 0.0, 1.0))
    gen_type: int = 0
    mass_dist: int = 0
    vel_dist: int = 0
    color: int = 0
    min_node_size: float = 0.0
    # extensions
    adaptive: bool = False
    min_adaptive_dt: float = 0.00333
    max_pos_change: float = 3.0
    max_vel_change: float = 3.0
    precision: int = 0


def set_default() -> Settings:
    """Defaults of src/main.cpp:1312-1357 (plus the README's adaptive-dt defaults)."""
    return Settings()


def _parse_tokens(s: Settings, tokens: list[str], warn) -> Settings:
    types = {f.name: f.type for f in fields(Settings)}
    i = 0
    while i < len(tokens):
        key = tokens[i]
        i += 1
        if key in ("true", "false"):
            continue
        if key == "rotation_vector":
            s.rotation_vector = tuple(float(t) for t in tokens[i:i + 3])
            i += 3
            continue
        if key not in types:
            warn(f"Unrecognized variable {key}")
            continue
        if i >= len(tokens):
            break
        val = tokens[i]
        i += 1
        t = types[key]
        if key in _ENUMS:
            if val not in _ENUMS[key]:
                raise ValueError(f"invalid value {val!r} for {key}")
            setattr(s, key, _ENUMS[key][val])
        elif t in (bool, "bool"):
            setattr(s, key, val == "true")
        elif t in (int, "int"):
            setattr(s, key, int(val, 0) if key == "seed" else int(val))
        else:
            setattr(s, key, float(val))
    return s


def read_settings(path: str, base: Settings | None = None, warn=None) -> Settings:
    """Parses a reference settings file over `base` (default: set_default())."""
    warn = warn or (lambda m: print(m, file=sys.stderr))
    with open(path) as f:
        tokens = f.read().split()
    return _parse_tokens(base if base is not None else set_default(), tokens, warn)


def parse_settings(text: str, base: Settings | None = None, warn=None) -> Settings:
    warn = warn or (lambda m: print(m, file=sys.stderr))
    return _parse_tokens(base if base is not None else set_default(), text.split(), warn)
