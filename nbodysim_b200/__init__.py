"""nbodysim_b200 -- B200-native Barnes-Hut engine for fosted3/nbodysim's hot path.

Python mirror of the library's C ABI (``include/nbody_b200.h``), loaded with
ctypes from the in-tree ``nbodysim_b200/lib/libnbody_b200.so``. There is no CPU
fallback: if the library is missing or no sm_100 GPU is present, calls raise.

Reference interfaces mirrored here:

* ``Engine.barnes_hut(pos, mass, damping, theta)`` -- ``barnes_hut_cuda(particles,
  root, damping, theta)`` (src/cuda_helper.h:8): overwrites every particle's
  acceleration with the Barnes-Hut sum.
* ``Engine.step`` -- the frame loop's build -> mass -> com -> force -> update
  (src/main.cpp:1420-1492) on resident device state.
* ``Settings`` / ``read_settings`` / ``set_default`` -- the reference's config
  struct, parser and defaults (src/main.cpp:115-160, 1123-1357).
* ``generate`` -- ``generate_particle`` (src/main.cpp:226-275), seeded.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

from .settings import Settings, read_settings, set_default  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnbody_b200.so")

OK = 0
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_COINCIDENT, ERR_NONFINITE, ERR_CAPACITY, ERR_NO_DEVICE, ERR_STATE = range(1, 9)
PRECISION_MIXED, PRECISION_FP64 = 0, 1
CUBE, SPHERE, SHELL = 0, 1, 2
LINEAR, EXP, NORMAL = 0, 1, 2


class NBodyError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("theta", C.c_double), ("dt", C.c_double), ("damping", C.c_int), ("adaptive", C.c_int),
        ("min_adaptive_dt", C.c_double), ("max_pos_change", C.c_double), ("max_vel_change", C.c_double),
        ("precision", C.c_int), ("device", C.c_int), ("autotune", C.c_int),
        ("collide", C.c_int), ("collision_range", C.c_double), ("min_node_size", C.c_double),
        ("datatype_bytes", C.c_int),
    ]


class GenParams(C.Structure):
    _fields_ = [
        ("gen_type", C.c_int), ("mass_dist", C.c_int), ("vel_dist", C.c_int),
        ("size", C.c_double), ("min_mass", C.c_double), ("max_mass", C.c_double),
        ("min_vel", C.c_double), ("max_vel", C.c_double), ("r_sphere", C.c_double),
        ("rotation_magnitude", C.c_double), ("rotation_vector", C.c_double * 3),
        ("scale", C.c_double * 3), ("seed", C.c_uint64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("interactions", C.c_uint64), ("interactions_total", C.c_uint64), ("kernel_launches", C.c_uint64),
        ("walk_entries", C.c_uint64), ("walk_tiles", C.c_uint64), ("walk_decisions", C.c_uint64),
        ("walk_list", C.c_uint64), ("walk_near", C.c_uint64),
        ("walk_warps_per_block", C.c_uint32), ("walk_blocks", C.c_uint32),
        ("tree_nodes", C.c_uint32), ("tree_depth", C.c_uint32),
        ("max_stack", C.c_uint32), ("fallback_tests", C.c_uint32), ("last_dt", C.c_double),
        ("root_center", C.c_double * 3), ("root_side", C.c_double),
        ("ms_tree", C.c_float), ("ms_com", C.c_float), ("ms_walk", C.c_float), ("ms_update", C.c_float),
        ("merged_min_size", C.c_uint64), ("merged_collisions", C.c_uint64), ("collision_pairs", C.c_uint64),
        ("sort_passes", C.c_uint32), ("sort_split_bits", C.c_uint32), ("sort_tie_runs", C.c_uint32),
        ("sort_next_passes", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["root_center"] = tuple(self.root_center)
        return d


class Diagnostics(C.Structure):
    _fields_ = [
        ("kinetic", C.c_double), ("potential", C.c_double), ("momentum", C.c_double * 3),
        ("angular_momentum", C.c_double * 3), ("mass", C.c_double), ("com", C.c_double * 3),
    ]

    def as_dict(self) -> dict:
        return dict(kinetic=self.kinetic, potential=self.potential, energy=self.kinetic + self.potential,
                    momentum=tuple(self.momentum), angular_momentum=tuple(self.angular_momentum),
                    mass=self.mass, com=tuple(self.com))


class ImageParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("projection", C.c_int), ("color", C.c_int),
                ("adaptive", C.c_int), ("nonlinear", C.c_int), ("scale", C.c_double), ("brightness", C.c_double)]


class DeviceView(C.Structure):
    _fields_ = [("n", C.c_uint32), ("pos", C.c_void_p), ("vel", C.c_void_p), ("mass", C.c_void_p),
                ("acc", C.c_void_p), ("acc_is_double", C.c_int)]


# Every entry point of include/nbody_b200.h with its ctypes signature.
_SIGS = {
    "nbody_default_params": (None, [C.POINTER(Params)]),
    "nbody_create": (C.c_int, [C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "nbody_destroy": (C.c_int, [C.c_void_p]),
    "nbody_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "nbody_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nbody_barnes_hut": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                   C.c_void_p, C.c_void_p]),
    "nbody_set_particles": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nbody_set_systems": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p]),
    "nbody_get_particles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nbody_step": (C.c_int, [C.c_void_p, C.c_uint32]),
    "nbody_compute_forces": (C.c_int, [C.c_void_p]),
    "nbody_step_host": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "nbody_device_view_get": (C.c_int, [C.c_void_p, C.POINTER(DeviceView)]),
    "nbody_get_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "nbody_set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "nbody_set_walk_stats": (C.c_int, [C.c_void_p, C.c_int]),
    "nbody_set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "nbody_autotune": (C.c_int, [C.c_void_p]),
    "nbody_get_diagnostics": (C.c_int, [C.c_void_p, C.POINTER(Diagnostics)]),
    "nbody_default_gen_params": (None, [C.POINTER(GenParams)]),
    "nbody_generate": (C.c_int, [C.POINTER(GenParams), C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nbody_status_string": (C.c_char_p, [C.c_int]),
    "nbody_last_error_message": (C.c_char_p, []),
    "nbody_force_vjp": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    "nbody_forward_checkpointed": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "nbody_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "nbody_frame_path": (C.c_int, [C.c_char_p, C.c_uint32, C.c_int, C.c_char_p, C.c_size_t]),
    "nbody_write_dat": (C.c_int, [C.c_char_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "nbody_read_dat": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "nbody_write_txt": (C.c_int, [C.c_char_p, C.c_uint32, C.c_void_p, C.c_int]),
    "nbody_find_resume_frame": (C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(C.c_int32)]),
    "nbody_get_masses": (C.c_int, [C.c_void_p, C.c_void_p]),
    "nbody_direct_forces": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p]),
    "nbody_save_frame": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32, C.c_int, C.c_int, C.c_int]),
    "nbody_load_frame": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32, C.c_int, C.POINTER(C.c_uint32)]),
    "nbody_default_image_params": (None, [C.POINTER(ImageParams)]),
    "nbody_render": (C.c_int, [C.c_void_p, C.POINTER(ImageParams), C.c_void_p]),
    "nbody_write_ppm": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_void_p]),
    "nbody_probe_fp32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "nbody_root_cube_noalloc_max_n": (C.c_uint32, []),
    "nbody_root_cube_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
}

_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m nbodysim_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != OK:
        lib = load_library()
        msg = lib.nbody_last_error_message().decode(errors="replace")
        raise NBodyError(status, f"{lib.nbody_status_string(status).decode()}: {msg}")


def _aos(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3 or (n is not None and a.shape[0] != n):
        raise ValueError("expected an (n, 3) array")
    return a


def _vec(a, n) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.shape[0] != n:
        raise ValueError("expected n masses")
    return a


def _ptr(a):
    return a.ctypes.data if a is not None else None


def default_params(**kw) -> Params:
    p = Params()
    load_library().nbody_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def params_from_settings(s: Settings, **kw) -> Params:
    """Engine parameters from the reference's config keys. As in the reference's
    frame loop (src/main.cpp:1425), min_node_size only takes effect with verbose."""
    return default_params(theta=s.theta, dt=s.dt, damping=int(s.damping), adaptive=int(s.adaptive),
                          min_adaptive_dt=s.min_adaptive_dt, max_pos_change=s.max_pos_change,
                          max_vel_change=s.max_vel_change, collide=int(s.collide),
                          collision_range=s.collision_range,
                          min_node_size=s.min_node_size if s.verbose else 0.0, **kw)


def gen_params(**kw) -> GenParams:
    g = GenParams()
    load_library().nbody_default_gen_params(C.byref(g))
    for k, v in kw.items():
        if k in ("rotation_vector", "scale"):
            getattr(g, k)[:] = [float(x) for x in v]
        else:
            setattr(g, k, v)
    return g


def gen_params_from_settings(s: Settings) -> GenParams:
    return gen_params(gen_type=s.gen_type, mass_dist=s.mass_dist, vel_dist=s.vel_dist, size=s.size,
                      min_mass=s.min_mass, max_mass=s.max_mass, min_vel=s.min_vel, max_vel=s.max_vel,
                      r_sphere=s.r_sphere, rotation_magnitude=s.rotation_magnitude,
                      rotation_vector=s.rotation_vector, scale=(s.scale_x, s.scale_y, s.scale_z),
                      seed=s.seed)


def generate(n: int, g: GenParams | None = None, **kw):
    """Seeded initial conditions: (pos (n,3), vel (n,3), mass (n,)), host arrays."""
    g = g if g is not None else gen_params(**kw)
    pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); mass = np.zeros(n)
    _check(load_library().nbody_generate(C.byref(g), n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data))
    return pos, vel, mass


class Engine:
    """One device context (include/nbody_b200.h `nbody_ctx`)."""

    def __init__(self, params: Params | None = None, **kw):
        lib = load_library()
        self._lib = lib
        self.params = params if params is not None else default_params(**kw)
        h = C.c_void_p()
        _check(lib.nbody_create(C.byref(self.params), C.byref(h)))
        self._h = h
        self.n = 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.nbody_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_params(self, **kw) -> None:
        for k, v in kw.items():
            setattr(self.params, k, v)
        _check(self._lib.nbody_set_params(self._h, C.byref(self.params)))

    def autotune(self) -> dict:
        """Picks the fastest walk block shape on the resident state."""
        _check(self._lib.nbody_autotune(self._h))
        s = self.stats()
        return {"warps_per_block": s["walk_warps_per_block"], "blocks": s["walk_blocks"]}

    def set_graphs(self, on: bool = True) -> None:
        _check(self._lib.nbody_set_graphs(self._h, int(on)))

    def set_timing(self, on: bool = True) -> None:
        _check(self._lib.nbody_set_timing(self._h, int(on)))

    def set_walk_stats(self, on: bool = True) -> None:
        """Collect the walk's statistics (stats() walk_* and max_stack)."""
        _check(self._lib.nbody_set_walk_stats(self._h, int(on)))

    def barnes_hut(self, pos, mass, damping: bool = False, theta: float = 0.5, counts: bool = False):
        """Accelerations (n, 3) of every particle (the reference's barnes_hut_cuda)."""
        pos = _aos(pos)
        n = pos.shape[0]
        mass = _vec(mass, n)
        acc = np.zeros((n, 3))
        cnt = np.zeros(n, np.uint32) if counts else None
        _check(self._lib.nbody_barnes_hut(self._h, n, pos.ctypes.data, mass.ctypes.data, int(damping),
                                          float(theta), acc.ctypes.data, _ptr(cnt)))
        return (acc, cnt) if counts else acc

    def set_systems(self, counts) -> None:
        """Independent systems stored one after another (counts per system)."""
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        _check(self._lib.nbody_set_systems(self._h, len(counts), counts.ctypes.data))

    def set_particles(self, pos, vel, mass) -> None:
        pos = _aos(pos)
        n = pos.shape[0]
        vel = _aos(vel, n) if vel is not None else None
        mass = _vec(mass, n)
        _check(self._lib.nbody_set_particles(self._h, n, pos.ctypes.data, _ptr(vel), mass.ctypes.data))
        self.n = n

    def get_particles(self, acc: bool = False):
        pos = np.zeros((self.n, 3)); vel = np.zeros((self.n, 3))
        a = np.zeros((self.n, 3)) if acc else None
        _check(self._lib.nbody_get_particles(self._h, pos.ctypes.data, vel.ctypes.data, _ptr(a)))
        return (pos, vel, a) if acc else (pos, vel)

    def step(self, nsteps: int = 1) -> None:
        _check(self._lib.nbody_step(self._h, nsteps))
        if self.n and (self.params.collide or self.params.min_node_size > 0):
            self.n = self.device_view().n  # merging may have removed particles

    def direct_forces(self, targets=None, damping: bool = False):
        """FP64 all-pairs accelerations of the resident particles `targets` (default: all)."""
        t = None if targets is None else np.ascontiguousarray(targets, dtype=np.uint32)
        m = self.n if t is None else len(t)
        out = np.zeros((m, 3))
        _check(self._lib.nbody_direct_forces(self._h, m, _ptr(t), int(damping), out.ctypes.data))
        return out

    def get_masses(self):
        m = np.zeros(self.n)
        _check(self._lib.nbody_get_masses(self._h, m.ctypes.data))
        return m

    def compute_forces(self) -> None:
        _check(self._lib.nbody_compute_forces(self._h))

    def step_host(self, pos, vel, mass, nsteps: int = 1):
        """Steps host arrays in place (upload, nsteps, download). Returns (pos, vel)."""
        n = pos.shape[0]
        if pos.dtype != np.float64 or not pos.flags.c_contiguous or vel.dtype != np.float64 \
                or not vel.flags.c_contiguous:
            raise ValueError("pos/vel must be C-contiguous float64 (n, 3) arrays (updated in place)")
        mass = _vec(mass, n)
        _check(self._lib.nbody_step_host(self._h, n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, nsteps))
        self.n = n
        return pos, vel

    def force_vjp(self, pos, mass, dL_dacc):
        """(dL/dpos, dL/dmass) of one force pass with frozen opening decisions."""
        pos = _aos(pos)
        n = pos.shape[0]
        mass = _vec(mass, n)
        la = _aos(dL_dacc, n)
        gp = np.zeros((n, 3)); gm = np.zeros(n)
        _check(self._lib.nbody_force_vjp(self._h, n, pos.ctypes.data, mass.ctypes.data, la.ctypes.data,
                                         gp.ctypes.data, gm.ctypes.data))
        return gp, gm

    def forward_checkpointed(self, nsteps: int, every: int = 0) -> None:
        _check(self._lib.nbody_forward_checkpointed(self._h, nsteps, every))

    def backward(self, dL_dpos, dL_dvel=None):
        """(dL/dpos0, dL/dvel0, dL/dmass) of the last forward_checkpointed."""
        gp = _aos(dL_dpos, self.n)
        gv = _aos(dL_dvel, self.n) if dL_dvel is not None else None
        p0 = np.zeros((self.n, 3)); v0 = np.zeros((self.n, 3)); m0 = np.zeros(self.n)
        _check(self._lib.nbody_backward(self._h, gp.ctypes.data, _ptr(gv), p0.ctypes.data, v0.ctypes.data,
                                        m0.ctypes.data))
        return p0, v0, m0

    def save_frame(self, dir: str, frame: int, binary: bool = True, text: bool = False,
                   datatype_bytes: int = 8) -> None:
        _check(self._lib.nbody_save_frame(self._h, dir.encode(), frame, int(binary), int(text), datatype_bytes))

    def load_frame(self, dir: str, num_frames: int, datatype_bytes: int = 8) -> int:
        """Resumes from the newest binary frame <= num_frames; returns the next frame (0: none found)."""
        nxt = C.c_uint32(0)
        _check(self._lib.nbody_load_frame(self._h, dir.encode(), num_frames, datatype_bytes, C.byref(nxt)))
        if nxt.value:
            self.n = self.device_view().n
        return nxt.value

    def render(self, params: ImageParams | None = None, **kw):
        """The reference's write_image on the resident positions: (height, width, 3) uint8, [y, x]."""
        p = params if params is not None else image_params(**kw)
        out = np.zeros((p.height, p.width, 3), np.uint8)
        _check(self._lib.nbody_render(self._h, C.byref(p), out.ctypes.data))
        return out

    def stats(self) -> dict:
        s = Stats()
        _check(self._lib.nbody_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def diagnostics(self) -> dict:
        d = Diagnostics()
        _check(self._lib.nbody_get_diagnostics(self._h, C.byref(d)))
        return d.as_dict()

    def device_view(self) -> DeviceView:
        v = DeviceView()
        _check(self._lib.nbody_device_view_get(self._h, C.byref(v)))
        return v


def frame_path(dir: str | None, frame: int, binary: bool) -> str:
    buf = C.create_string_buffer(4096)
    _check(load_library().nbody_frame_path(dir.encode() if dir else None, frame, int(binary), buf, 4096))
    return buf.value.decode()


def write_dat(path: str, pos, vel, mass, acc=None, datatype_bytes: int = 8) -> None:
    """The reference's binary frame (resume) format."""
    pos = _aos(pos); n = pos.shape[0]; vel = _aos(vel, n); mass = _vec(mass, n)
    acc = _aos(acc, n) if acc is not None else None
    _check(load_library().nbody_write_dat(path.encode(), n, pos.ctypes.data, vel.ctypes.data, _ptr(acc),
                                          mass.ctypes.data, datatype_bytes))


def read_dat(path: str, datatype_bytes: int = 8):
    """(pos, vel, acc, mass) of a binary frame, in file order."""
    lib = load_library()
    n = C.c_uint32(0)
    _check(lib.nbody_read_dat(path.encode(), datatype_bytes, C.byref(n), None, None, None, None))
    pos = np.zeros((n.value, 3)); vel = np.zeros((n.value, 3)); acc = np.zeros((n.value, 3)); mass = np.zeros(n.value)
    _check(lib.nbody_read_dat(path.encode(), datatype_bytes, C.byref(n), pos.ctypes.data, vel.ctypes.data,
                              acc.ctypes.data, mass.ctypes.data))
    return pos, vel, acc, mass


def write_txt(path: str, pos, datatype_bytes: int = 8) -> None:
    pos = _aos(pos)
    _check(load_library().nbody_write_txt(path.encode(), pos.shape[0], pos.ctypes.data, datatype_bytes))


def find_resume_frame(dir: str, num_frames: int) -> int:
    f = C.c_int32(0)
    _check(load_library().nbody_find_resume_frame(dir.encode(), num_frames, C.byref(f)))
    return f.value


def image_params(**kw) -> ImageParams:
    p = ImageParams()
    load_library().nbody_default_image_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def write_ppm(path: str, rgb) -> None:
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    h, w, _ = rgb.shape
    _check(load_library().nbody_write_ppm(path.encode(), w, h, rgb.ctypes.data))


def probe_fp32_peak(device: int = 0) -> tuple[float, float]:
    """Measured FP32 FMA throughput (TFLOP/s) and the probe kernel's time (ms)."""
    tf = C.c_double(); ms = C.c_double()
    _check(load_library().nbody_probe_fp32_peak(device, C.byref(tf), C.byref(ms)))
    return tf.value, ms.value


def header_symbols(path: str | None = None) -> list[str]:
    """Names of the functions declared in include/*.h."""
    import glob
    import re
    inc = os.path.join(os.path.dirname(HERE), "include")
    paths = [path] if path else sorted(glob.glob(os.path.join(inc, "*.h")))
    names = set()
    for p in paths:
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(nbody_\w+)\s*\(", open(p).read(), re.M))
    return sorted(names)


__all__ = ["Engine", "NBodyError", "Params", "GenParams", "Settings", "read_settings", "set_default",
           "generate", "gen_params", "default_params", "load_library", "params_from_settings",
           "gen_params_from_settings", "header_symbols"]
if sys.version_info < (3, 9):  # pragma: no cover
    raise ImportError("python >= 3.9 required")
