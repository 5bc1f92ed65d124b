"""Test infrastructure only: the oracle.

Python access to the two CPU checkers of the Barnes-Hut hot path:

* ``Reference`` -- ``oracle/_ref/libnbref.so``: fosted3/nbodysim's own CPU path
  (``src/main.cpp``, ``src/octree.cpp``, ``src/particle.cpp``, ``src/vector.cpp``)
  compiled unmodified by ``oracle/Makefile`` and wrapped by ``ref_harness.cpp``.
* ``Oracle`` -- ``oracle/lib/libbh_oracle.so``: the plain-C restatement in
  ``bh_oracle.c`` (bit-identical to the reference in the DOUBLE build) plus an
  FP64 direct-sum oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, as the checker. The product (``nbodysim_b200``)
never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libnbref.so")
REF_LIB_F32 = os.path.join(HERE, "_ref", "libnbref_f32.so")
# the DOUBLE build with the reference's release flags (-march=x86-64-v3 for
# -march=native): the timed CPU baseline, not a parity checker
REF_LIB_REL = os.path.join(HERE, "_ref", "libnbref_rel.so")


def release_build_usable() -> bool:
    """The release build needs AVX2, FMA and BMI2 on the host running it."""
    if not os.path.exists(REF_LIB_REL):
        return False
    try:
        flags = open("/proc/cpuinfo").read().split()
    except OSError:
        return False
    return all(f in flags for f in ("avx2", "fma", "bmi2"))
ORACLE_LIB = os.path.join(HERE, "lib", "libbh_oracle.so")

CUBE, SPHERE, SHELL = 0, 1, 2
LINEAR, EXP, NORMAL = 0, 1, 2


@dataclass
class GenParams:
    """Initial-condition keys of the reference config (src/main.cpp:115-160, defaults 1312-1357)."""

    gen_type: int = CUBE
    mass_dist: int = LINEAR
    vel_dist: int = LINEAR
    size: float = 512.0
    min_mass: float = 5e10
    max_mass: float = 5e11
    min_vel: float = 0.0
    max_vel: float = 0.0
    r_sphere: float = 100.0
    rotation_magnitude: float = 0.1
    rotation_vector: tuple = field(default=(0.0, 0.0, 1.0))
    scale: tuple = field(default=(1.0, 1.0, 1.0))
    seed: int = 0xDEADBEEF


class _CGen(C.Structure):
    _fields_ = [
        ("gen_type", C.c_int), ("mass_dist", C.c_int), ("vel_dist", C.c_int),
        ("size", C.c_double), ("min_mass", C.c_double), ("max_mass", C.c_double),
        ("min_vel", C.c_double), ("max_vel", C.c_double), ("r_sphere", C.c_double),
        ("rotation_magnitude", C.c_double),
        ("rot_x", C.c_double), ("rot_y", C.c_double), ("rot_z", C.c_double),
        ("scale_x", C.c_double), ("scale_y", C.c_double), ("scale_z", C.c_double),
        ("seed", C.c_ulong),
    ]


def _cgen(g: GenParams) -> _CGen:
    return _CGen(g.gen_type, g.mass_dist, g.vel_dist, g.size, g.min_mass, g.max_mass,
                 g.min_vel, g.max_vel, g.r_sphere, g.rotation_magnitude,
                 *[float(v) for v in g.rotation_vector], *[float(v) for v in g.scale],
                 g.seed)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _up(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Reference:
    """The reference's own CPU code (DOUBLE build by default; REF_LIB_F32 is its FLOAT build)."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_generate.argtypes = [C.POINTER(_CGen), C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_forces.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_uint,
                                 C.c_void_p, C.c_void_p]
        L.ref_forces_sample.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_uint,
                                        C.c_void_p, C.c_uint, C.c_void_p, C.c_void_p]
        L.ref_run_frames.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                     C.c_double, C.c_uint, C.c_uint, C.c_void_p]
        L.ref_tree_nodes.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_uint, C.c_int,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        L.ref_write_image.argtypes = [C.c_uint, C.c_void_p, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_int, C.c_int,
                                      C.c_double, C.c_double, C.c_void_p]
        L.ref_frame_merging.argtypes = [C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                        C.c_double, C.c_int, C.c_double, C.c_double, C.c_uint,
                                        C.POINTER(C.c_uint), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        self.datatype_bytes = L.ref_datatype_bytes()

    def generate(self, g: GenParams, n: int):
        pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); mass = np.zeros(n)
        self.lib.ref_generate(C.byref(_cgen(g)), n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data)
        return pos, vel, mass

    def forces(self, pos, mass, theta=0.5, damping=False, threads=1):
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        acc = np.zeros((n, 3)); t = np.zeros(3)
        self.lib.ref_forces(n, pos.ctypes.data, mass.ctypes.data, theta, int(damping), threads,
                            acc.ctypes.data, t.ctypes.data)
        return acc, t

    def forces_sample(self, pos, mass, sample, theta=0.5, damping=False, threads=1):
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        sample = np.ascontiguousarray(sample, dtype=np.uint32); m = len(sample)
        acc = np.zeros((m, 3)); t = np.zeros(3)
        self.lib.ref_forces_sample(n, pos.ctypes.data, mass.ctypes.data, theta, int(damping), threads,
                                   sample.ctypes.data, m, acc.ctypes.data, t.ctypes.data)
        return acc, t

    def run_frames(self, pos, vel, mass, frames, theta=0.5, damping=False, dt=0.0333, threads=1,
                   keep_frames=False):
        pos = _c64(pos).copy(); vel = _c64(vel).copy(); mass = _c64(mass); n = len(mass)
        out = np.zeros((frames, n, 3)) if keep_frames else None
        self.lib.ref_run_frames(n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, theta, int(damping),
                                dt, threads, frames, out.ctypes.data if out is not None else None)
        return pos, vel, out

    def frame_merging(self, pos, vel, mass, theta=0.5, damping=False, dt=0.0333, collide=False,
                      collision_range=0.01, min_size=0.0):
        """One reference frame with collisions and/or apply_minimum_size; returns the
        surviving particles (pos, vel, acc, mass) in the set's iteration order."""
        pos = np.ascontiguousarray(pos, dtype=np.float64); vel = np.ascontiguousarray(vel, dtype=np.float64)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        n = len(mass)
        po = np.zeros((n, 3)); vo = np.zeros((n, 3)); ao = np.zeros((n, 3)); mo = np.zeros(n)
        k = C.c_uint(0)
        self.lib.ref_frame_merging(n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, C.c_double(theta),
                                   int(damping), C.c_double(dt), int(collide), C.c_double(collision_range),
                                   C.c_double(min_size), n, C.byref(k), po.ctypes.data, vo.ctypes.data,
                                   ao.ctypes.data, mo.ctypes.data)
        m = k.value
        return po[:m], vo[:m], ao[:m], mo[:m]

    def write_image(self, pos, width=1920, height=1080, projection=3, color=0, adaptive=False, nonlinear=False,
                    scale=1.0, brightness=255.0):
        """The reference's write_image; returns an (height, width, 3) uint8 array indexed [y, x]."""
        pos = _c64(pos)
        out = np.zeros((height, width, 3), np.uint8)
        rc = self.lib.ref_write_image(len(pos), pos.ctypes.data, width, height, projection, color, int(adaptive),
                                      int(nonlinear), scale, brightness, out.ctypes.data)
        if rc:
            raise RuntimeError("reference write_image failed")
        return out

    def tree_nodes(self, pos, mass, threads=1):
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        depth = C.c_int(0)
        cap = 2 * n + 8
        lv = np.zeros(cap, np.int32); ct = np.zeros(cap, np.int32); mi = np.zeros(cap, np.int32)
        nm = np.zeros(cap); com = np.zeros((cap, 3)); sd = np.zeros(cap)
        k = self.lib.ref_tree_nodes(n, pos.ctypes.data, mass.ctypes.data, threads, cap, lv.ctypes.data,
                                    ct.ctypes.data, mi.ctypes.data, nm.ctypes.data, com.ctypes.data,
                                    sd.ctypes.data, C.byref(depth))
        return dict(level=lv[:k], count=ct[:k], min_index=mi[:k], mass=nm[:k], com=com[:k],
                    side=sd[:k], depth=depth.value)


class Oracle:
    """The C restatement (bh_oracle.c) and the FP64 direct sum."""

    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        self.lib = C.CDLL(path)
        L = self.lib
        L.bho_generate.argtypes = [C.POINTER(_CGen), C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.bho_root_cube.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.bho_root_cube_f32.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.bho_build.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p]
        L.bho_build.restype = C.c_void_p
        L.bho_build_f32.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p]
        L.bho_build_f32.restype = C.c_void_p
        L.bho_update_f32.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.bho_free.argtypes = [C.c_void_p]
        L.bho_node_count.argtypes = [C.c_void_p]
        L.bho_node_count.restype = C.c_int64
        L.bho_depth.argtypes = [C.c_void_p]
        L.bho_forces.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_uint32,
                                 C.c_void_p, C.c_void_p]
        L.bho_update.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]
        L.bho_run_frames.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                     C.c_double, C.c_int, C.c_uint32, C.c_void_p]
        L.bho_run_frames_f32.argtypes = L.bho_run_frames.argtypes
        L.bho_direct.argtypes = [C.c_uint32, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_uint32,
                                 C.c_int, C.c_void_p]
        L.bho_tree_nodes.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]

    def generate(self, g: GenParams, n: int):
        pos = np.zeros((n, 3)); vel = np.zeros((n, 3)); mass = np.zeros(n)
        rc = self.lib.bho_generate(C.byref(_cgen(g)), n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data)
        if rc:
            raise ValueError("invalid generation parameters")
        return pos, vel, mass

    def root_cube(self, pos, single=False):
        """Root cube; single=True: as the reference's FLOAT build computes it."""
        pos = _c64(pos)
        c = np.zeros(3); s = np.zeros(1)
        fn = self.lib.bho_root_cube_f32 if single else self.lib.bho_root_cube
        fn(len(pos), pos.ctypes.data, c.ctypes.data, s.ctypes.data)
        return c, float(s[0])

    def _build(self, pos, mass, single):
        fn = self.lib.bho_build_f32 if single else self.lib.bho_build
        return fn(len(mass), pos.ctypes.data, mass.ctypes.data)

    def forces(self, pos, mass, theta=0.5, damping=False, threads=None, sample=None, with_stats=False,
               single=False):
        """Accelerations (and per-particle accepted-node counts) from the BH walk.
        single=True follows the reference's FLOAT build (results are floats)."""
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        threads = threads or os.cpu_count() or 1
        t = self._build(pos, mass, single)
        if not t and n:
            raise RuntimeError("oracle tree build failed (coincident particles or out of memory)")
        try:
            if sample is not None:
                sample = np.ascontiguousarray(sample, dtype=np.uint32)
                m = len(sample)
            else:
                m = n
            acc = np.zeros((m, 3)); cnt = np.zeros(m, np.uint32)
            if n:
                rc = self.lib.bho_forces(t, theta, int(damping), threads,
                                         sample.ctypes.data if sample is not None else None, m,
                                         acc.ctypes.data, cnt.ctypes.data)
                if rc:
                    raise RuntimeError("oracle walk failed")
            stats = dict(nodes=int(self.lib.bho_node_count(t)) if n else 0,
                         depth=int(self.lib.bho_depth(t)) if n else 0)
        finally:
            if t:
                self.lib.bho_free(t)
        if with_stats:
            return acc, cnt, stats
        return acc, cnt

    def tree_nodes(self, pos, mass, single=False):
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        t = self._build(pos, mass, single)
        cap = 4 * n + 8
        lv = np.zeros(cap, np.int32); ct = np.zeros(cap, np.int32); mi = np.zeros(cap, np.int32)
        nm = np.zeros(cap); com = np.zeros((cap, 3)); sd = np.zeros(cap)
        try:
            k = self.lib.bho_tree_nodes(t, cap, lv.ctypes.data, ct.ctypes.data, mi.ctypes.data,
                                        nm.ctypes.data, com.ctypes.data, sd.ctypes.data)
            depth = int(self.lib.bho_depth(t))
        finally:
            self.lib.bho_free(t)
        return dict(level=lv[:k], count=ct[:k], min_index=mi[:k], mass=nm[:k], com=com[:k],
                    side=sd[:k], depth=depth)

    def update(self, pos, vel, acc, dt, single=False):
        pos = _c64(pos).copy(); vel = _c64(vel).copy(); acc = _c64(acc)
        fn = self.lib.bho_update_f32 if single else self.lib.bho_update
        fn(len(pos), pos.ctypes.data, vel.ctypes.data, acc.ctypes.data, dt)
        return pos, vel

    def run_frames(self, pos, vel, mass, frames, theta=0.5, damping=False, dt=0.0333, threads=None,
                   keep_frames=False, single=False):
        pos = _c64(pos).copy(); vel = _c64(vel).copy(); mass = _c64(mass); n = len(mass)
        if single:
            pos = pos.astype(np.float32).astype(np.float64)
            vel = vel.astype(np.float32).astype(np.float64)
        out = np.zeros((frames, n, 3)) if keep_frames else None
        fn = self.lib.bho_run_frames_f32 if single else self.lib.bho_run_frames
        rc = fn(n, pos.ctypes.data, vel.ctypes.data, mass.ctypes.data, theta,
                                     int(damping), dt, threads or os.cpu_count() or 1, frames,
                                     out.ctypes.data if out is not None else None)
        if rc:
            raise RuntimeError(f"oracle run failed ({rc})")
        return pos, vel, out

    def direct(self, pos, mass, targets=None, damping=False, threads=None):
        """FP64 direct-sum accelerations (compensated) for `targets` (default: all)."""
        pos = _c64(pos); mass = _c64(mass); n = len(mass)
        if targets is not None:
            targets = np.ascontiguousarray(targets, dtype=np.uint32)
            m = len(targets)
        else:
            m = n
        acc = np.zeros((m, 3))
        self.lib.bho_direct(n, pos.ctypes.data, mass.ctypes.data, int(damping),
                            targets.ctypes.data if targets is not None else None, m,
                            threads or os.cpu_count() or 1, acc.ctypes.data)
        return acc


def rel_err(a, b):
    """Per-particle relative acceleration error |a - b| / |b| (b is the reference)."""
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    den = np.linalg.norm(b, axis=1)
    num = np.linalg.norm(a - b, axis=1)
    den = np.where(den > 0, den, 1.0)
    return num / den
