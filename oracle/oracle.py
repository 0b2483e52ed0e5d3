"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs as the checker and as the
timed CPU baseline.  The product package never imports this module.

The class mirrors the product's :class:`pigment_mixing_b200.Simulation` call surface so that
a parity test can drive both with the same scene description.  The restated algorithm lives in
``mpm_oracle.cpp`` (reference: matter/src/simulation/simulation.cpp:225-291 and the files it calls).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build(reference_root: str | None = None) -> None:
    """Compile the oracle libraries, and oracle/_ref from the reference tree at reference_root
    (default: the environment variable PM_REFERENCE_ROOT) when that tree is present."""
    ref = reference_root if reference_root is not None else os.environ.get("PM_REFERENCE_ROOT", "")
    subprocess.run(["make", "-s", "-C", _HERE, f"REF={ref}"], check=True)


def _lib(fast: bool = False) -> C.CDLL:
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(_HERE, "_build", name)
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    vp, dp, fp, up = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint)
    lib.pmo_create.restype = vp
    lib.pmo_create.argtypes = [C.c_int]
    lib.pmo_destroy.argtypes = [vp]
    lib.pmo_set_param.argtypes = [vp, C.c_char_p, C.c_double]
    lib.pmo_get_param.argtypes = [vp, C.c_char_p, dp]
    lib.pmo_set_param3.argtypes = [vp, C.c_char_p, dp]
    lib.pmo_set_particles.argtypes = [vp, C.c_uint, fp, fp, fp]
    lib.pmo_add_plate.argtypes = [vp, C.c_double, C.c_int, C.c_int] + [C.c_double] * 8
    lib.pmo_add_spatula.argtypes = [vp, C.c_int, C.c_double, fp, C.c_uint]
    lib.pmo_add_box_knife.argtypes = [vp, C.c_int, C.c_double, dp, dp, C.c_uint, C.c_double, dp]
    lib.pmo_add_ground.argtypes = [vp, C.c_int, C.c_double, C.c_double]
    lib.pmo_add_curve.argtypes = [vp, C.c_int, C.c_double]
    lib.pmo_prepare.argtypes = [vp]
    lib.pmo_step.argtypes = [vp, C.c_uint]
    lib.pmo_advance.argtypes = [vp, C.c_uint, up]
    lib.pmo_simulate.argtypes = [vp]
    lib.pmo_frame_finished.argtypes = [vp, C.POINTER(C.c_int)]
    lib.pmo_is_finished.argtypes = [vp, C.POINTER(C.c_int)]
    lib.pmo_get_grid_boundaries.argtypes = [vp, dp, dp]
    lib.pmo_get_particles.argtypes = [vp, fp, fp, fp, fp, C.POINTER(C.c_ubyte), fp, fp, fp]
    lib.pmo_get_particles_f64.argtypes = [vp, dp, dp, dp]
    lib.pmo_get_grid.argtypes = [vp, dp, up, fp, fp, fp, fp, fp, fp]
    lib.pmo_get_knife.argtypes = [vp, dp, dp, dp]
    lib.pmo_svd3.argtypes = [dp, dp, dp, dp]
    lib.pmo_sd_spatula.argtypes = [dp]
    lib.pmo_sd_spatula.restype = C.c_double
    lib.pmo_slerp.argtypes = [dp, dp, C.c_double, dp]
    _LIBS[name] = lib
    return lib


def _f(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class OracleSim:
    """One oracle simulation.  ``precision`` 64 is the FP64 oracle, 32 the float restatement."""

    def __init__(self, precision: int = 64, fast: bool = False):
        self.lib = _lib(fast)
        self.h = self.lib.pmo_create(precision)
        self.np = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.pmo_destroy(h)
            self.h = None

    # -- parameters -------------------------------------------------------------------
    def set(self, **kw):
        for k, v in kw.items():
            if isinstance(v, (list, tuple, np.ndarray)):
                a = np.ascontiguousarray(v, dtype=np.float64)
                rc = self.lib.pmo_set_param3(self.h, k.encode(), _d(a))
            else:
                rc = self.lib.pmo_set_param(self.h, k.encode(), float(v))
            if rc != 0:
                raise KeyError(k)
        return self

    def get(self, name: str) -> float:
        out = C.c_double()
        if self.lib.pmo_get_param(self.h, name.encode(), C.byref(out)) != 0:
            raise KeyError(name)
        return out.value

    # -- scene --------------------------------------------------------------------------
    def set_particles(self, x, latent=None, v=None):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        lat = None if latent is None else np.ascontiguousarray(latent, dtype=np.float32)
        vv = None if v is None else np.ascontiguousarray(v, dtype=np.float32)
        self.lib.pmo_set_particles(self.h, n, _f(x), _f(lat), _f(vv))
        self.np = n

    def add_plate(self, pos, plate_type, bc, friction=0.0, lower=-1e15, upper=1e15, vx=0.0, vy=0.0, vz=0.0,
                  vmin_factor=1.0, load_factor=0.0):
        self.lib.pmo_add_plate(self.h, pos, plate_type, bc, friction, lower, upper, vx, vy, vz, vmin_factor,
                               load_factor)

    def add_spatula(self, bc, friction, frames):
        fr = np.ascontiguousarray(frames, dtype=np.float32).reshape(-1, 7)
        self.lib.pmo_add_spatula(self.h, bc, friction, _f(fr), fr.shape[0])

    def add_box_knife(self, bc, friction, half, waypoints, speed, quat_wxyz=(1.0, 0.0, 0.0, 0.0)):
        h = np.ascontiguousarray(half, dtype=np.float64)
        w = np.ascontiguousarray(waypoints, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(quat_wxyz, dtype=np.float64)
        self.lib.pmo_add_box_knife(self.h, bc, friction, _d(h), _d(w), w.shape[0], speed, _d(q))

    def add_ground(self, bc, friction, y0=0.0):
        self.lib.pmo_add_ground(self.h, bc, friction, y0)

    def add_curve(self, bc, friction):
        self.lib.pmo_add_curve(self.h, bc, friction)

    # -- stepping -------------------------------------------------------------------------
    def prepare(self):
        self.lib.pmo_prepare(self.h)

    def step(self, n: int = 1):
        self.lib.pmo_step(self.h, n)

    def advance(self, n: int) -> int:
        fd = C.c_uint()
        self.lib.pmo_advance(self.h, n, C.byref(fd))
        return fd.value

    def simulate(self):
        self.lib.pmo_simulate(self.h)

    def frame_finished(self) -> bool:
        o = C.c_int()
        self.lib.pmo_frame_finished(self.h, C.byref(o))
        return bool(o.value)

    def is_finished(self) -> bool:
        o = C.c_int()
        self.lib.pmo_is_finished(self.h, C.byref(o))
        return bool(o.value)

    # -- readback -------------------------------------------------------------------------
    def grid_boundaries(self):
        lo, hi = np.zeros(3), np.zeros(3)
        self.lib.pmo_get_grid_boundaries(self.h, _d(lo), _d(hi))
        return lo, hi

    def particles(self) -> dict:
        n = self.np
        out = dict(x=np.zeros((n, 3), np.float32), v=np.zeros((n, 3), np.float32),
                   latent=np.zeros((n, 7), np.float32), diffusion=np.zeros(n, np.float32),
                   active=np.zeros(n, np.uint8), F=np.zeros((n, 3, 3), np.float32),
                   B=np.zeros((n, 3, 3), np.float32), plastic=np.zeros((n, 4), np.float32))
        self.lib.pmo_get_particles(self.h, _f(out["x"]), _f(out["v"]), _f(out["latent"]), _f(out["diffusion"]),
                                   out["active"].ctypes.data_as(C.POINTER(C.c_ubyte)), _f(out["F"]), _f(out["B"]),
                                   _f(out["plastic"]))
        return out

    def particles_f64(self) -> dict:
        n = self.np
        out = dict(x=np.zeros((n, 3)), v=np.zeros((n, 3)), latent=np.zeros((n, 7)))
        self.lib.pmo_get_particles_f64(self.h, _d(out["x"]), _d(out["v"]), _d(out["latent"]))
        return out

    def grid(self) -> dict:
        origin = np.zeros(3)
        dims = np.zeros(3, np.uint32)
        self.lib.pmo_get_grid(self.h, _d(origin), dims.ctypes.data_as(C.POINTER(C.c_uint)), None, None, None,
                              None, None, None)
        n = int(dims.prod())
        out = dict(origin=origin, dims=dims.astype(int), mass=np.zeros(n, np.float32),
                   v_update=np.zeros((n, 3), np.float32), v=np.zeros((n, 3), np.float32),
                   flip=np.zeros((n, 3), np.float32), latent=np.zeros((n, 7), np.float32),
                   shear=np.zeros(n, np.float32))
        self.lib.pmo_get_grid(self.h, _d(origin), dims.ctypes.data_as(C.POINTER(C.c_uint)), _f(out["mass"]),
                              _f(out["v_update"]), _f(out["v"]), _f(out["flip"]), _f(out["latent"]),
                              _f(out["shear"]))
        return out

    def knife(self):
        inv = np.zeros(16)
        vl, om = np.zeros(3), np.zeros(3)
        if self.lib.pmo_get_knife(self.h, _d(inv), _d(vl), _d(om)) != 0:
            return None
        return inv.reshape(4, 4), vl, om


def svd3(A):
    A = np.ascontiguousarray(A, dtype=np.float64)
    U, s, V = np.zeros((3, 3)), np.zeros(3), np.zeros((3, 3))
    _lib().pmo_svd3(_d(A), _d(U), _d(s), _d(V))
    return U, s, V


def sd_spatula(p):
    p = np.ascontiguousarray(p, dtype=np.float64)
    return _lib().pmo_sd_spatula(_d(p))


def slerp(q0, q1, t):
    a = np.ascontiguousarray(q0, dtype=np.float64)
    b = np.ascontiguousarray(q1, dtype=np.float64)
    o = np.zeros(4)
    _lib().pmo_slerp(_d(a), _d(b), float(t), _d(o))
    return o


def mixbox_ref_lib():
    """The reference's mixbox compiled in place (oracle/_ref), or None when absent."""
    path = os.path.join(_HERE, "_ref", "libmixbox_ref.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    lib.mixbox_float_rgb_to_latent.argtypes = [C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float)]
    lib.mixbox_latent_to_float_rgb.argtypes = [C.POINTER(C.c_float)] + [C.POINTER(C.c_float)] * 3
    return lib
