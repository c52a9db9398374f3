"""ctypes wrapper of the CPU oracle (liboracle.so, built from spectral_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the checker that tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg compare against.  The product path never imports it.
``dtype=np.float32`` runs the reference's FP32 path, ``np.float64`` its dprec path.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-C", HERE], stdout=subprocess.DEVNULL)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.orc_create_f32.restype = ctypes.c_void_p
        _lib.orc_create_f64.restype = ctypes.c_void_p
        for suf in ("f32", "f64"):
            getattr(_lib, f"orc_destroy_{suf}").argtypes = [ctypes.c_void_p]
    return _lib


class OrcParams(ctypes.Structure):
    _fields_ = [("size_x", ctypes.c_uint64), ("size_y", ctypes.c_uint64), ("delta", ctypes.c_uint64),
                ("dt", ctypes.c_double), ("c", ctypes.c_double), ("dens", ctypes.c_uint32),
                ("gamma_inj", ctypes.c_double), ("n_pass", ctypes.c_uint32), ("periodic_x", ctypes.c_int32),
                ("left_wall", ctypes.c_int32)]


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


FIELD_IDS = {"Ex": 0, "Ey": 1, "Ez": 2, "Bx": 3, "By": 4, "Bz": 5, "Jx": 6, "Jy": 7, "Jz": 8,
             "Rho": 9, "Dens": 10}


class OracleSim:
    """CPU restatement of the reference's Sim + Flds + Vec<Prtl>."""

    def __init__(self, size_x, size_y, delta, dt, c, dens, gamma_inj, n_pass, periodic_x, dtype=np.float32,
                 left_wall=False):
        self.lib = load()
        self.dtype = np.dtype(dtype)
        self.suf = "f32" if self.dtype == np.float32 else "f64"
        self.size_x, self.size_y = size_x, size_y
        self.dt, self.c = dt, c
        prm = OrcParams(size_x, size_y, delta, dt, c, dens, gamma_inj, n_pass, 1 if periodic_x else 0,
                        1 if left_wall else 0)
        self.h = ctypes.c_void_p(getattr(self.lib, f"orc_create_{self.suf}")(ctypes.byref(prm)))
        if not self.h:
            raise ValueError("bad oracle parameters")
        self.nspecies = 0
        self.counts = []

    @staticmethod
    def from_params(p, dtype=np.float32):
        return OracleSim(p.size_x, p.size_y, p.delta, p.dt, p.c, p.dens, p.gamma_inj, p.n_pass, p.periodic_x,
                         dtype, getattr(p, "left_wall", False))

    def close(self):
        if self.h:
            getattr(self.lib, f"orc_destroy_{self.suf}")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _f(self, name):
        return getattr(self.lib, f"orc_{name}_{self.suf}")

    def _chk(self, code, what):
        if code != 0:
            raise RuntimeError(f"oracle {what} failed with code {code}")

    def add_species(self, charge, mass, vth, ix, iy, dx, dy, px, py, pz, psa):
        t = self.dtype
        arrs = [np.ascontiguousarray(ix, dtype=np.uint64), np.ascontiguousarray(iy, dtype=np.uint64)]
        arrs += [np.ascontiguousarray(a, dtype=t) for a in (dx, dy, px, py, pz, psa)]
        self._chk(self._f("add_species")(self.h, ctypes.c_double(charge), ctypes.c_double(mass),
                                         ctypes.c_double(vth), ctypes.c_uint64(len(ix)), *[_p(a) for a in arrs]),
                  "add_species")
        self.nspecies += 1
        self.counts.append(len(ix))
        return self.nspecies - 1

    def state(self, s):
        n = self.counts[s]
        out = {k: np.empty(n, dtype=np.uint64) for k in ("ix", "iy")}
        out.update({k: np.empty(n, dtype=self.dtype) for k in ("dx", "dy", "px", "py", "pz", "psa")})
        self._chk(self._f("get_species")(self.h, s, *[_p(out[k]) for k in
                                                      ("ix", "iy", "dx", "dy", "px", "py", "pz", "psa")]),
                  "get_species")
        return out

    def move_and_deposit(self, s):
        self._chk(self._f("move_and_deposit")(self.h, s), "move_and_deposit")

    def boris_push(self, s):
        self._chk(self._f("boris_push")(self.h, s), "boris_push")

    def zero_sources(self):
        self._f("zero_sources")(self.h)

    def fold_sources(self):
        self._f("fold_sources")(self.h)

    def fields_update(self):
        self._f("fields_update")(self.h)

    def prepare(self):
        self._chk(self._f("prepare")(self.h), "prepare")

    def step(self, n=1):
        self._chk(self._f("step")(self.h, ctypes.c_uint32(n)), "step")

    def spatial(self, name):
        out = np.empty((self.size_y + 2, self.size_x + 2), dtype=self.dtype)
        self._chk(self._f("get_field")(self.h, FIELD_IDS[name], _p(out)), "get_field")
        return out

    def set_spatial(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        self._chk(self._f("set_field")(self.h, FIELD_IDS[name], _p(a)), "set_field")

    def b_wrk(self, comp):
        out = np.empty((self.size_y, self.size_x), dtype=np.complex64 if self.suf == "f32" else np.complex128)
        self._chk(self._f("get_bwrk")(self.h, comp, _p(out)), "get_bwrk")
        return out

    def set_b_wrk(self, comp, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex64 if self.suf == "f32" else np.complex128)
        self._chk(self._f("set_bwrk")(self.h, comp, _p(a)), "set_bwrk")


def field_op(size_x, size_y, op, spatial, n_pass=0, dtype=np.float64):
    lib = load()
    a = np.ascontiguousarray(spatial, dtype=dtype).copy()
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_field_op_{suf}")(ctypes.c_uint64(size_x), ctypes.c_uint64(size_y), op, _p(a),
                                         ctypes.c_uint32(n_pass))
    return a


def copy_to_spectral(size_x, size_y, spatial, dtype=np.float64):
    lib = load()
    a = np.ascontiguousarray(spatial, dtype=dtype)
    ct = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    out = np.empty(size_x * size_y, dtype=ct)
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_copy_to_spectral_{suf}")(ctypes.c_uint64(size_x), ctypes.c_uint64(size_y), _p(a), _p(out))
    return out


def copy_to_spatial(size_x, size_y, spectral, dtype=np.float64):
    lib = load()
    ct = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    a = np.ascontiguousarray(spectral, dtype=ct)
    out = np.empty((size_x + 2) * (size_y + 2), dtype=dtype)
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_copy_to_spatial_{suf}")(ctypes.c_uint64(size_x), ctypes.c_uint64(size_y), _p(a), _p(out))
    return out


def fft2d(data, inverse=False, dtype=np.float64):
    lib = load()
    ct = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    a = np.ascontiguousarray(data, dtype=ct).copy()
    ny, nx = a.shape
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_fft2d_{suf}")(ctypes.c_uint64(nx), ctypes.c_uint64(ny), _p(a), 1 if inverse else 0)
    return a


def fft1d(data, inverse=False, dtype=np.float64):
    lib = load()
    ct = np.complex64 if np.dtype(dtype) == np.float32 else np.complex128
    a = np.ascontiguousarray(data, dtype=ct).copy()
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_fft1d_{suf}")(ctypes.c_uint64(len(a)), _p(a), 1 if inverse else 0)
    return a


def wave_numbers(size_x, size_y, dtype=np.float64):
    lib = load()
    kx, ky, kn = (np.empty(size_x * size_y, dtype=dtype) for _ in range(3))
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    getattr(lib, f"orc_wave_numbers_{suf}")(ctypes.c_uint64(size_x), ctypes.c_uint64(size_y), _p(kx), _p(ky), _p(kn))
    return kx, ky, kn


def init_velocities(normals, uniforms, c, vth, gamma_inj, sign=1.0, dtype=np.float32):
    lib = load()
    n = len(uniforms)
    nrm = np.ascontiguousarray(normals, dtype=dtype)
    uni = np.ascontiguousarray(uniforms, dtype=dtype)
    px, py, pz, psa = (np.empty(n, dtype=dtype) for _ in range(4))
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    f = getattr(lib, f"orc_init_velocities_{suf}")
    f(ctypes.c_uint64(n), ctypes.c_double(c), ctypes.c_double(vth), ctypes.c_double(gamma_inj),
      ctypes.c_double(sign), _p(nrm), _p(uni), _p(px), _p(py), _p(pz), _p(psa))
    return px, py, pz, psa


def num_threads():
    return int(load().orc_num_threads())
