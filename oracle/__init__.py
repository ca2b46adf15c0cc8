"""TEST INFRASTRUCTURE ONLY: ctypes wrapper over the CPU oracle (oracle/mrlbm_oracle.cpp).

The oracle restates 2d_mrlbm.f90 on the CPU.  It is imported by tests/, by
__graft_entry__.smoke() as the checker, and by bench.py's CPU-baseline arm; the product
(mrlbm_2d_b200) never imports it.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_size.restype = ctypes.c_longlong
        L.orc_size.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        L.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
        L.orc_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p, ctypes.c_longlong]
        L.orc_scalars.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_iter.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_forces.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4 + [ctypes.c_int]
        _lib = L
    return _lib


class Oracle:
    """One reference-equivalent CPU simulation.  `cfg` is an mrlbm_2d_b200.Config."""

    def __init__(self, cfg, threads=None):
        L = lib()
        if threads:
            L.orc_set_threads(int(threads))
        err = ctypes.create_string_buffer(512)
        self._h = L.orc_create(ctypes.byref(cfg), err, 512)
        if not self._h:
            raise ValueError("oracle setup failed: " + err.value.decode())
        s = self.scalars()
        self.nx, self.ny, self.nbct = int(s["nx"]), int(s["ny"]), int(s["nbct"])

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    __del__ = close

    def step(self, n=1):
        lib().orc_step(self._h, int(n))

    def get(self, name):
        kind = ctypes.c_int()
        n = lib().orc_size(self._h, name.encode(), ctypes.byref(kind))
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64 if kind.value == 0 else np.int32)
        rc = lib().orc_get(self._h, name.encode(), out.ctypes.data, n)
        assert rc == 0
        return out

    def field(self, name):
        """A field as an (nx, ny) or (nx, ny, 9) array indexed [i-1, j-1(, k)]."""
        a = self.get(name)
        if a.size == self.nx * self.ny * 9:
            return a.reshape(9, self.ny, self.nx).transpose(2, 1, 0)
        return a.reshape(self.ny, self.nx).T

    def set_state(self, f_fortran):
        a = np.ascontiguousarray(f_fortran, dtype=np.float64).ravel()
        assert lib().orc_set(self._h, b"f", a.ctypes.data, a.size) == 0

    def set_inlet_profile(self, u_in):
        if u_in is None:
            lib().orc_set(self._h, b"u_in", None, 0)
            return
        a = np.ascontiguousarray(u_in, dtype=np.float64)
        assert lib().orc_set(self._h, b"u_in", a.ctypes.data, a.size) == 0

    def set_iter(self, it):
        lib().orc_set_iter(self._h, int(it))

    def scalars(self):
        out = np.zeros(11)
        lib().orc_scalars(self._h, out.ctypes.data)
        keys = ["nx", "ny", "nbct", "iter", "r_cyl", "nu", "omega", "x_c", "y_c", "r_c", "rho_inf_mean"]
        return dict(zip(keys, out.tolist()))

    def surface(self):
        """(p_surface (n, nbct), p_smooth (n, nbct), probes (n, 12)) of the stats steps so far."""
        ps, pf, pr = self.get("p_surface"), self.get("p_surface_smooth"), self.get("probes")
        n = pr.size // 12
        nb = ps.size // n if n else 0
        return ps.reshape(n, nb), pf.reshape(n, nb), pr.reshape(n, 12)

    def forces(self):
        n = lib().orc_forces(self._h, None, None, None, None, 0)
        it = np.zeros(n, np.int32)
        fd, fl, rin = np.zeros(n), np.zeros(n), np.zeros(n)
        lib().orc_forces(self._h, it.ctypes.data, fd.ctypes.data, fl.ctypes.data, rin.ctypes.data, n)
        return it, fd, fl, rin


def set_threads(n):
    return lib().orc_set_threads(int(n))
