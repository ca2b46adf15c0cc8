"""ctypes binding of include/mrlbm.h and a thin Simulation object over it.

The reference's "API" is its main program driven by input.dat (2d_mrlbm.f90:77-555).
`Simulation` mirrors that run: it is created from the same configuration, advances with
`step` (one call per main-loop iteration or a batch of them), and hands back the outputs the
reference writes: macroscopic fields (the PLOT3D function file, 2d_mrlbm.f90:2163-2184), the
post-streaming populations (restart.dat, 2d_mrlbm.f90:2186-2202) and the force history
(data_mean/forces_time.dat, 2d_mrlbm.f90:492-494).  Errors raise `MrlbmError` with the
library's status code, as the reference stops on bad input (2d_mrlbm.f90:2235-2238).

There is no CPU fallback: without the compiled library or a CUDA device every call raises.
"""
import ctypes
import os

import numpy as np

from .config import Config

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmrlbm.so")

FP64, FP32 = 64, 32
N_TILE_CONFIGS = 31   # MRLBM_N_TILE_CONFIGS: 0..9 tiles, 10..15 TMA, 16..21 128-bit vector, 22..26 pipelined, 27..30 TMA + tensor stores
STEP_MACRO = 1

EXPORTED = [
    "mrlbm_config_sizeof", "mrlbm_config_defaults", "mrlbm_config_from_namelist", "mrlbm_config_resolve_geometry",
    "mrlbm_create", "mrlbm_destroy", "mrlbm_last_error", "mrlbm_status", "mrlbm_set_stream",
    "mrlbm_get_geometry_info", "mrlbm_get_boundary_nodes", "mrlbm_get_node_classes",
    "mrlbm_load_state", "mrlbm_get_state", "mrlbm_set_inlet_profile", "mrlbm_step",
    "mrlbm_get_iter", "mrlbm_get_macro", "mrlbm_get_forces", "mrlbm_get_launch_count",
    "mrlbm_force_statistics", "mrlbm_cp_statistics", "mrlbm_step_noalloc",
    "mrlbm_set_tile_config", "mrlbm_get_tile_config", "mrlbm_autotune",
    "mrlbm_field_stats_window", "mrlbm_field_stats_get",
    "mrlbm_batch_create", "mrlbm_batch_destroy", "mrlbm_batch_case", "mrlbm_batch_step",
    "mrlbm_batch_set_schedule", "mrlbm_batch_get_schedule", "mrlbm_batch_autotune", "mrlbm_batch_status",
    "mrlbm_batch_last_error", "mrlbm_batch_launch_count", "mrlbm_batch_get_stream",
    "mrlbm_batch_set_wait_limit",
    "mrlbm_set_body_force", "mrlbm_adjoint_drag",
    "mrlbm_surface_enable", "mrlbm_get_probe_nodes", "mrlbm_get_surface",
    "mrlbm_create_slab", "mrlbm_halo_size", "mrlbm_halo_pack", "mrlbm_halo_unpack", "mrlbm_slabs_step",
    "mrlbm_step_faces", "mrlbm_halo_pack_next", "mrlbm_halo_unpack_next",
]
BATCH_PERSISTENT, BATCH_GRAPH, BATCH_STREAMS = 0, 1, 2


class MrlbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mrlbm error {code}: {msg}")
        self.code = code


class GeometryInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nbct", ctypes.c_int32),
                ("n_label15", ctypes.c_int32), ("x_c", ctypes.c_double), ("y_c", ctypes.c_double),
                ("r_c", ctypes.c_double), ("r_cyl", ctypes.c_double), ("nu", ctypes.c_double),
                ("omega", ctypes.c_double), ("pitch", ctypes.c_int32), ("off", ctypes.c_int32),
                ("plane", ctypes.c_int64), ("state_bytes", ctypes.c_int64)]


_lib = None


def load_library(path=None):
    """Load libmrlbm.so (built by `python -m mrlbm_2d_b200.build`).  Raises if missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise MrlbmError(-3, f"{p} is not built; run `python -m mrlbm_2d_b200.build`")
    L = ctypes.CDLL(p)
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_double
    sig = {
        "mrlbm_config_defaults": [vp],
        "mrlbm_config_from_namelist": [ctypes.c_char_p, vp],
        "mrlbm_config_resolve_geometry": [vp],
        "mrlbm_create": [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)],
        "mrlbm_destroy": [vp],
        "mrlbm_last_error": [vp, ctypes.c_char_p, ctypes.c_size_t],
        "mrlbm_status": [vp],
        "mrlbm_set_stream": [vp, vp],
        "mrlbm_get_geometry_info": [vp, vp],
        "mrlbm_get_boundary_nodes": [vp] * 7,
        "mrlbm_get_node_classes": [vp] * 4,
        "mrlbm_load_state": [vp, vp, i32],
        "mrlbm_get_state": [vp, vp],
        "mrlbm_set_inlet_profile": [vp, vp],
        "mrlbm_step": [vp, i32, i32],
        "mrlbm_get_iter": [vp, vp],
        "mrlbm_get_macro": [vp] * 7,
        "mrlbm_get_forces": [vp, vp, vp, vp, vp, i32, vp],
        "mrlbm_get_launch_count": [vp, vp],
        "mrlbm_force_statistics": [vp, vp, i32, dbl, dbl, dbl, vp, vp, vp, vp, vp, vp],
        "mrlbm_cp_statistics": [vp, i32, i32, i32, i32, i32, dbl, dbl, vp],
        "mrlbm_step_noalloc": [vp, vp, vp, i32, vp, vp, vp],
        "mrlbm_set_tile_config": [vp, i32],
        "mrlbm_get_tile_config": [vp, vp],
        "mrlbm_autotune": [vp, i32, vp, vp],
        "mrlbm_field_stats_window": [vp, i32, i32],
        "mrlbm_field_stats_get": [vp] * 8,
        "mrlbm_batch_create": [vp, i32, ctypes.c_int, ctypes.c_int, vp],
        "mrlbm_batch_destroy": [vp],
        "mrlbm_batch_case": [vp, i32, vp],
        "mrlbm_batch_step": [vp, i32, i32],
        "mrlbm_batch_set_schedule": [vp, i32, i32, i32],
        "mrlbm_batch_get_schedule": [vp, vp, vp, vp],
        "mrlbm_batch_autotune": [vp, i32, vp],
        "mrlbm_batch_status": [vp],
        "mrlbm_batch_last_error": [vp, ctypes.c_char_p, ctypes.c_size_t],
        "mrlbm_batch_launch_count": [vp, vp],
        "mrlbm_batch_get_stream": [vp, vp],
        "mrlbm_batch_set_wait_limit": [vp, ctypes.c_int64],
        "mrlbm_set_body_force": [vp, vp],
        "mrlbm_adjoint_drag": [vp, i32, i32, i32, vp, vp, vp],
        "mrlbm_surface_enable": [vp, i32],
        "mrlbm_get_probe_nodes": [vp, vp, vp],
        "mrlbm_get_surface": [vp, vp, vp, vp, vp, i32, vp],
        "mrlbm_create_slab": [vp, ctypes.c_int, ctypes.c_int, i32, i32, vp],
        "mrlbm_halo_size": [vp, vp, vp],
        "mrlbm_halo_pack": [vp, i32, vp],
        "mrlbm_halo_unpack": [vp, i32, vp],
        "mrlbm_step_faces": [vp],
        "mrlbm_halo_pack_next": [vp, i32, vp],
        "mrlbm_halo_unpack_next": [vp, i32, vp],
        "mrlbm_slabs_step": [vp, i32, i32],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    if path is None:
        _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def force_statistics(f_drag, f_lift, r_cy, uo, rho_infty):
    """St, Cd, Cl_rms and the cycle window of a force history (2d_statistics.f90:90-131)."""
    L = load_library()
    fd = np.ascontiguousarray(f_drag, dtype=np.float64)
    fl = np.ascontiguousarray(f_lift, dtype=np.float64)
    st, cd, cl = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cs, per, nc = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    rc = L.mrlbm_force_statistics(_ptr(fd), _ptr(fl), fd.size, float(r_cy), float(uo), float(rho_infty),
                                  ctypes.byref(st), ctypes.byref(cd), ctypes.byref(cl), ctypes.byref(cs),
                                  ctypes.byref(per), ctypes.byref(nc))
    if rc != 0:
        raise MrlbmError(rc, "could not detect two lift peaks" if rc == 5 else "bad arguments")
    return {"St": st.value, "Cd": cd.value, "Cl_rms": cl.value, "cycle_start": cs.value, "period": per.value,
            "n_cycle": nc.value}


def cp_statistics(p_surface, cycle_start, period, n_cycle, rho_infty, uo):
    """Cycle-averaged Cp per wall node (2d_statistics.f90:114-122)."""
    L = load_library()
    ps = np.ascontiguousarray(p_surface, dtype=np.float64)
    nstep, nbct = ps.shape
    cp = np.empty(nbct)
    rc = L.mrlbm_cp_statistics(_ptr(ps), nstep, nbct, int(cycle_start), int(period), int(n_cycle),
                               float(rho_infty), float(uo), _ptr(cp))
    if rc != 0:
        raise MrlbmError(rc, "bad arguments")
    return cp


def rho_inlet_running_mean(iters, rho_inlet_sum, ny, statsbegin):
    """rho_inf_mean as the reference updates it each stats step (2d_mrlbm.f90:357-360)."""
    m = 0.0
    out = np.empty(len(iters))
    for n, (it, s) in enumerate(zip(iters, rho_inlet_sum)):
        c = float(np.float32(it - statsbegin))          # real(iter - statsbegin): default REAL
        rho_infty = s / ny
        m = ((c * m) + rho_infty) / (c + 1.0)
        out[n] = m
    return out


def config_from_namelist(path):
    """Read input.dat the way read_input_file does (2d_mrlbm.f90:2222-2275)."""
    L = load_library()
    c = Config()
    L.mrlbm_config_defaults(ctypes.byref(c))
    rc = L.mrlbm_config_from_namelist(os.fsencode(path), ctypes.byref(c))
    if rc != 0:
        buf = ctypes.create_string_buffer(512)
        L.mrlbm_last_error(None, buf, 512)
        raise MrlbmError(rc, buf.value.decode())
    return c


class Simulation:
    """One cylinder-flow case resident on one GPU."""

    def __init__(self, cfg, precision=FP64, device=0, slab=None):
        """slab=(gx0, gx1): only global columns gx0..gx1 of the domain (mrlbm_create_slab)."""
        self._L = load_library()
        self._h = ctypes.c_void_p()
        self.slab = slab
        if slab is None:
            rc = self._L.mrlbm_create(ctypes.byref(cfg), int(precision), int(device), ctypes.byref(self._h))
        else:
            rc = self._L.mrlbm_create_slab(ctypes.byref(cfg), int(precision), int(device), int(slab[0]),
                                           int(slab[1]), ctypes.byref(self._h))
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self._L.mrlbm_last_error(None, buf, 1024)
            raise MrlbmError(rc, buf.value.decode())
        self.precision = precision
        info = GeometryInfo()
        self._L.mrlbm_get_geometry_info(self._h, ctypes.byref(info))
        self.info = info
        self.nx, self.ny, self.nbct = info.nx, info.ny, info.nbct

    # -- lifetime --------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.mrlbm_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self._L.mrlbm_last_error(self._h, buf, 1024)
            raise MrlbmError(rc, buf.value.decode())

    @property
    def handle(self):
        return self._h

    # -- stepping --------------------------------------------------------------------
    def step(self, n=1, macro=False):
        self._check(self._L.mrlbm_step(self._h, int(n), STEP_MACRO if macro else 0))

    def autotune(self, trial_steps=20):
        """Pick the fastest bulk tile shape for this case (state and history are restored)."""
        best, ms = ctypes.c_int32(), ctypes.c_double()
        self._check(self._L.mrlbm_autotune(self._h, int(trial_steps), ctypes.byref(best), ctypes.byref(ms)))
        return best.value, ms.value

    @property
    def tile_config(self):
        c = ctypes.c_int32()
        self._check(self._L.mrlbm_get_tile_config(self._h, ctypes.byref(c)))
        return c.value

    @tile_config.setter
    def tile_config(self, cfg):
        self._check(self._L.mrlbm_set_tile_config(self._h, int(cfg)))

    def set_stream(self, stream_ptr):
        self._check(self._L.mrlbm_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)))

    def status(self):
        return self._L.mrlbm_status(self._h)

    @property
    def iter(self):
        it = ctypes.c_int32()
        self._check(self._L.mrlbm_get_iter(self._h, ctypes.byref(it)))
        return it.value

    def launch_count(self):
        n = ctypes.c_int64()
        self._check(self._L.mrlbm_get_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def step_noalloc(self, d_state_ptr, nsteps, d_f0_ptr=None, stream_ptr=None):
        """Step a host-only handle in caller-owned device memory (see mrlbm_step_noalloc).
        Returns the (n, 4) records (iter, F_drag_net, F_lift_net, sum(rho(1,:)))."""
        rec = np.empty((max(int(nsteps), 1), 4))
        n = ctypes.c_int32()
        self._check(self._L.mrlbm_step_noalloc(self._h, ctypes.c_void_p(d_state_ptr),
                                               ctypes.c_void_p(d_f0_ptr) if d_f0_ptr else None, int(nsteps),
                                               _ptr(rec), ctypes.byref(n),
                                               ctypes.c_void_p(stream_ptr) if stream_ptr else None))
        return rec[:n.value].copy()

    # -- state and outputs -----------------------------------------------------------
    def get_state(self, out=None):
        """Post-streaming populations f as an (nx, ny, 9) array, f[i-1, j-1, k].  With `out` (a
        flat float64 array of nx*ny*9, e.g. a pinned buffer) the reference's Fortran-order f
        is written there and `out` is returned as is."""
        f = np.empty(self.nx * self.ny * 9) if out is None else out
        assert f.dtype == np.float64 and f.size == self.nx * self.ny * 9 and f.flags.c_contiguous
        self._check(self._L.mrlbm_get_state(self._h, _ptr(f)))
        return f.reshape(9, self.ny, self.nx).transpose(2, 1, 0) if out is None else out

    def load_state(self, f, iter=0):
        """Load populations: an (nx, ny, 9) array f[i-1, j-1, k], or a flat float64 array in the
        reference's Fortran order f(i, j, k) (passed to the device as is)."""
        f = np.asarray(f)
        if f.ndim == 1 and f.dtype == np.float64 and f.flags.c_contiguous and f.size == self.nx * self.ny * 9:
            flat = f
        else:
            a = np.asfortranarray(np.asarray(f, dtype=np.float64).reshape(self.nx, self.ny, 9))
            flat = np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()
        self._check(self._L.mrlbm_load_state(self._h, _ptr(flat), int(iter)))

    def set_inlet_profile(self, u_in):
        if u_in is None:
            self._check(self._L.mrlbm_set_inlet_profile(self._h, None))
            return
        a = np.ascontiguousarray(u_in, dtype=np.float64)
        assert a.size == self.ny
        self._check(self._L.mrlbm_set_inlet_profile(self._h, _ptr(a)))

    def macro(self, out=None):
        """dict of (nx, ny) arrays rho, ux, uy, mxx, myy, mxy of the last MACRO step.  With
        `out` = [rho, ux, uy] flat float64 buffers (e.g. pinned), only those three are read back."""
        N = self.nx * self.ny
        if out is not None:
            self._check(self._L.mrlbm_get_macro(self._h, *[_ptr(o) for o in out], None, None, None))
            return out
        outs = [np.empty(N) for _ in range(6)]
        self._check(self._L.mrlbm_get_macro(self._h, *[_ptr(o) for o in outs]))
        names = ["rho", "ux", "uy", "mxx", "myy", "mxy"]
        return {n: o.reshape(self.ny, self.nx).T for n, o in zip(names, outs)}

    def surface_enable(self, on=True):
        """Record wall pressure, its smoothing and the probes on every statistics step."""
        self._check(self._L.mrlbm_surface_enable(self._h, 1 if on else 0))

    def probe_nodes(self):
        pi, pj = (ctypes.c_int32 * 4)(), (ctypes.c_int32 * 4)()
        self._check(self._L.mrlbm_get_probe_nodes(self._h, pi, pj))
        return list(zip(pi, pj))

    def surface(self, cap=1 << 16):
        """Drain: (iter, p_surface (n, nbct), p_smooth (n, nbct), probes (n, 12) = p1..4, ux1..4, uy1..4)."""
        nb = self.nbct
        it = np.empty(cap, np.int32)
        ps, pf, pr = np.empty((cap, nb)), np.empty((cap, nb)), np.empty((cap, 12))
        n = ctypes.c_int32()
        self._check(self._L.mrlbm_get_surface(self._h, _ptr(it), _ptr(ps), _ptr(pf), _ptr(pr), cap, ctypes.byref(n)))
        m = n.value
        return it[:m].copy(), ps[:m].copy(), pf[:m].copy(), pr[:m].copy()

    def halo_size(self):
        """(values per halo face, bytes per value)."""
        n, e = ctypes.c_int64(), ctypes.c_int32()
        self._check(self._L.mrlbm_halo_size(self._h, ctypes.byref(n), ctypes.byref(e)))
        return n.value, e.value

    def halo_pack(self, side, dst_ptr):
        """Copy the outgoing populations of face `side` (0 left, 1 right) to device memory dst_ptr."""
        self._check(self._L.mrlbm_halo_pack(self._h, int(side), ctypes.c_void_p(int(dst_ptr))))

    def halo_unpack(self, side, src_ptr):
        """Copy a neighbour's packed face from device memory src_ptr into this slab's ghost column."""
        self._check(self._L.mrlbm_halo_unpack(self._h, int(side), ctypes.c_void_p(int(src_ptr))))

    def step_faces(self):
        """Compute the halo-face columns of the next step into the next time level (ahead of
        step(1), which writes the same bits), so the faces can travel while the step runs."""
        self._check(self._L.mrlbm_step_faces(self._h))

    def halo_pack_next(self, side, dst_ptr):
        """halo_pack from the time level the next step writes (after step_faces)."""
        self._check(self._L.mrlbm_halo_pack_next(self._h, int(side), ctypes.c_void_p(int(dst_ptr))))

    def halo_unpack_next(self, side, src_ptr):
        """halo_unpack into the ghost column of the time level the next step writes."""
        self._check(self._L.mrlbm_halo_unpack_next(self._h, int(side), ctypes.c_void_p(int(src_ptr))))

    def set_body_force(self, g):
        """Body force g of shape (2, nx, ny) (x and y components, [c, i-1, j-1]); None removes it."""
        if g is None:
            self._check(self._L.mrlbm_set_body_force(self._h, None))
            return
        g = np.asarray(g, dtype=np.float64)
        assert g.shape == (2, self.nx, self.ny)
        flat = np.ascontiguousarray(g.transpose(0, 2, 1)).ravel()     # Fortran node order per component
        self._check(self._L.mrlbm_set_body_force(self._h, _ptr(flat)))

    def adjoint_drag(self, nsteps, window, checkpoint_every=100, grads=True):
        """J = mean drag over the last `window` of the next `nsteps` steps (state not advanced)
        and, with grads, dJ/d(body force) as (2, nx, ny) and dJ/d(u_in) as (ny,)."""
        J = ctypes.c_double()
        gb = np.zeros(2 * self.nx * self.ny) if grads else None
        gu = np.zeros(self.ny) if grads else None
        self._check(self._L.mrlbm_adjoint_drag(self._h, int(nsteps), int(window), int(checkpoint_every),
                                               ctypes.byref(J), _ptr(gb) if grads else None,
                                               _ptr(gu) if grads else None))
        if not grads:
            return J.value
        return J.value, gb.reshape(2, self.ny, self.nx).transpose(0, 2, 1).copy(), gu

    def field_stats_window(self, begin_iter, end_iter):
        """Accumulate FP64 mean/rms sums of u, v, p over steps begin_iter..end_iter (clears them)."""
        self._check(self._L.mrlbm_field_stats_window(self._h, int(begin_iter), int(end_iter)))

    def field_stats(self):
        """dict of (nx, ny) arrays mean_u, mean_v, mean_p, rms_u, rms_v, rms_p, plus n (steps)."""
        N = self.nx * self.ny
        outs = [np.empty(N) for _ in range(6)]
        n = ctypes.c_int64()
        self._check(self._L.mrlbm_field_stats_get(self._h, *[_ptr(o) for o in outs], ctypes.byref(n)))
        names = ["mean_u", "mean_v", "mean_p", "rms_u", "rms_v", "rms_p"]
        d = {k: o.reshape(self.ny, self.nx).T for k, o in zip(names, outs)}
        d["n"] = n.value
        return d

    def forces(self, cap=1 << 22):
        """Drain the force history: (iter, F_drag_net, F_lift_net, sum(rho(1,:)))."""
        it = np.empty(cap, np.int32)
        fd, fl, rin = np.empty(cap), np.empty(cap), np.empty(cap)
        n = ctypes.c_int32()
        self._check(self._L.mrlbm_get_forces(self._h, _ptr(it), _ptr(fd), _ptr(fl), _ptr(rin), cap,
                                             ctypes.byref(n)))
        m = n.value
        return it[:m].copy(), fd[:m].copy(), fl[:m].copy(), rin[:m].copy()

    # -- geometry --------------------------------------------------------------------
    def boundary_nodes(self):
        nb = self.nbct
        bi, bj, lab = (np.empty(nb, np.int32) for _ in range(3))
        delta = np.empty(nb)
        ref = np.empty(8 * nb)
        sten = np.empty(24 * nb, np.int32)
        self._check(self._L.mrlbm_get_boundary_nodes(self._h, _ptr(bi), _ptr(bj), _ptr(lab), _ptr(delta),
                                                     _ptr(ref), _ptr(sten)))
        return {"bou_i": bi, "bou_j": bj, "label_bc": lab, "delta_uk": delta,
                "ref_xy": ref.reshape(nb, 8), "stencil": sten.reshape(nb, 24)}

    def node_classes(self):
        N = self.nx * self.ny
        a, b, c = (np.empty(N, np.int32) for _ in range(3))
        self._check(self._L.mrlbm_get_node_classes(self._h, _ptr(a), _ptr(b), _ptr(c)))
        return {k: v.reshape(self.ny, self.nx).T for k, v in zip(["isfluid", "issolid", "isbound"], (a, b, c))}


class _BorrowedSimulation(Simulation):
    """A case owned by a Batch: the single-case calls work on it; closing does nothing."""

    def __init__(self, lib, h, precision):
        self._L = lib
        self._h = h
        self.precision = precision
        info = GeometryInfo()
        self._L.mrlbm_get_geometry_info(self._h, ctypes.byref(info))
        self.info = info
        self.nx, self.ny, self.nbct = info.nx, info.ny, info.nbct

    def close(self):
        self._h = ctypes.c_void_p()

    def step(self, n=1, macro=False):
        raise MrlbmError(1, "a batch case steps only through Batch.step")


class Batch:
    """Many independent cases of one precision advanced together by one kernel per step (or
    one persistent launch per steps_per_launch steps); see mrlbm_batch_* in include/mrlbm.h."""

    def __init__(self, cfgs, precision=FP32, device=0):
        self._L = load_library()
        arr = (Config * len(cfgs))(*cfgs)
        self._b = ctypes.c_void_p()
        rc = self._L.mrlbm_batch_create(arr, len(cfgs), int(precision), int(device), ctypes.byref(self._b))
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self._L.mrlbm_batch_last_error(None, buf, 1024)
            raise MrlbmError(rc, buf.value.decode())
        self.precision = precision
        self.cases = []
        for c in range(len(cfgs)):
            h = ctypes.c_void_p()
            self._check(self._L.mrlbm_batch_case(self._b, c, ctypes.byref(h)))
            self.cases.append(_BorrowedSimulation(self._L, h, precision))

    def _check(self, rc):
        if rc != 0:
            buf = ctypes.create_string_buffer(1024)
            self._L.mrlbm_batch_last_error(self._b, buf, 1024)
            raise MrlbmError(rc, buf.value.decode())

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            for c in self.cases:
                c.close()
            self._L.mrlbm_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n=1, macro=False):
        self._check(self._L.mrlbm_batch_step(self._b, int(n), STEP_MACRO if macro else 0))

    def set_schedule(self, tile_cfg, schedule, steps_per_launch):
        self._check(self._L.mrlbm_batch_set_schedule(self._b, int(tile_cfg), int(schedule), int(steps_per_launch)))

    @property
    def schedule(self):
        t, s, n = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self._L.mrlbm_batch_get_schedule(self._b, ctypes.byref(t), ctypes.byref(s), ctypes.byref(n)))
        return t.value, s.value, n.value

    def autotune(self, trial_steps=50):
        ms = ctypes.c_double()
        self._check(self._L.mrlbm_batch_autotune(self._b, int(trial_steps), ctypes.byref(ms)))
        return self.schedule, ms.value

    def status(self):
        return self._L.mrlbm_batch_status(self._b)

    def set_wait_limit(self, polls):
        """Grid-barrier polls (about 0.1 us each) before a block of the persistent schedule
        gives up with MRLBM_EDEVICE_TIMEOUT; 0 restores the default."""
        self._check(self._L.mrlbm_batch_set_wait_limit(self._b, int(polls)))

    def launch_count(self):
        n = ctypes.c_int64()
        self._check(self._L.mrlbm_batch_launch_count(self._b, ctypes.byref(n)))
        return n.value

    @property
    def stream(self):
        """The batch's CUDA stream handle (an int), e.g. for torch.cuda.ExternalStream."""
        p = ctypes.c_void_p()
        self._check(self._L.mrlbm_batch_get_stream(self._b, ctypes.byref(p)))
        return p.value or 0


def slabs_step(sims, nsteps):
    """Advance adjacent slab simulations (left to right) with their halo exchange."""
    if not sims:
        return
    L = sims[0]._L
    arr = (ctypes.c_void_p * len(sims))(*[s._h.value for s in sims])
    rc = L.mrlbm_slabs_step(arr, len(sims), int(nsteps))
    if rc != 0:
        for s in sims:
            buf = ctypes.create_string_buffer(1024)
            L.mrlbm_last_error(s._h, buf, 1024)
            if buf.value:
                raise MrlbmError(rc, buf.value.decode())
        raise MrlbmError(rc, "mrlbm_slabs_step failed")
