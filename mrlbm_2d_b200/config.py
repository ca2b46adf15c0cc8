"""ctypes mirror of `mrlbm_config` (include/mrlbm.h) and the named cases used by tests/bench.

The reference reads its run configuration from the namelists of input.dat
(2d_mrlbm.f90:2222-2275).  `Config.reference_defaults()` holds the values of the shipped
input.dat (input.dat:1-45); `case_*` helpers build the cylinder cases of the benchmark
suite (explicit real-valued centre, free-slip walls, seeded noise).
"""
import ctypes

GEOM_REFERENCE, GEOM_EXPLICIT = 0, 1
WALL_REFERENCE, WALL_FREESLIP = 0, 1
LABEL15_REJECT, LABEL15_ALLNINE = 0, 1
NU_REFERENCE, NU_DIAMETER = 0, 1
INIT_REFERENCE, INIT_NOISE = 0, 1

_INT_FIELDS = [
    "nx", "ny", "channel_with_cylinder", "ncy", "L_front", "L_back", "L_top", "L_bot",
    "iplot", "max_iter", "isave", "irestart", "statsbegin", "statsend", "iplotstats",
    "num_threads", "lattice_type", "post_process", "x_periodic", "y_periodic",
    "channel_with_square", "incomp_bc", "incomp_bulk", "vel_interp", "mom_interp",
    "rotated_coordinate", "strong_mass_bc", "eq_mass_bc", "weak_mass_bc",
    "geometry_mode", "wall_mode", "label15_rule", "nu_length", "init_mode", "reserved",
]


class Config(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double) for n in ("x_c", "y_c", "r_c", "Re", "uo", "rho_infty", "noise_amp")]
                + [("seed", ctypes.c_uint64)]
                + [(n, ctypes.c_int32) for n in _INT_FIELDS])

    @classmethod
    def reference_defaults(cls):
        """The shipped input.dat (input.dat:1-45)."""
        c = cls()
        c.nx, c.ny, c.lattice_type = 320, 32, 9
        c.ncy, c.L_front, c.L_back, c.L_top, c.L_bot = 20, 10, 35, 10, 10
        c.Re = 100.0
        c.num_threads = 16
        c.uo, c.rho_infty = 0.1, 1.0
        c.iplot, c.max_iter, c.isave, c.irestart = 100, 900000000, 10000, 0
        c.statsbegin, c.statsend, c.iplotstats = 100001, 200001, 1000
        c.post_process, c.x_periodic, c.y_periodic = 1, 0, 1
        c.channel_with_cylinder, c.channel_with_square = 1, 0
        c.incomp_bc, c.incomp_bulk = 0, 0
        c.vel_interp, c.mom_interp, c.rotated_coordinate = 1, 1, 1
        c.strong_mass_bc, c.eq_mass_bc, c.weak_mass_bc = 1, 0, 0
        return c

    def copy(self):
        c = Config()
        ctypes.pointer(c)[0] = self
        return c

    def replace(self, **kw):
        c = self.copy()
        for k, v in kw.items():
            if not hasattr(c, k):
                raise AttributeError(k)
            setattr(c, k, v)
        return c

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def reference_case(ncy=20, L_front=3, L_back=16, L_top=2, L_bot=2, Re=100.0, uo=0.05, **kw):
    """A case the unmodified reference can express (centre/radius from ncy and L_*)."""
    c = Config.reference_defaults().replace(ncy=ncy, L_front=L_front, L_back=L_back, L_top=L_top,
                                            L_bot=L_bot, Re=Re, uo=uo, geometry_mode=GEOM_REFERENCE)
    c.nx = (L_front + 1 + L_back) * ncy
    c.ny = (L_top + 1 + L_bot) * ncy
    return c.replace(**kw) if kw else c


def cylinder_case(nx, ny, D, xc, yc, Re, U, seed=1234, noise=1e-4, **kw):
    """A benchmark-suite cylinder case: explicit centre, free-slip top/bottom, outlet and
    inlet edges, seeded-noise start, nu on the nominal diameter, label-15 closure on all
    nine links."""
    c = Config.reference_defaults().replace(
        nx=nx, ny=ny, x_c=float(xc), y_c=float(yc), r_c=float(D) / 2.0, Re=float(Re), uo=float(U),
        geometry_mode=GEOM_EXPLICIT, wall_mode=WALL_FREESLIP, label15_rule=LABEL15_ALLNINE,
        nu_length=NU_DIAMETER, init_mode=INIT_NOISE, seed=seed, noise_amp=noise,
        x_periodic=0, y_periodic=0, post_process=1, statsbegin=1, statsend=2**31 - 1,
        iplot=2**30, isave=2**30, max_iter=2**30, num_threads=0)
    return c.replace(**kw) if kw else c


# The benchmark suite's cylinder cases (seeded synthetic inputs; no external data).
def case_small():
    """400 x 100, D = 20 at (80.0, 50.5), Re = 100, U = 0.05 (nu = 0.01, tau = 0.53)."""
    return cylinder_case(400, 100, 20, 80.0, 50.5, 100.0, 0.05)


def case_mid():
    """2048 x 512, D = 80 at (320.0, 256.5), Re = 200, U = 0.04 (nu = 0.016)."""
    return cylinder_case(2048, 512, 80, 320.0, 256.5, 200.0, 0.04)


def case_adjoint():
    """512 x 128, D = 32 at (128.0, 64.5), Re = 100, U = 0.05."""
    return cylinder_case(512, 128, 32, 128.0, 64.5, 100.0, 0.05)


def case_quarter():
    """8192 x 2048, D = 128 at (1024.0, 1024.5), Re = 500, U = 0.04: a quarter of the large case
    (2.4 GB of FP32 populations), for profiler captures."""
    return cylinder_case(8192, 2048, 128, 1024.0, 1024.5, 500.0, 0.04)


def case_large():
    """16384 x 4096, D = 256 at (2048.0, 2048.5), Re = 1000, U = 0.04."""
    return cylinder_case(16384, 4096, 256, 2048.0, 2048.5, 1000.0, 0.04)


def sweep_cases(n=64, seed=4242, U=0.05):
    """A seeded sweep of independent cylinder cases: nx uniform in [256, 1024] in steps of 32,
    ny = nx / 4, D = ny / 5 at (nx / 5, ny / 2 + 0.5), Re uniform in [40, 200], U = 0.05."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        nx = int(rng.integers(256 // 32, 1024 // 32 + 1)) * 32
        ny = nx // 4
        D = ny / 5.0
        Re = float(rng.uniform(40.0, 200.0))
        out.append(cylinder_case(nx, ny, D, nx / 5.0, ny / 2.0 + 0.5, Re, U, seed=seed * 1000 + c))
    return out
