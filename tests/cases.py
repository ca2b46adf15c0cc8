"""Named configurations shared by the parity tests (small enough for the CPU oracle)."""
from mrlbm_2d_b200.config import (GEOM_EXPLICIT, INIT_NOISE, LABEL15_ALLNINE, NU_DIAMETER, WALL_FREESLIP,
                                  Config, case_small, cylinder_case, reference_case)


def _stats(c, **kw):
    base = dict(post_process=1, statsbegin=1, statsend=10 ** 9, iplot=7, init_mode=INIT_NOISE, seed=7,
                noise_amp=1e-2, num_threads=4)
    base.update(kw)
    return c.replace(**base)


def small_reference(**kw):
    # ncy=10: 80 x 50 lattice, centre (26, 25), r_c = 5 -- expressible by the unmodified reference
    return _stats(reference_case(ncy=10, L_front=2, L_back=5, L_top=2, L_bot=2, Re=100.0, uo=0.05), **kw)


CASES = {
    "reference_default_bcs": lambda: small_reference(),
    "reference_rest_start": lambda: small_reference(init_mode=0),
    "reference_walls": lambda: small_reference(y_periodic=0),
    "reference_walls_incomp": lambda: small_reference(y_periodic=0, incomp_bc=1, incomp_bulk=1),
    "closure_weak": lambda: small_reference(strong_mass_bc=0, weak_mass_bc=1),
    "closure_rhoeq": lambda: small_reference(strong_mass_bc=0, eq_mass_bc=1),
    "closure_unrotated": lambda: small_reference(rotated_coordinate=0),
    "no_velocity_interp": lambda: small_reference(vel_interp=0),
    "x_and_y_periodic": lambda: small_reference(x_periodic=1, y_periodic=1),
    "periodic_channel_no_cylinder": lambda: small_reference(channel_with_cylinder=0, nx=64, ny=40,
                                                            x_periodic=1, y_periodic=1, post_process=0),
    "freeslip_label15": lambda: _stats(cylinder_case(120, 48, 12, 30.0, 24.5, 100.0, 0.05), noise_amp=1e-2),
    "freeslip_xperiodic": lambda: _stats(cylinder_case(96, 40, 10, 40.0, 20.5, 80.0, 0.05), x_periodic=1,
                                         noise_amp=1e-2),
    "benchmark_small_400x100": lambda: case_small().replace(iplot=50, num_threads=8),
}
