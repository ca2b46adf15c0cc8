"""FP32 deviation-form step against the FP64 step (same case, same seeded start).

Short horizons only (the long-horizon Cd / Cl_rms / St comparison is
`python -m mrlbm_2d_b200.precision_study`).  Tolerances: the FP32
form keeps only small quantities in FP32, so after 2000 steps of the 400 x 100 benchmark case
the velocity field agrees to 5e-5 U (max), density and populations to 1e-5 absolute
(observed 2e-6) and the per-step drag to 1e-5 relative."""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu


def _pair(mrlbm, cfg, steps):
    out = {}
    for prec in (64, 32):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.step(steps, macro=True)
        out[prec] = (s.macro(), s.forces(), s.get_state())
        assert s.status() == 0
        s.close()
    return out


def test_fp32_tracks_fp64_benchmark_small(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    r = _pair(mrlbm, cfg, 2000)
    m64, m32 = r[64][0], r[32][0]
    du = np.abs(m32["ux"] - m64["ux"]).max() / cfg.uo
    dv = np.abs(m32["uy"] - m64["uy"]).max() / cfg.uo
    drho = np.abs(m32["rho"] - m64["rho"]).max()
    assert du < 5e-5 and dv < 5e-5, (du, dv)
    assert drho < 1e-5, drho
    fd64, fd32 = r[64][1][1], r[32][1][1]
    assert np.abs(fd32 - fd64).max() / np.abs(fd64).max() < 1e-5
    # the populations round-trip through the deviation storage within FP32 resolution
    f64, f32 = r[64][2], r[32][2]
    assert np.abs(f32 - f64).max() < 1e-5


@pytest.mark.parametrize("name", ["reference_default_bcs", "reference_walls", "reference_walls_incomp",
                                  "x_and_y_periodic", "freeslip_label15", "periodic_channel_no_cylinder",
                                  "closure_weak", "closure_rhoeq", "closure_unrotated", "no_velocity_interp"])
def test_fp32_boundary_variants_track_fp64(mrlbm, name):
    cfg = CASES[name]()
    r = _pair(mrlbm, cfg, 200)
    m64, m32 = r[64][0], r[32][0]
    scale = max(cfg.uo, 1e-3)
    assert np.abs(m32["ux"] - m64["ux"]).max() / scale < 1e-4
    assert np.abs(m32["uy"] - m64["uy"]).max() / scale < 1e-4
    assert np.abs(m32["rho"] - m64["rho"]).max() < 1e-5
