"""The library's 2d_statistics port against the reference's statistics program executed on
synthetic histories (tests/golden/stats_*.npz, made by tests/golden/make_golden.py --stats)."""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "stats_*.npz")))


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(c) for c in CASES])
def test_force_and_cp_statistics_match_reference(mrlbm, path):
    d = np.load(path)
    r = mrlbm.force_statistics(d["f_drag"], d["f_lift"], float(d["r_cy"]), float(d["uo"]), float(d["rho_infty"]))
    assert r["St"] == float(d["St"])
    assert r["Cd"] == float(d["Cd"])
    assert r["Cl_rms"] == float(d["Cl_rms"])
    # the reference writes Cd(i), Cl(i) over the window; its first column is (i - start)/period
    assert len(d["cd_time"]) == r["n_cycle"] * r["period"] + 1
    cp = mrlbm.cp_statistics(d["p_surface"], r["cycle_start"], r["period"], r["n_cycle"], float(d["rho_infty"]),
                             float(d["uo"]))
    theta = d["theta"]
    sel = theta <= np.pi
    ref = d["cp"]                                       # (|theta*180/pi - 180|, Cp) for theta <= pi
    assert np.array_equal(ref[:, 1], cp[sel])
    assert np.allclose(ref[:, 0], np.abs(theta[sel] * 180.0 / np.pi - 180.0), rtol=0, atol=1e-12)
    cpf = mrlbm.cp_statistics(d["p_surface_smooth"], r["cycle_start"], r["period"], r["n_cycle"],
                              float(d["rho_infty"]), float(d["uo"]))
    assert np.array_equal(d["cp_fit"][:, 1], cpf[sel])


def test_no_two_peaks_is_an_error(mrlbm):
    with pytest.raises(mrlbm.MrlbmError):
        mrlbm.force_statistics(np.ones(50), np.linspace(0, 1, 50), 10.0, 0.05, 1.0)


def test_spectral_strouhal_recovers_a_seeded_shedding_period():
    """The precision study's spectral St finds the period of a noisy synthetic lift to 1e-4."""
    from mrlbm_2d_b200.precision_study import spectral_strouhal
    rng = np.random.default_rng(7)
    t = np.arange(30000)
    for period in (1234.5, 2424.0, 317.0):
        fl = 0.2 * np.sin(2 * np.pi * t / period + 0.3) + 2e-3 * rng.standard_normal(t.size)
        st = spectral_strouhal(fl, 20.0, 0.05)
        assert abs(st - 20.0 / (period * 0.05)) < 1e-4 * max(1.0, st)
