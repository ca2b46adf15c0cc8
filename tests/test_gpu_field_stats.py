"""Field statistics (time-mean and rms of u, v, p accumulated in FP64 inside the step) against
the oracle's per-step fields summed on the host in the same order: bit for bit in FP64."""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu


def _host_stats(o, steps, begin, end):
    su = sv = sp = suu = svv = spp = None
    n = 0
    for k in range(steps):
        o.step(1)
        it = 2 + k                       # fresh runs start at iteration 2 (restart_step = 1)
        if not (begin <= it <= end):
            continue
        ux, uy = o.field("ux"), o.field("uy")
        p = o.field("rho") * (1.0 / 3.0)
        if su is None:
            su, sv, sp = np.zeros_like(ux), np.zeros_like(ux), np.zeros_like(ux)
            suu, svv, spp = np.zeros_like(ux), np.zeros_like(ux), np.zeros_like(ux)
        su = su + ux
        sv = sv + uy
        sp = sp + p
        suu = suu + ux * ux
        svv = svv + uy * uy
        spp = spp + p * p
        n += 1
    out = {}
    for name, s, ss in (("u", su, suu), ("v", sv, svv), ("p", sp, spp)):
        mean = s / n
        var = ss / n - mean * mean
        out["mean_" + name] = mean
        out["rms_" + name] = np.sqrt(np.maximum(var, 0.0))
    return out, n


@pytest.mark.parametrize("name", ["freeslip_label15", "reference_default_bcs"])
def test_fp64_field_stats_bit_exact(mrlbm, oracle_mod, name):
    cfg = CASES[name]()
    s = mrlbm.Simulation(cfg)
    s.field_stats_window(5, 24)
    o = oracle_mod.Oracle(cfg)
    ref, n = _host_stats(o, 30, 5, 24)
    s.step(30)
    got = s.field_stats()
    assert got["n"] == n == 20
    for k, v in ref.items():
        assert np.array_equal(got[k], v), k
    s.close()


def test_fp32_field_stats_track_fp64(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    out = {}
    for prec in (64, 32):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.field_stats_window(101, 600)
        s.step(600)
        out[prec] = s.field_stats()
        s.close()
    assert out[32]["n"] == out[64]["n"] == 500
    for k in ("mean_u", "mean_v", "rms_u", "rms_v"):
        assert np.abs(out[32][k] - out[64][k]).max() / cfg.uo < 1e-4, k
    assert np.abs(out[32]["mean_p"] - out[64]["mean_p"]).max() < 1e-6


def test_field_stats_window_rules(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    s = mrlbm.Simulation(cfg)
    with pytest.raises(mrlbm.MrlbmError):
        s.field_stats()                   # no window yet
    with pytest.raises(mrlbm.MrlbmError):
        s.field_stats_window(10, 5)
    s.field_stats_window(100, 200)
    s.step(10)
    with pytest.raises(mrlbm.MrlbmError):
        s.field_stats()                   # nothing inside the window yet
    s.step(200)
    assert s.field_stats()["n"] == 101
    s.field_stats_window(1, 10 ** 9)      # a new window clears the sums
    s.step(3)
    assert s.field_stats()["n"] == 3
    s.close()


def test_autotune_keeps_field_sums_and_surface_records(mrlbm):
    """The autotuner's trial steps leave the field sums, their count and the surface-pressure
    records as they were: a tuned run equals an untuned one."""
    cfg = CASES["freeslip_label15"]()
    out = []
    for tune in (False, True):
        s = mrlbm.Simulation(cfg)
        s.field_stats_window(3, 40)
        s.surface_enable()
        s.step(10)
        if tune:
            s.autotune(trial_steps=3)
        s.step(20)
        fs = s.field_stats()
        it, ps, pf, pr = s.surface()
        out.append((fs, it, ps))
        s.close()
    (f0, i0, p0), (f1, i1, p1) = out
    assert f0["n"] == f1["n"] == 29
    for k in ("mean_u", "rms_v", "mean_p", "rms_p"):
        assert np.array_equal(f0[k], f1[k]), k
    assert np.array_equal(i0, i1) and np.array_equal(p0, p1)


def test_fp32_surface_pressure_tracks_fp64(mrlbm):
    """Wall pressure, its smoothing and the probes from an FP32 handle (deviation storage read
    back as w + g in FP64) against the FP64 handle, after 300 steps of the 400 x 100 case."""
    cfg = CASES["benchmark_small_400x100"]()
    out = {}
    for prec in (64, 32):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.surface_enable()
        s.step(300)
        out[prec] = s.surface()
        assert s.probe_nodes() == [(100, 51), (110, 51), (120, 51), (130, 51)]
        s.close()
    it64, ps64, pf64, pr64 = out[64]
    it32, ps32, pf32, pr32 = out[32]
    assert np.array_equal(it32, it64) and len(it64) == 300
    assert np.abs(ps32 - ps64).max() < 1e-6          # p ~ 1/3; deviations ~1e-4
    assert np.abs(pf32 - pf64).max() < 1e-6
    assert np.abs(pr32 - pr64).max() < 1e-6


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("tile", [0, 17, 22, 27])
def test_optional_outputs_leave_the_populations_unchanged(mrlbm, prec, tile):
    """With field statistics and macroscopic output the kernels run their full instantiation,
    without them the lean one; the populations must not depend on which ran."""
    cfg = CASES["benchmark_small_400x100"]()
    runs = []
    for extras in (False, True):
        s = mrlbm.Simulation(cfg, precision=prec)
        try:
            s.tile_config = tile
        except mrlbm.MrlbmError:
            s.close()
            pytest.skip("shape does not fit this precision")
        if extras:
            s.field_stats_window(1, 10 ** 6)
        for _ in range(5):
            s.step(4, macro=extras)
        runs.append(s.get_state())
        assert s.status() == 0
        s.close()
    assert np.array_equal(runs[0], runs[1])
