"""The benchmark suite's own cylinder cases, at full size, on the GPU.

FP64 against the CPU oracle, bit for bit (np.array_equal on populations, the per-step force
sums and the inlet density sums):
  * 400 x 100, D = 20 at (80.0, 50.5), Re = 100: 2000 steps, every step's drag and lift;
  * 2048 x 512, D = 80 at (320.0, 256.5), Re = 200: 20 steps;
  * 512 x 128, D = 32 at (128.0, 64.5), Re = 100 (the adjoint case): 50 steps;
  * three cases of the 64-case sweep (the smallest, the median and a 1024 x 256 one), stepped
    through the batch under all three schedules.
FP32 deviation form against the FP64 GPU step on the same cases (and on 16384 x 4096): the
mean drag coefficient within |dCd|/Cd <= 1e-3 and the velocity field within 1e-3 relative L2,
the accuracy bar the FP32 form is built to (the oracle's arithmetic is the FP64 step's, pinned
above).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _assert_exact(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if bad.any():
        d = np.max(np.abs(a[bad] - b[bad]) / np.maximum(np.abs(b[bad]), 1e-300))
        raise AssertionError(f"{what}: {bad.sum()} of {a.size} differ (max rel {d:.3e})")


def _config(name):
    from mrlbm_2d_b200 import config
    return {"small": config.case_small, "mid": config.case_mid, "adjoint": config.case_adjoint,
            "large": config.case_large}[name]()


def _against_oracle(mrlbm, oracle_mod, cfg, chunks):
    o = oracle_mod.Oracle(cfg)
    s = mrlbm.Simulation(cfg, precision=mrlbm.FP64)
    _assert_exact(s.get_state(), o.field("f"), "initial state")
    for n in chunks:
        o.step(n)
        s.step(n)
        _assert_exact(s.get_state(), o.field("f"), f"populations after step {s.iter}")
    it_o, fd_o, fl_o, rin_o = o.forces()
    it_g, fd_g, fl_g, rin_g = s.forces()
    assert np.array_equal(it_g, it_o) and len(it_g) == sum(chunks)
    _assert_exact(fd_g, fd_o, "drag per step")
    _assert_exact(fl_g, fl_o, "lift per step")
    _assert_exact(rin_g, rin_o, "inlet density sum per step")
    assert s.status() == 0
    s.close()
    o.close()


def test_small_case_2000_steps_every_force_record(mrlbm, oracle_mod):
    _against_oracle(mrlbm, oracle_mod, _config("small"), [1, 999, 1000])


def test_mid_case_20_steps(mrlbm, oracle_mod):
    _against_oracle(mrlbm, oracle_mod, _config("mid"), [1, 19])


def test_adjoint_case_50_steps(mrlbm, oracle_mod):
    _against_oracle(mrlbm, oracle_mod, _config("adjoint"), [1, 49])


def test_sweep_cases_through_the_batch(mrlbm, oracle_mod):
    """The batch (persistent schedule, then split graph steps, then per-case streams) against
    the oracle stepping each case alone."""
    from mrlbm_2d_b200.config import sweep_cases
    cfgs = sweep_cases(64)
    order = sorted(range(len(cfgs)), key=lambda i: cfgs[i].nx * cfgs[i].ny)
    pick = [order[0], order[len(order) // 2], next(i for i in order if cfgs[i].nx == 1024)]
    sel = [cfgs[i] for i in pick]
    assert (sel[0].nx, sel[2].nx, sel[2].ny) == (256, 1024, 256)
    b = mrlbm.Batch(sel, precision=mrlbm.FP64)
    b.set_schedule(18, mrlbm.BATCH_PERSISTENT, 6)
    b.step(12)
    b.set_schedule(17, mrlbm.BATCH_GRAPH, 4)
    b.step(8)
    b.set_schedule(7, mrlbm.BATCH_STREAMS, 5)
    b.step(10)
    assert b.status() == 0
    for c, cfg in enumerate(sel):
        o = oracle_mod.Oracle(cfg)
        o.step(30)
        h = b.cases[c]
        _assert_exact(h.get_state(), o.field("f"), f"sweep case {pick[c]} ({cfg.nx} x {cfg.ny})")
        it_o, fd_o, fl_o, rin_o = o.forces()
        it_g, fd_g, fl_g, rin_g = h.forces()
        assert np.array_equal(it_g, it_o)
        _assert_exact(fd_g, fd_o, "drag")
        _assert_exact(fl_g, fl_o, "lift")
        _assert_exact(rin_g, rin_o, "inlet density")
        o.close()
    b.close()


# FP32 against FP64: (case, steps).  The drag coefficient is averaged over the second half.
FP32_CASES = [("small", 6000), ("adjoint", 6000), ("mid", 4000), ("large", 300)]
CD_TOL = 1e-3           # |dCd| / Cd
VEL_TOL = 1e-3          # || u32 - u64 ||_2 / || u64 ||_2 over the final velocity field


@pytest.mark.parametrize("name,steps", FP32_CASES)
def test_fp32_tracks_fp64(mrlbm, name, steps):
    cfg = _config(name)
    out = {}
    for prec in (mrlbm.FP64, mrlbm.FP32):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.tile_config = 18
        s.step(steps - 1)
        s.step(1, macro=True)
        assert s.status() == 0
        _, fd, _, _ = s.forces()
        m = s.macro()
        out[prec] = (fd, m["ux"], m["uy"])
        s.close()
    fd64, ux64, uy64 = out[mrlbm.FP64]
    fd32, ux32, uy32 = out[mrlbm.FP32]
    half = len(fd64) // 2
    norm = 0.5 * cfg.rho_infty * cfg.uo ** 2 * (2.0 * cfg.r_c)
    cd64, cd32 = fd64[half:].mean() / norm, fd32[half:].mean() / norm
    assert abs(cd32 - cd64) <= CD_TOL * abs(cd64), (cd32, cd64)
    dv = np.sqrt(((ux32 - ux64) ** 2 + (uy32 - uy64) ** 2).sum())
    v = np.sqrt((ux64 ** 2 + uy64 ** 2).sum())
    assert dv <= VEL_TOL * v, dv / v
