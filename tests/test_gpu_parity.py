"""FP64 GPU step vs the CPU oracle, through the C ABI.

The FP64 kernels evaluate every expression in the reference's order without contraction,
and the two per-step sums (net force over the wall nodes and sum(rho(1,:))) run in index
order like the reference's sum(), so populations, macroscopic fields, forces and the inlet
density sum are all compared for exact equality.
"""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu



def _assert_exact(a, b, what):
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if bad.any():
        idx = np.argwhere(bad)[:5]
        d = np.max(np.abs(a[bad] - b[bad]) / np.maximum(np.abs(b[bad]), 1e-300))
        raise AssertionError(f"{what}: {bad.sum()} of {a.size} differ (max rel {d:.3e}); first {idx.tolist()}")


def _run(mrlbm, oracle_mod, cfg, chunks, inlet=None):
    o = oracle_mod.Oracle(cfg)
    s = mrlbm.Simulation(cfg, precision=mrlbm.FP64)
    if inlet is not None:
        o.set_inlet_profile(inlet)
        s.set_inlet_profile(inlet)
    _assert_exact(s.get_state(), o.field("f"), "initial state")
    for n in chunks:
        o.step(n)
        s.step(n, macro=True)
        _assert_exact(s.get_state(), o.field("f"), f"populations after step {o.scalars()['iter']:.0f}")
        mac = s.macro()
        for name in ("rho", "ux", "uy"):
            _assert_exact(mac[name], o.field(name), f"{name} after step {o.scalars()['iter']:.0f}")
    it_o, fd_o, fl_o, rin_o = o.forces()
    it_g, fd_g, fl_g, rin_g = s.forces()
    assert np.array_equal(it_o, it_g)
    if cfg.channel_with_cylinder:
        assert np.array_equal(fd_g, fd_o) and np.array_equal(fl_g, fl_o), "force sums"
    assert np.array_equal(rin_g, rin_o), "inlet density sums"
    assert s.status() == 0
    s.close()
    o.close()


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_step_matches_oracle(mrlbm, oracle_mod, name):
    _run(mrlbm, oracle_mod, CASES[name](), [1, 9, 40])


def test_fp64_inlet_profile(mrlbm, oracle_mod):
    cfg = CASES["freeslip_label15"]()
    rng = np.random.default_rng(5)
    u_in = cfg.uo + 1e-3 * rng.standard_normal(cfg.ny)
    _run(mrlbm, oracle_mod, cfg, [1, 20], inlet=u_in)


def test_state_roundtrip_and_arbitrary_state(mrlbm, oracle_mod):
    """load_state/get_state are exact inverses (including the edge populations the
    reference never overwrites), and stepping from an arbitrary state matches."""
    for name in ("reference_walls", "freeslip_xperiodic", "x_and_y_periodic"):
        cfg = CASES[name]()
        s = mrlbm.Simulation(cfg)
        o = oracle_mod.Oracle(cfg)
        rng = np.random.default_rng(11)
        f = o.field("f") * (1.0 + 1e-3 * rng.standard_normal((s.nx, s.ny, 9)))
        s.load_state(f, iter=3)
        _assert_exact(s.get_state(), f, f"{name} roundtrip")
        o.set_state(np.ascontiguousarray(f.transpose(2, 1, 0)).ravel())
        o.set_iter(3)
        o.step(5)
        s.step(5)
        _assert_exact(s.get_state(), o.field("f"), f"{name} after 5 steps from a loaded state")
        assert s.iter == 8
        s.close()


def test_benchmark_mid_size_first_steps(mrlbm, oracle_mod):
    """The 2048 x 512 benchmark case itself, at full size, for a few steps."""
    from mrlbm_2d_b200.config import case_mid
    cfg = case_mid().replace(num_threads=0)
    _run(mrlbm, oracle_mod, cfg, [1, 2])


def test_forces_per_step_ring_drains_in_order(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    s = mrlbm.Simulation(cfg)
    n0 = s.launch_count()                      # the initial-state upload
    s.step(100)
    it, fd, fl, rin = s.forces()
    assert np.array_equal(it, np.arange(2, 102))
    assert np.all(np.isfinite(fd)) and np.all(np.isfinite(fl))
    s.step(5)
    it2, *_ = s.forces()
    assert np.array_equal(it2, np.arange(102, 107))
    # two launches per step (wall and edge nodes, then the bulk tiles); the last stats step's
    # record is summed by the next step's launch, or, when the history is read first, by one
    # small kernel per read
    assert s.launch_count() - n0 == 2 * 105 + 2
