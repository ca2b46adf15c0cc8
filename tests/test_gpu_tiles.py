"""Every bulk tile shape computes the same step (bit for bit), and the autotuner leaves the
simulation untouched."""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [64, 32])
def test_all_tile_shapes_bit_identical(mrlbm, prec):
    cfg = CASES["freeslip_label15"]()
    ref = None
    ran = []
    for c in range(mrlbm.N_TILE_CONFIGS):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.tile_config = c
        try:
            s.step(25)
        except mrlbm.MrlbmError as e:
            assert e.code == 4 and (10 <= c < 16 or c >= 27), (c, str(e))   # a TMA shape too large for this precision
            s.close()
            continue
        ran.append(c)
        assert s.status() == 0
        st = s.get_state()
        _, fd, fl, rin = s.forces()
        s.close()
        if ref is None:
            ref = (st, fd, fl, rin)
        else:
            assert np.array_equal(st, ref[0]), f"tile shape {c}"
            assert np.array_equal(fd, ref[1]) and np.array_equal(fl, ref[2]), f"tile shape {c}"
            assert np.array_equal(rin, ref[3]), f"tile shape {c}: inlet density sum"
    assert len([c for c in ran if 10 <= c < 16]) >= 3 and len([c for c in ran if c >= 27]) >= 2, ran


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("name", ["closure_weak", "closure_rhoeq", "closure_unrotated"])
def test_closure_variants_same_bits_in_every_launch_structure(mrlbm, prec, name):
    """A closure variant gives the same bits whether its wall blocks run inside the one-launch
    step (FP32 tile shapes) or in the auxiliary launch (vector, pipelined and TMA shapes, FP64)."""
    cfg = CASES[name]()
    ref = None
    for c in (0, 9, 7, 18, 22, 15, 27):
        s = mrlbm.Simulation(cfg, precision=prec)
        s.tile_config = c
        try:
            s.step(20)
        except mrlbm.MrlbmError as e:
            assert e.code == 4 and c >= 10 and c not in (18, 22), (c, str(e))
            s.close()
            continue
        assert s.status() == 0
        st = s.get_state()
        fd = s.forces()[1]
        s.close()
        if ref is None:
            ref = (st, fd)
        else:
            assert np.array_equal(st, ref[0]), f"{name}: tile shape {c}"
            assert np.array_equal(fd, ref[1]), f"{name}: tile shape {c}"


@pytest.mark.parametrize("prec", [64, 32])
def test_tma_shapes_many_steps(mrlbm, oracle_mod, prec):
    """The persistent tile counter keeps its running base across many launches: a TMA shape
    stepped 300 times in separate calls matches a one-tile-per-block shape."""
    cfg = CASES["reference_default_bcs"]()
    a = mrlbm.Simulation(cfg, precision=prec)
    b = mrlbm.Simulation(cfg, precision=prec)
    a.tile_config = 1
    b.tile_config = 10
    for _ in range(30):
        a.step(10)
        b.step(10)
    assert a.status() == 0 and b.status() == 0
    assert np.array_equal(a.get_state(), b.get_state())
    if prec == 64:
        o = oracle_mod.Oracle(cfg)
        o.step(300)
        assert np.array_equal(b.get_state(), o.field("f"))


def test_autotune_restores_state(mrlbm, oracle_mod):
    """Trials run on a saved copy of the state; stepping afterwards matches the oracle."""
    cfg = CASES["reference_default_bcs"]()
    s = mrlbm.Simulation(cfg)
    o = oracle_mod.Oracle(cfg)
    s.step(5)
    o.step(5)
    before = s.get_state()
    best, ms = s.autotune(trial_steps=3)
    assert 0 <= best < mrlbm.N_TILE_CONFIGS and ms > 0
    assert s.iter == 6
    assert np.array_equal(s.get_state(), before)
    s.step(5)
    o.step(5)
    assert np.array_equal(s.get_state(), o.field("f"))
    it, fd, fl, rin = s.forces()
    it_o, fd_o, fl_o, _ = o.forces()
    assert np.array_equal(it, it_o)
    assert np.array_equal(fd, fd_o)
