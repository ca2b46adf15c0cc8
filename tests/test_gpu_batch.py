"""Batched cases: one kernel advancing several independent cases (persistent cooperative
launches, or CUDA-graph replays of split steps: an auxiliary launch and a bulk launch per step,
with vector or one-tile-per-block bulk shapes), or each case's own step launches on per-case
streams captured into one replayed graph, gives every case exactly the bits it gets when
stepped alone."""
import numpy as np
import pytest

from cases import CASES
from mrlbm_2d_b200.config import cylinder_case

pytestmark = pytest.mark.gpu

NAMES = ["freeslip_label15", "reference_default_bcs", "x_and_y_periodic", "reference_walls", "freeslip_xperiodic"]


def _cfgs():
    return [CASES[n]() for n in NAMES] + [cylinder_case(256, 64, 12.8, 51.2, 32.5, 150.0, 0.05)]


def _alone(mrlbm, cfg, prec, steps, macro=False, fields=None):
    s = mrlbm.Simulation(cfg, precision=prec)
    s.tile_config = 18
    if fields:
        s.field_stats_window(*fields)
    s.step(steps, macro=macro)
    out = dict(f=s.get_state(), forces=s.forces(), status=s.status())
    if macro:
        out["macro"] = s.macro()
    if fields:
        out["fields"] = s.field_stats()
    s.close()
    return out


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("tile,sched,spl", [(18, 0, 7), (16, 1, 5), (21, 0, 1), (17, 1, 13), (20, 0, 23),
                                            (9, 1, 5), (6, 1, 23), (0, 1, 1), (3, 1, 7),
                                            (9, 2, 5), (7, 2, 8), (0, 2, 23), (6, 2, 1)])
def test_batch_matches_single_cases(mrlbm, prec, tile, sched, spl):
    cfgs = _cfgs()
    b = mrlbm.Batch(cfgs, precision=prec)
    b.set_schedule(tile, sched, spl)
    b.step(10)
    b.step(13)                                   # calls that do not divide into launches
    assert b.status() == 0
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, prec, 23)
        assert np.array_equal(c.get_state(), ref["f"])
        it, fd, fl, rin = c.forces()
        assert np.array_equal(it, ref["forces"][0])
        assert np.array_equal(fd, ref["forces"][1]) and np.array_equal(fl, ref["forces"][2])
        assert np.array_equal(rin, ref["forces"][3])
    b.close()


@pytest.mark.parametrize("sched", [0, 1])
def test_batch_macro_fields_and_loaded_state(mrlbm, sched):
    cfgs = _cfgs()
    b = mrlbm.Batch(cfgs, precision=64)
    b.set_schedule(18, sched, 6)
    # a loaded state (x-and-y periodic case: override list on the first step) and field stats
    f0 = [c.get_state() for c in b.cases]
    for c, f in zip(b.cases, f0):
        c.load_state(f, iter=0)
        c.field_stats_window(3, 17)
    b.step(20, macro=True)
    for cfg, c, f in zip(cfgs, b.cases, f0):
        s = mrlbm.Simulation(cfg, precision=64)
        s.tile_config = 18
        s.load_state(f, iter=0)
        s.field_stats_window(3, 17)
        s.step(20, macro=True)
        assert np.array_equal(c.get_state(), s.get_state())
        m1, m2 = c.macro(), s.macro()
        for k in m1:
            assert np.array_equal(m1[k], m2[k]), k
        f1, f2 = c.field_stats(), s.field_stats()
        assert f1["n"] == f2["n"] == 15
        for k in ("mean_u", "rms_v", "mean_p"):
            assert np.array_equal(f1[k], f2[k]), k
        s.close()
    b.close()


def test_batch_autotune_restores_state(mrlbm):
    cfgs = _cfgs()
    b = mrlbm.Batch(cfgs, precision=32)
    b.step(4)
    before = [c.get_state() for c in b.cases]
    (tile, sched, spl), ms = b.autotune(trial_steps=8)
    # vector shapes under the persistent or split-graph schedule; one-tile-per-block shapes as
    # split-graph steps or per-case streams
    assert (16 <= tile <= 21 and sched in (0, 1)) or (0 <= tile < 10 and sched in (1, 2))
    assert ms > 0
    for c, f in zip(b.cases, before):
        assert np.array_equal(c.get_state(), f)
        assert c.iter == 5
    b.step(6)
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, 32, 10)
        assert np.array_equal(c.get_state(), ref["f"])
        assert np.array_equal(c.forces()[1], ref["forces"][1])
    assert b.status() == 0
    b.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_batch_streams_calls_interleave_with_split_calls(mrlbm, prec):
    """Per-case streams calls replay captured launches with each call's iteration and record
    slots; calls they cannot take (a field-statistics window, macroscopic output) run as split
    steps in between, and the records, fields and states still equal stepping each case alone."""
    cfgs = _cfgs()
    b = mrlbm.Batch(cfgs, precision=prec)
    b.set_schedule(9, mrlbm.BATCH_STREAMS, 6)
    for c in b.cases:
        c.field_stats_window(14, 19)
    b.step(6)                                    # iterations 2..7: the periodic case's first step
                                                 # carries its corner overrides: split steps
    n0 = b.launch_count()
    b.step(6)                                    # 8..13: one replay
    per_step = 1 if prec == 32 else 2            # FP32 tile shapes: one launch per step
    assert b.launch_count() - n0 == 6 * len(cfgs) * per_step
    b.step(9)                                    # iterations 14..19 in the window: split; 20..22 replayed,
                                                 # plot step 21 included
    b.step(8, macro=True)                        # 23..28 replayed; 29..30 with fields: split
    assert b.status() == 0
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, prec, 29, macro=True, fields=(14, 19))
        assert np.array_equal(c.get_state(), ref["f"])
        it, fd, fl, rin = c.forces()
        assert np.array_equal(it, ref["forces"][0])
        assert np.array_equal(fd, ref["forces"][1]) and np.array_equal(fl, ref["forces"][2])
        assert np.array_equal(rin, ref["forces"][3])
        m1, m2 = c.macro(), ref["macro"]
        for k in m1:
            assert np.array_equal(m1[k], m2[k]), k
        f1, f2 = c.field_stats(), ref["fields"]
        assert f1["n"] == f2["n"] == 6
        for k in ("mean_u", "rms_v", "mean_p"):
            assert np.array_equal(f1[k], f2[k]), k
    b.close()


def test_batch_step_rejects_surface_records(mrlbm):
    """Surface-pressure records come from single-case steps; a batch step refuses a case that
    has them switched on instead of silently skipping them."""
    b = mrlbm.Batch(_cfgs()[:2], precision=64)
    b.cases[0].surface_enable()
    with pytest.raises(mrlbm.MrlbmError) as e:
        b.step(2)
    assert e.value.code == 4
    b.cases[0].surface_enable(False)
    b.step(2)
    assert b.status() == 0
    b.close()


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("sched,tile", [(1, 9), (2, 7), (0, 18)])
def test_batch_closure_variants_match_single_cases(mrlbm, prec, sched, tile):
    """The curved-wall closure variants (weak, rho_eq, unrotated, none, no velocity
    extrapolation) through every batch schedule, bit for bit against stepping alone."""
    names = ["closure_weak", "closure_rhoeq", "closure_unrotated", "no_velocity_interp"]
    cfgs = [CASES[n]() for n in names] + [CASES["reference_default_bcs"]().replace(strong_mass_bc=0)]
    b = mrlbm.Batch(cfgs, precision=prec)
    b.set_schedule(tile, sched, 6)
    b.step(15)
    assert b.status() == 0
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, prec, 15)
        assert np.array_equal(c.get_state(), ref["f"])
        assert np.array_equal(c.forces()[1], ref["forces"][1])
    b.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_batch_streams_statistics_window_inside_calls(mrlbm, prec):
    """A statistics window that opens and closes inside replayed calls: each replay derives
    which of its steps keep a record, and in which ring slot, from the uploaded call state."""
    cfgs = [c.replace(statsbegin=10, statsend=25) for c in _cfgs()]
    b = mrlbm.Batch(cfgs, precision=prec)
    b.set_schedule(9, mrlbm.BATCH_STREAMS, 7)
    b.step(7)                                    # the periodic case's overrides: split steps
    b.step(23)                                   # replays (7, 7, 7) and a 2-step call
    assert b.status() == 0
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, prec, 30)
        assert np.array_equal(c.get_state(), ref["f"])
        it, fd, fl, rin = c.forces()
        assert np.array_equal(it, ref["forces"][0]) and it[0] == 10 and it[-1] == 25
        assert np.array_equal(fd, ref["forces"][1]) and np.array_equal(rin, ref["forces"][3])
    b.close()


def test_batch_streams_ring_drains_between_replays(mrlbm):
    """More records than the device ring holds (8192): the streams schedule drains the ring
    between replays and the history still equals stepping alone."""
    cfgs = [CASES["reference_default_bcs"](), CASES["freeslip_label15"]()]
    b = mrlbm.Batch(cfgs, precision=32)
    b.set_schedule(0, mrlbm.BATCH_STREAMS, 100)
    b.step(8300)
    assert b.status() == 0
    for cfg, c in zip(cfgs, b.cases):
        ref = _alone(mrlbm, cfg, 32, 8300)
        it, fd, fl, rin = c.forces()
        assert len(it) == 8300
        assert np.array_equal(it, ref["forces"][0])
        assert np.array_equal(fd, ref["forces"][1]) and np.array_equal(fl, ref["forces"][2])
        assert np.array_equal(c.get_state(), ref["f"])
    b.close()
