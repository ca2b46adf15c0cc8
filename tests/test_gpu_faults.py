"""Failure detection without a GPU fault.

The reference stops on a bad read and prints-and-continues elsewhere (2d_mrlbm.f90:2236-2237,
1362); here a step that meets a non-positive or NaN density raises a device flag the host reads
as MRLBM_EDEVICE_NAN, and a bounded wait inside a kernel that gives up ends the launch with
MRLBM_EDEVICE_TIMEOUT.  Both are provoked with ordinary inputs: a loaded state holding a node of
negative density, and a persistent batch launch whose grid-barrier watchdog is set to one poll,
so healthy blocks that arrive early give up.  No load, copy or wait is left in flight by either,
and the context stays usable afterwards.
"""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu

EDEVICE_NAN, EDEVICE_TIMEOUT = -2, -4


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("tile", [1, 18])
def test_negative_density_raises_the_device_flag(mrlbm, prec, tile):
    cfg = CASES["reference_default_bcs"]()
    s = mrlbm.Simulation(cfg, precision=prec)
    s.tile_config = tile
    s.step(3)
    assert s.status() == 0
    f = s.get_state()
    f[60, 10, :] = -0.1                         # node (61, 11): rho = -0.9, far from the cylinder
    s.load_state(f, iter=s.iter)
    s.step(1)
    assert s.status() == EDEVICE_NAN
    assert s.status() == EDEVICE_NAN            # sticky until the handle is destroyed
    s.close()
    t = mrlbm.Simulation(cfg, precision=prec)
    t.step(5)
    assert t.status() == 0
    t.close()


def test_nan_population_raises_the_device_flag(mrlbm):
    cfg = CASES["freeslip_label15"]()
    s = mrlbm.Simulation(cfg, precision=64)
    f = s.get_state()
    f[90, 30, 2] = np.nan
    s.load_state(f, iter=1)
    s.step(1)
    assert s.status() == EDEVICE_NAN
    s.close()


def test_batch_grid_barrier_watchdog(mrlbm):
    """A persistent launch of several steps whose barrier watchdog allows a single poll: blocks
    that reach a barrier before the last one give up, the launch ends, and the batch reports
    MRLBM_EDEVICE_TIMEOUT.  A fresh simulation on the same device then steps normally."""
    from mrlbm_2d_b200.config import sweep_cases
    cfgs = sweep_cases(4)
    b = mrlbm.Batch(cfgs, precision=mrlbm.FP32)
    b.set_schedule(18, mrlbm.BATCH_PERSISTENT, 16)
    b.step(16)
    assert b.status() == 0                      # default watchdog: no timeout
    b.set_wait_limit(1)
    b.step(32)
    assert b.status() == EDEVICE_TIMEOUT
    b.close()
    s = mrlbm.Simulation(CASES["reference_default_bcs"](), precision=32)
    s.step(10)
    assert s.status() == 0
    s.close()
