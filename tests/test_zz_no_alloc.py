"""mrlbm_step_noalloc: stepping for callers that cannot let the library allocate device
memory (their device memory comes from their own runtime, pool or arena).

The case comes from a host-only handle (no device allocation); the caller -- here the test,
through torch -- owns the two population time levels and the initial populations.  The
result must equal the ordinary entry point's (mrlbm_step on a device handle) within the
tolerances of the parity tests -- exact equality for the populations and for the per-step
force and inlet-density sums -- over two calls in a row.  The file is collected last on purpose.
"""
import numpy as np
import pytest

from cases import CASES

pytestmark = pytest.mark.gpu

EX = [0, 1, 0, -1, 0, 1, -1, -1, 1]
EY = [0, 0, 1, 0, -1, 1, 1, -1, -1]
MIRROR = [0, 1, 4, 3, 2, 8, 7, 6, 5]


def _source(nx, ny, i, j, k, xper, yper, freeslip):
    """Slot whose value is population (i,j,k) at the next step (lattice.h stream_source)."""
    dx, dy = EX[k], EY[k]
    if freeslip and not yper and ((j == ny and dy == -1) or (j == 1 and dy == 1)):
        ti = i - dx
        if 1 <= ti <= nx:
            return ti, j, MIRROR[k]
        if xper:
            return (nx if ti < 1 else 1), j, MIRROR[k]
        return i - dx, j - dy, k
    if yper and j == 1 and dy == 1:
        return i, ny, k
    if yper and j == ny and dy == -1:
        return i, 1, k
    if xper and i == 1 and dx == 1:
        return nx, j, k
    if xper and i == nx and dx == -1:
        return 1, j, k
    return i - dx, j - dy, k


def _unpad(buf, info, cfg):
    """Populations f[i-1, j-1, k] from one padded time level."""
    nx, ny = info.nx, info.ny
    idx = np.empty((nx, ny, 9), dtype=np.int64)
    fs = cfg.wall_mode == 1 and not cfg.y_periodic
    for k in range(9):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                si, sj, sk = _source(nx, ny, i, j, k, cfg.x_periodic, cfg.y_periodic, fs)
                idx[i - 1, j - 1, k] = sk * info.plane + sj * info.pitch + si + info.off
    return buf[idx]


@pytest.mark.parametrize("name", ["x_and_y_periodic", "benchmark_small_400x100"])
def test_step_noalloc_matches_step(mrlbm, name):
    torch = pytest.importorskip("torch")
    cfg = CASES[name]()
    n1, n2 = 7, 6
    ref = mrlbm.Simulation(cfg, precision=mrlbm.FP64, device=0)
    f0 = ref.get_state()
    ref.step(n1)
    it_a, fd_a, fl_a, rin_a = ref.forces()
    f_a = ref.get_state()
    ref.step(n2)
    it_b, fd_b, fl_b, rin_b = ref.forces()
    f_b = ref.get_state()
    ref.close()

    host = mrlbm.Simulation(cfg, precision=mrlbm.FP64, device=-1)
    info = host.info
    assert np.array_equal(host.get_state(), f0)
    state = torch.zeros(int(info.state_bytes) // 8, dtype=torch.float64, device="cuda")
    d_f0 = torch.from_numpy(np.ascontiguousarray(f0.transpose(2, 1, 0)).ravel()).to("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rec1 = host.step_noalloc(state.data_ptr(), n1, d_f0_ptr=d_f0.data_ptr(), stream_ptr=stream)
    half = int(info.state_bytes) // 16
    cur = n1 % 2
    f1 = _unpad(state.cpu().numpy()[cur * half:(cur + 1) * half], info, cfg)
    assert np.array_equal(f1, f_a)
    rec2 = host.step_noalloc(state.data_ptr(), n2, stream_ptr=stream)
    cur = (n1 + n2) % 2
    f2 = _unpad(state.cpu().numpy()[cur * half:(cur + 1) * half], info, cfg)
    assert np.array_equal(f2, f_b)
    for rec, it, fd, fl, rin in ((rec1, it_a, fd_a, fl_a, rin_a), (rec2, it_b, fd_b, fl_b, rin_b)):
        assert np.array_equal(rec[:, 0].astype(int), it)
        assert np.array_equal(rec[:, 1], fd) and np.array_equal(rec[:, 2], fl)
        assert np.array_equal(rec[:, 3], rin)
    assert host.iter == ref_iter(n1 + n2)
    host.close()


def ref_iter(n):
    return 1 + n


def test_step_noalloc_rejects_device_handles_and_oversize_cases(mrlbm):
    torch = pytest.importorskip("torch")
    from mrlbm_2d_b200.config import cylinder_case
    dev = mrlbm.Simulation(CASES["benchmark_small_400x100"](), device=0)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(mrlbm.MrlbmError) as e:
        dev.step_noalloc(buf.data_ptr(), 1)
    assert e.value.code == 1
    dev.close()
    big = mrlbm.Simulation(cylinder_case(3000, 800, 400, 800.0, 400.5, 100.0, 0.05), device=-1)
    assert big.nbct > 1024
    with pytest.raises(mrlbm.MrlbmError) as e:
        big.step_noalloc(buf.data_ptr(), 1)
    assert e.value.code == 1 and "1024" in str(e.value)
