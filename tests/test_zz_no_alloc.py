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


# the reference's single-rounded weights (default-real literals, 2d_mrlbm.f90:129)
W = np.array([np.float32(16.0) / np.float32(36.0)] + [np.float32(4.0) / np.float32(36.0)] * 4 +
             [np.float32(1.0) / np.float32(36.0)] * 4, dtype=np.float64)


def _unpad(buf, info, cfg, prec):
    """Populations f[i-1, j-1, k] from one padded time level (FP32 levels hold f_k - w_k)."""
    nx, ny = info.nx, info.ny
    idx = np.empty((nx, ny, 9), dtype=np.int64)
    fs = cfg.wall_mode == 1 and not cfg.y_periodic
    for k in range(9):
        for j in range(1, ny + 1):
            for i in range(1, nx + 1):
                si, sj, sk = _source(nx, ny, i, j, k, cfg.x_periodic, cfg.y_periodic, fs)
                idx[i - 1, j - 1, k] = sk * info.plane + sj * info.pitch + si + info.off
    f = buf[idx]
    return f if prec == 64 else W[None, None, :] + f.astype(np.float64)


# (case, precision, tile shape): the default one-tile-per-block shape 1 in both precisions and
# the 128-bit vector shape 18, which accesses the caller's buffer 16 bytes at a time
PARAMS = [("x_and_y_periodic", 64, 1), ("benchmark_small_400x100", 64, 1), ("benchmark_small_400x100", 32, 1),
          ("freeslip_label15", 64, 18), ("freeslip_label15", 32, 18)]


@pytest.mark.parametrize("name,prec,tile", PARAMS)
def test_step_noalloc_matches_step(mrlbm, name, prec, tile):
    torch = pytest.importorskip("torch")
    cfg = CASES[name]()
    n1, n2 = 7, 6
    ref = mrlbm.Simulation(cfg, precision=prec, device=0)
    ref.tile_config = tile
    f0 = ref.get_state()
    ref.step(n1)
    it_a, fd_a, fl_a, rin_a = ref.forces()
    f_a = ref.get_state()
    ref.step(n2)
    it_b, fd_b, fl_b, rin_b = ref.forces()
    f_b = ref.get_state()
    assert ref.status() == 0
    ref.close()

    host = mrlbm.Simulation(cfg, precision=prec, device=-1)
    host.tile_config = tile
    info = host.info
    f0_host = host.get_state()
    if prec == 64:
        assert np.array_equal(f0_host, f0)
    dt = torch.float64 if prec == 64 else torch.float32
    esz = 8 if prec == 64 else 4
    # torch's allocations start on 256-byte boundaries, so the buffer meets the 16-byte rule
    state = torch.zeros(int(info.state_bytes) // esz, dtype=dt, device="cuda")
    d_f0 = torch.from_numpy(np.ascontiguousarray(f0_host.transpose(2, 1, 0)).ravel()).to("cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rec1 = host.step_noalloc(state.data_ptr(), n1, d_f0_ptr=d_f0.data_ptr(), stream_ptr=stream)
    half = int(info.state_bytes) // (2 * esz)
    cur = n1 % 2
    f1 = _unpad(state.cpu().numpy()[cur * half:(cur + 1) * half], info, cfg, prec)
    assert np.array_equal(f1, f_a)
    rec2 = host.step_noalloc(state.data_ptr(), n2, stream_ptr=stream)
    cur = (n1 + n2) % 2
    f2 = _unpad(state.cpu().numpy()[cur * half:(cur + 1) * half], info, cfg, prec)
    assert np.array_equal(f2, f_b)
    for rec, it, fd, fl, rin in ((rec1, it_a, fd_a, fl_a, rin_a), (rec2, it_b, fd_b, fl_b, rin_b)):
        assert np.array_equal(rec[:, 0].astype(int), it)
        assert np.array_equal(rec[:, 1], fd) and np.array_equal(rec[:, 2], fl)
        assert np.array_equal(rec[:, 3], rin)
    assert host.iter == ref_iter(n1 + n2)
    host.close()


def ref_iter(n):
    return 1 + n


def test_step_noalloc_rejects_misaligned_buffers(mrlbm):
    """A state buffer that does not start on a 16-byte boundary (a view at an odd offset) is
    refused before anything is uploaded or launched."""
    torch = pytest.importorskip("torch")
    cfg = CASES["benchmark_small_400x100"]()
    host = mrlbm.Simulation(cfg, precision=64, device=-1)
    host.tile_config = 18
    buf = torch.zeros(int(host.info.state_bytes) // 8 + 2, dtype=torch.float64, device="cuda")
    with pytest.raises(mrlbm.MrlbmError) as e:
        host.step_noalloc(buf.data_ptr() + 8, 1)
    assert e.value.code == 1 and "16-byte" in str(e.value)
    assert host.iter == 1
    host.close()


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
