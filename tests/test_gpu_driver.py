"""mrlbm_run as a drop-in for the reference's a.out: run it in a directory holding an
input.dat the reference was executed with (tests/golden), then compare the files it writes
with the reference's own outputs for that input."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(os.path.dirname(HERE), "mrlbm_2d_b200", "mrlbm_run")


def read_records(path):
    """Fortran unformatted sequential records (4-byte markers, gfortran subrecords)."""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos < len(data):
        rec = b""
        while True:
            lead = int(np.frombuffer(data[pos:pos + 4], np.int32)[0])
            n = abs(lead)
            rec += data[pos + 4:pos + 4 + n]
            pos += 8 + n
            if lead >= 0:
                break
        out.append(rec)
    return out


def test_driver_reproduces_reference_outputs(mrlbm, tmp_path):
    d = dict(np.load(os.path.join(HERE, "golden", "ref_rest_start.npz")))
    (tmp_path / "input.dat").write_text(str(d["input_dat"]))
    r = subprocess.run([DRIVER, "--print-every", "3"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "STEP:" in r.stdout
    nx, ny = int(d["nx"]), int(d["ny"])
    # restart.dat: soln_time, f, f_eq, ux, uy, rho of the last save (iter 6)
    rec = read_records(tmp_path / "restart" / "restart.dat")[0]
    it = int(np.frombuffer(rec[:4], np.int32)[0])
    assert it == 6
    vals = np.frombuffer(rec[4:], np.float64)
    n = nx * ny
    f = vals[:9 * n].reshape(9, ny, nx).transpose(2, 1, 0)
    assert np.array_equal(f, d["f_6"])
    ux = vals[18 * n:19 * n].reshape(ny, nx).T
    rho = vals[20 * n:21 * n].reshape(ny, nx).T
    assert np.array_equal(ux, d["ux_6"]) and np.array_equal(rho, d["rho_6"])
    # PLOT3D function files at the plot steps
    for step in (3, 6):
        recs = read_records(tmp_path / "output" / f"grid{10000000 + step}.bin")
        assert np.frombuffer(recs[1], np.int32).tolist() == [nx, ny, 3]
        v = np.frombuffer(recs[2], np.float32).reshape(3, ny, nx)
        assert np.array_equal(v, d[f"plot3d_{step}"])
    g = read_records(tmp_path / "output" / "grid.x")
    assert np.frombuffer(g[1], np.int32).tolist() == [nx, ny]
    # forces_time.dat: iter, F_drag_net, F_lift_net (list-directed text)
    rows = np.loadtxt(tmp_path / "data_mean" / "forces_time.dat")
    assert np.array_equal(rows[:, 0], d["forces"][:, 0])
    # list-directed REAL(8) output carries 17 significant digits, so the text reads back exactly
    assert np.array_equal(rows[:, 1:], d["forces"][:, 1:])
    theta = np.loadtxt(tmp_path / "data_mean" / "theta.dat")
    assert np.array_equal(theta, d["theta"])
    # unformatted wall-pressure records: iter and the theta-ordered values (2d_mrlbm.f90:609-616)
    for fname, key in (("p_surface_time.dat", "p_surface"), ("p_surface_smooth_time.dat", "p_surface_smooth")):
        recs = read_records(tmp_path / "data_mean" / fname)
        assert len(recs) == len(d[key])
        for rec, ref in zip(recs, d[key]):
            assert int(np.frombuffer(rec[:4], np.int32)[0]) == int(ref[0])
            assert np.array_equal(np.frombuffer(rec[4:], np.float64), ref[1:]), fname
