"""The input_stat.dat-driven post-processing run (mrlbm_statistics) against the reference's.

The fixtures tests/golden/stats_*.npz hold what 2d_statistics.f90 itself computed and wrote
(plots/cp.dat, cp_fit.dat, cd_time.dat, cl_time.dat, drag_lift.dat) when executed on two
synthetic force and surface-pressure histories.  Here the same histories are laid out as the
reference's input files (input_stat.dat, data_mean/forces_time.dat, theta.dat and the two
unformatted p_surface*_time.dat), the driver is run in that directory, and every value it
writes must equal the reference's bit for bit.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _record(payload):
    return struct.pack("<i", len(payload)) + payload + struct.pack("<i", len(payload))


def _write_inputs(d, g):
    (d / "data_mean").mkdir()
    (d / "input_stat.dat").write_text(
        f"&parameters\n\tnbct = {int(g['nbct'])}\n\tr_cy = {float(g['r_cy'])!r}\n\tuo = {float(g['uo'])!r}\n"
        f"\trho_infty = {float(g['rho_infty'])!r}\n/\n")
    with open(d / "data_mean" / "forces_time.dat", "w") as f:
        for it, a, b in zip(g["iter"], g["f_drag"], g["f_lift"]):
            f.write(f"{int(it):12d} {float(a)!r} {float(b)!r}\n")
    with open(d / "data_mean" / "theta.dat", "w") as f:
        for t in g["theta"]:
            f.write(f"{float(t)!r}\n")
    for name, key in (("p_surface_time.dat", "p_surface"), ("p_surface_smooth_time.dat", "p_surface_smooth")):
        with open(d / "data_mean" / name, "wb") as f:
            for it, row in zip(g["iter"], g[key]):
                f.write(_record(struct.pack("<i", int(it)) + np.asarray(row, dtype="<f8").tobytes()))


def _read_table(path):
    rows = []
    for line in open(path):
        parts = line.split()
        if parts:
            rows.append([float(x) for x in parts])
    return np.array(rows)


@pytest.mark.parametrize("case", ["stats_sine", "stats_short_cycles"])
def test_statistics_driver_matches_reference_outputs(mrlbm, tmp_path, case):
    g = np.load(os.path.join(GOLDEN, case + ".npz"))
    _write_inputs(tmp_path, g)
    exe = os.path.join(ROOT, "mrlbm_2d_b200", "mrlbm_statistics")
    out = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Averging over" in out.stdout
    for name in ("cp", "cp_fit", "cd_time", "cl_time"):
        got = _read_table(tmp_path / "plots" / f"{name}.dat")
        ref = g[name]
        assert got.shape == ref.shape, (name, got.shape, ref.shape)
        if name in ("cd_time", "cl_time"):
            # the phase column is a default REAL (single precision) in the reference
            assert np.array_equal(got[:, 0].astype(np.float32), ref[:, 0].astype(np.float32)), name
            assert np.array_equal(got[:, 1], ref[:, 1]), name
        else:
            assert np.array_equal(got, ref), name
    lines = (tmp_path / "plots" / "drag_lift.dat").read_text().splitlines()
    vals = [float(ln.split(":")[-1]) for ln in lines]
    assert vals == [float(g["St"]), float(g["Cd"]), float(g["Cl_rms"])]


def test_statistics_driver_reports_missing_peaks(mrlbm, tmp_path):
    """A lift history without two local maxima stops the run as the reference does."""
    g = dict(np.load(os.path.join(GOLDEN, "stats_sine.npz")))
    g["f_lift"] = np.linspace(0.0, 1.0, len(g["f_lift"]))
    _write_inputs(tmp_path, g)
    exe = os.path.join(ROOT, "mrlbm_2d_b200", "mrlbm_statistics")
    out = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "Could not detect two peaks" in out.stdout
