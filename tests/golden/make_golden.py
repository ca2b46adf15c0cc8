"""Generate golden fixtures by executing the reference's own source text.

    python tests/golden/make_golden.py [--only NAME]

Reads 2d_mrlbm.f90 and 2d_statistics.f90 from the reference checkout named by the
REFERENCE_DIR environment variable (required), runs them with tests/golden/fortran_subset.py on
small inputs the unmodified reference can express, and writes tests/golden/<case>.npz.  Every
random input is drawn from a generator keyed by a stable function of the case name, and the
archives are written with fixed member timestamps, so a second run reproduces the committed
files byte for byte.  Each case is an input.dat (written below)
plus, for the restart cases, a restart.dat record (soln_time, f, f_eq, ux, uy, rho) that
the reference reads through its own irestart = 1 path (2d_mrlbm.f90:208-212, 2204-2220), so
the curved-wall closure runs on a developed, non-symmetric flow from the first step.

Captured outputs (the reference's own files, as records of values):
  restart/restart.dat       f, ux, uy, rho after each isave steps (2d_mrlbm.f90:2198)
  data_mean/forces_time.dat iter, F_drag_net, F_lift_net per stats step (2d_mrlbm.f90:493)
  data_mean/p_surface*.dat  surface pressure, raw and smoothed (2d_mrlbm.f90:609-616)
  data_probe/*_probe.dat    probe signals (2d_mrlbm.f90:471-476)
  output/grid1*.bin         PLOT3D rho, ux, uy (float32) every iplot steps (2d_mrlbm.f90:2177-2180)
  data_mean/theta.dat       sorted wall angles (2d_mrlbm.f90:1158-1162)
The fixtures are committed; this script is only re-run when the cases change.
"""
import argparse
import io
import os
import sys
import time
import zipfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from fortran_subset import Interpreter  # noqa: E402

REF = os.environ.get("REFERENCE_DIR")


def reference_source(name):
    if not REF:
        raise SystemExit("set REFERENCE_DIR to the reference checkout (the directory holding 2d_mrlbm.f90)")
    return open(os.path.join(REF, name)).read()


def save_npz(path, **arrays):
    """np.savez_compressed with fixed member timestamps (byte-reproducible archives)."""
    with zipfile.ZipFile(path, "w", compression=zipfile.ZIP_DEFLATED) as z:
        for key in sorted(arrays):
            buf = io.BytesIO()
            np.lib.format.write_array(buf, np.asanyarray(arrays[key]), allow_pickle=False)
            info = zipfile.ZipInfo(key + ".npy", date_time=(1980, 1, 1, 0, 0, 0))
            info.compress_type = zipfile.ZIP_DEFLATED
            info.external_attr = 0o600 << 16
            z.writestr(info, buf.getvalue())

INPUT = """&DomainSize
\tnx = 16
\tny = 16
\tlattice_type = 9
/
&Cylinder
\tncy = {ncy}
\tL_front = {L_front}
\tL_back = {L_back}
\tL_top = {L_top}
\tL_bot = {L_bot}
/
&Numbers
\tRe = {Re}
/
&Parallel
\tnum_threads=1
/
&Controls
\tuo = {uo}
\trho_infty = 1.0
\tiplot = {iplot}
\tmax_iter = {max_iter}
\tisave = {isave}
\tirestart = {irestart}
\tstatsbegin = {statsbegin}
\tstatsend = {statsend}
\tiplotstats = 1000
/
&LogicalControls
\tpost_process = .true.
\tx_periodic = {x_periodic}
\ty_periodic = {y_periodic}
\tchannel_with_cylinder = .true.
\tchannel_with_square = .false.
\tincomp_bc = {incomp_bc}
\tincomp_bulk = {incomp_bulk}
\tvel_interp = {vel_interp}
\tmom_interp = .true.
\trotated_coordinate = {rotated}
\tstrong_mass_bc = {strong}
\teq_mass_bc = {eq}
\tweak_mass_bc = {weak}
/
"""

T, F = ".true.", ".false."
BASE = dict(ncy=10, L_front=2, L_back=3, L_top=1, L_bot=1, Re=60, uo=0.05, iplot=4, max_iter=8, isave=4,
            irestart=1, statsbegin=1, statsend=1000, x_periodic=F, y_periodic=T, incomp_bc=F, incomp_bulk=F,
            vel_interp=T, rotated=T, strong=T, eq=F, weak=F)

CASES = {
    "ref_default_restart": dict(),
    "ref_rest_start": dict(irestart=0, max_iter=6, isave=3, iplot=3),
    "ref_walls": dict(y_periodic=F),
    "ref_walls_incomp": dict(y_periodic=F, incomp_bc=T, incomp_bulk=T),
    "ref_weak": dict(strong=F, weak=T),
    "ref_rhoeq": dict(strong=F, eq=T),
    "ref_unrotated": dict(rotated=F),
    "ref_no_vel_interp": dict(vel_interp=F),
    "ref_periodic_xy": dict(x_periodic=T),
}


def restart_state(case, nx, ny):
    """A seeded, developed-looking population field: regularized equilibrium of a
    perturbed uniform flow (rho = 1 + 1e-2 n, u = U + 0.2 U n, v = 0.2 U n)."""
    rng = np.random.default_rng(zlib.crc32(case.encode()))      # stable across processes
    U = 0.05
    rho = 1.0 + 1e-2 * rng.standard_normal((nx, ny))
    u = U + 0.2 * U * rng.standard_normal((nx, ny))
    v = 0.2 * U * rng.standard_normal((nx, ny))
    w = np.array([np.float32(16.0) / np.float32(36.0)] + [np.float32(4.0) / np.float32(36.0)] * 4 +
                 [np.float32(1.0) / np.float32(36.0)] * 4, dtype=np.float64)
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
    f = np.empty((nx, ny, 9), order="F")
    for k in range(9):
        cu = ex[k] * u + ey[k] * v
        hxx, hyy = ex[k] ** 2 - 1 / 3, ey[k] ** 2 - 1 / 3
        f[:, :, k] = w[k] * rho * (1 + 3 * cu + 4.5 * u * u * hxx + 4.5 * v * v * hyy + 9 * u * v * ex[k] * ey[k])
    return f


def run_case(name, over):
    prm = dict(BASE, **over)
    src = reference_source("2d_mrlbm.f90")
    text = INPUT.format(**prm)
    ncy = prm["ncy"]
    nx = (prm["L_front"] + 1 + prm["L_back"]) * ncy
    ny = (prm["L_top"] + 1 + prm["L_bot"]) * ncy
    it = Interpreter(src, inputs={"input.dat": text})
    f0 = None
    if prm["irestart"] == 1:
        f0 = restart_state(name, nx, ny)
        z = np.zeros((nx, ny), order="F")
        it.unformatted_inputs["restart/restart.dat"] = [[0, f0, np.zeros_like(f0), z, z, z + 1.0]]
    t0 = time.time()
    it.run()
    el = time.time() - t0
    files = it.files
    out = {"input_dat": np.array(text), "nx": nx, "ny": ny}
    print(f"{name}: interpreted in {el:.1f} s", flush=True)
    if f0 is not None:
        out["restart_in_f"] = f0
        out["restart_in_iter"] = 0
    snaps = it.history.get("restart/restart.dat", [])
    # each open rewrote the file; keep every record written (one per isave)
    for rec in snaps:
        t = int(rec[0])
        out[f"f_{t}"] = np.asarray(rec[1])
        out[f"ux_{t}"] = np.asarray(rec[3])
        out[f"uy_{t}"] = np.asarray(rec[4])
        out[f"rho_{t}"] = np.asarray(rec[5])
    fr = files.get("data_mean/forces_time.dat", [])
    out["forces"] = np.array([[float(r[0]), float(r[1]), float(r[2])] for r in fr])
    ps = files.get("data_mean/p_surface_time.dat", [])
    out["p_surface"] = np.array([[float(x) for x in r] for r in ps])
    pss = files.get("data_mean/p_surface_smooth_time.dat", [])
    out["p_surface_smooth"] = np.array([[float(x) for x in r] for r in pss])
    for nm in ("p", "ux", "uy"):
        rr = files.get(f"data_probe/{nm}_probe.dat", [])
        out[f"probe_{nm}"] = np.array([[float(x) for x in r] for r in rr])
    out["theta"] = np.array([float(r[0]) for r in files.get("data_mean/theta.dat", [])])
    for fname, recs in files.items():
        if fname.startswith("output/grid1") and fname.endswith(".bin\x00"):
            step = int(fname[len("output/grid"):len("output/grid") + 8]) - 10000000
            vals = recs[2]
            n = nx * ny
            arr = np.array([float(x) for x in vals], dtype=np.float32)
            out[f"plot3d_{step}"] = arr.reshape(3, ny, nx)
    sp = files.get("simulation_parameters.dat", [])
    out["sim_params"] = np.array([str(r) for r in sp])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default=None)
    ap.add_argument("--stats", action="store_true")
    a = ap.parse_args()
    for name, over in CASES.items():
        if a.only and name != a.only:
            continue
        out = run_case(name, over)
        path = os.path.join(HERE, name + ".npz")
        save_npz(path, **out)
        print(f"{name}: {len(out['forces'])} force records -> {path}", flush=True)


if __name__ == "__main__" and "--stats" not in sys.argv:
    main()


# ---------------------------------------------------------------------------------------
# 2d_statistics.f90 on synthetic force / surface-pressure histories
STAT_CASES = {
    # name: (nstep, period, lift amplitude, mean drag, nbct, r_cy, uo, rho_infty)
    "stats_sine": (400, 37.3, 0.02, 0.09, 24, 10.5, 0.05, 1.01),
    "stats_short_cycles": (260, 61.7, 0.015, 0.07, 16, 5.3851648071345, 0.04, 0.998),
}


def run_stats_case(name, prm):
    nstep, period, amp, fd0, nbct, r_cy, uo, rho_inf = prm
    rng = np.random.default_rng(len(name) * 7919)
    t = np.arange(1, nstep + 1)
    phase = rng.uniform(0, 2 * np.pi)
    fl = amp * np.sin(2 * np.pi * t / period + phase) + 1e-5 * rng.standard_normal(nstep)
    fd = fd0 + 0.1 * amp * np.sin(4 * np.pi * t / period + 2 * phase) + 1e-5 * rng.standard_normal(nstep)
    theta = np.sort(rng.uniform(0, 2 * np.pi, nbct))
    ps = (1.0 / 3.0) * (1 + 1e-3 * rng.standard_normal((nstep, nbct)))
    psf = ps + 1e-5 * rng.standard_normal((nstep, nbct))
    src = reference_source("2d_statistics.f90")
    text = (f"&parameters\n\tnbct = {nbct}\n\tr_cy = {r_cy!r}\n\tuo = {uo!r}\n\trho_infty = {rho_inf!r}\n/\n")
    it = Interpreter(src, inputs={"input_stat.dat": text})
    it.text_records["data_mean/forces_time.dat"] = [[int(a), float(b), float(c)] for a, b, c in zip(t, fd, fl)]
    it.text_records["data_mean/theta.dat"] = [[float(x)] for x in theta]
    it.unformatted_inputs["data_mean/p_surface_time.dat"] = [[int(a)] + [float(x) for x in row] for a, row in zip(t, ps)]
    it.unformatted_inputs["data_mean/p_surface_smooth_time.dat"] = [[int(a)] + [float(x) for x in row]
                                                                   for a, row in zip(t, psf)]
    it.run()
    f = it.files
    dl = f["plots/drag_lift.dat"]
    out = {"nstep": nstep, "nbct": nbct, "r_cy": r_cy, "uo": uo, "rho_infty": rho_inf, "iter": t, "f_drag": fd,
           "f_lift": fl, "theta": theta, "p_surface": ps, "p_surface_smooth": psf,
           "St": float(dl[0][-1]), "Cd": float(dl[1][-1]), "Cl_rms": float(dl[2][-1]),
           "cp": np.array([[float(x) for x in r] for r in f["plots/cp.dat"]]),
           "cp_fit": np.array([[float(x) for x in r] for r in f["plots/cp_fit.dat"]]),
           "cd_time": np.array([[float(x) for x in r] for r in f["plots/cd_time.dat"]]),
           "cl_time": np.array([[float(x) for x in r] for r in f["plots/cl_time.dat"]])}
    return out


def main_stats(only=None):
    for name, prm in STAT_CASES.items():
        if only and name != only:
            continue
        out = run_stats_case(name, prm)
        save_npz(os.path.join(HERE, name + ".npz"), **out)
        print(f"{name}: St={out['St']:.6f} Cd={out['Cd']:.6f} Cl_rms={out['Cl_rms']:.6f}", flush=True)


if __name__ == "__main__" and "--stats" in sys.argv:
    main_stats()
