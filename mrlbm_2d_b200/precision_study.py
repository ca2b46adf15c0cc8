"""FP32 (deviation storage) against FP64 on the same case: force statistics and fields.

    python -m mrlbm_2d_b200.precision_study --case small --steps 20000 [--stats-from 8000]

Runs the case twice on one GPU (FP64 reference-order step, FP32 deviation step) from the
same seeded initial state, records the per-step drag and lift, and reports
  * St, Cd (mean), Cl_rms of each run over whole shedding cycles (2d_statistics.f90:90-131,
    normalised by 0.5 rho_infty U^2 D with rho_infty = 1 and D = 2 r_c),
  * a spectral Strouhal number (peak of the windowed lift spectrum), which unlike the
    reference's first-two-maxima period is not thrown off by small ripples on the lift,
  * |dCd|/Cd, |dSt|, |dCl_rms|/Cl_rms of FP32 against FP64,
  * the relative L2 error of the final velocity field, max |du|/U,
  * with --fields, the relative L2 and max errors of the FP64-accumulated mean and rms fields
    of u, v and p over the statistics window,
and the wall-clock MLUPS of each run.  One JSON line on stdout.
"""
import argparse
import json
import time

import numpy as np

from . import api
from .config import case_adjoint, case_large, case_mid, case_small

CASES = {"small": case_small, "mid": case_mid, "adjoint": case_adjoint, "large": case_large}


def run(cfg, precision, steps, chunk=5000, fields_from=None):
    sim = api.Simulation(cfg, precision=precision)
    if fields_from is not None:
        sim.field_stats_window(fields_from, steps + 1)
    fd, fl = [], []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        sim.step(n, macro=(done + n == steps))
        _, d, l, _ = sim.forces()
        fd.append(d)
        fl.append(l)
        done += n
    mac = sim.macro()
    el = time.perf_counter() - t0
    fields = sim.field_stats() if fields_from is not None else None
    st = sim.status()
    sim.close()
    if st != 0:
        raise RuntimeError(f"device error flag in fp{precision} run")
    return np.concatenate(fd), np.concatenate(fl), mac, cfg.nx * cfg.ny * steps / el / 1e6, fields


def spectral_strouhal(fl, D, U, rho_infty=1.0, pad=16):
    """St = f D / U with f the peak frequency (cycles per step) of the Hann-windowed,
    mean-removed lift, refined by a parabola through the peak bin and its neighbours."""
    x = np.asarray(fl, dtype=np.float64)
    x = (x - x.mean()) * np.hanning(len(x))
    n = len(x) * pad
    a = np.abs(np.fft.rfft(x, n))
    a[0] = 0.0
    k = int(np.argmax(a))
    d = 0.0
    if 0 < k < len(a) - 1:
        den = a[k - 1] - 2.0 * a[k] + a[k + 1]
        if den != 0.0:
            d = 0.5 * (a[k - 1] - a[k + 1]) / den
    f = (k + d) / n
    return f * D / U


def study(case="small", steps=20000, stats_from=None, fields=False, chunk=5000):
    """Both precisions on one case; returns the comparison as a dict (see the module text)."""
    cfg = CASES[case]()
    start = stats_from if stats_from is not None else steps // 2
    cfg = cfg.replace(statsbegin=start, statsend=steps + 10)
    out = {"case": case, "nx": cfg.nx, "ny": cfg.ny, "steps": steps, "stats_from": start,
           "D": 2 * cfg.r_c, "U": cfg.uo, "Re": cfg.Re}
    res = {}
    for prec in (64, 32):
        fd, fl, mac, mlups, flds = run(cfg, prec, steps, chunk=chunk, fields_from=start if fields else None)
        res.setdefault("fields", {})[prec] = flds
        r = {"mlups_wall": mlups}
        try:
            s = api.force_statistics(fd, fl, cfg.r_c, cfg.uo, 1.0)
            r.update(s)
        except api.MrlbmError as e:
            r["error"] = str(e)
        r["St_spectral"] = spectral_strouhal(fl, 2 * cfg.r_c, cfg.uo)
        res[prec] = (r, fd, fl, mac)
        out[f"fp{prec}"] = r
    r64, fd64, fl64, m64 = res[64]
    r32, fd32, fl32, m32 = res[32]
    if "Cd" in r64 and "Cd" in r32:
        out["rel_err_Cd"] = abs(r32["Cd"] - r64["Cd"]) / abs(r64["Cd"])
        out["abs_err_St"] = abs(r32["St"] - r64["St"])
        out["rel_err_Cl_rms"] = abs(r32["Cl_rms"] - r64["Cl_rms"]) / abs(r64["Cl_rms"])
    out["abs_err_St_spectral"] = abs(r32["St_spectral"] - r64["St_spectral"])
    du = np.sqrt((m32["ux"] - m64["ux"]) ** 2 + (m32["uy"] - m64["uy"]) ** 2)
    u64 = np.sqrt(m64["ux"] ** 2 + m64["uy"] ** 2)
    out["velocity_rel_l2"] = float(np.sqrt((du ** 2).sum() / (u64 ** 2).sum()))
    out["velocity_max_abs_over_U"] = float(du.max() / cfg.uo)
    out["drag_history_rel_l2"] = float(np.linalg.norm(fd32 - fd64) / np.linalg.norm(fd64))
    if fields:
        f32, f64 = res["fields"][32], res["fields"][64]
        for k in ("mean_u", "mean_v", "mean_p", "rms_u", "rms_v", "rms_p"):
            ref = f64[k] - (1.0 / 3.0 if k == "mean_p" else 0.0)   # p relative to rest pressure
            out[f"{k}_rel_l2"] = float(np.linalg.norm(f32[k] - f64[k]) / max(np.linalg.norm(ref), 1e-300))
            out[f"{k}_max_abs"] = float(np.abs(f32[k] - f64[k]).max())
        out["field_samples"] = int(f64["n"])
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="small", choices=sorted(CASES))
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--stats-from", type=int, default=None, help="first step of the statistics window")
    ap.add_argument("--fields", action="store_true",
                    help="also accumulate FP64 mean/rms fields of u, v, p over the statistics window")
    a = ap.parse_args(argv)
    out = study(a.case, a.steps, a.stats_from, a.fields)
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
