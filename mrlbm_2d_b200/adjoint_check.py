"""Adjoint gradient of mean drag against central finite differences on the 512 x 128 case.

    python -m mrlbm_2d_b200.adjoint_check [--steps 8000] [--window 2000] [--checkpoint 100]
                                          [--directions 16] [--rel-step 1e-4]

Case: 512 x 128, D = 32 at (128.0, 64.5), Re = 100, U = 0.05 (config.case_adjoint), FP64.
Parameters: a per-node body force (2 x 512 x 128, seeded N(0, 1e-7)) and the inlet profile
u_in(j) = U + seeded N(0, 1e-3).  J = mean drag over the last `window` of `steps` steps.  For
each seeded random direction d (body part N(0, 1e-7), inlet part N(0, 1e-3)) the adjoint's
directional derivative g . d is compared with (J(theta + h d) - J(theta - h d)) / 2h, h the
relative step.  Timing: wall clock of the forward-only and the gradient calls (second calls,
after warm-up).  One JSON line.
"""
import argparse
import json
import time

import numpy as np

from . import api
from .config import case_adjoint


def check(steps=8000, window=2000, checkpoint=100, directions=16, rel_step=1e-4, seed=2026, fp32=False):
    """Adjoint against central differences on the 512 x 128 case; returns the record as a dict."""
    cfg = case_adjoint()
    sim = api.Simulation(cfg, precision=api.FP64)
    rng = np.random.default_rng(seed)
    body = 1e-7 * rng.standard_normal((2, sim.nx, sim.ny))
    uin = cfg.uo + 1e-3 * rng.standard_normal(sim.ny)
    sim.set_body_force(body)
    sim.set_inlet_profile(uin)
    N, T, K = steps, window, checkpoint
    sim.adjoint_drag(N, T, K)                                  # warm-up
    t0 = time.perf_counter()
    J0 = sim.adjoint_drag(N, T, K, grads=False)
    t1 = time.perf_counter()
    J, gb, gu = sim.adjoint_drag(N, T, K)
    t2 = time.perf_counter()
    errs = []
    h = rel_step
    for _ in range(directions):
        db = 1e-7 * rng.standard_normal(body.shape)
        du = 1e-3 * rng.standard_normal(uin.shape)
        vals = []
        for sgn in (1.0, -1.0):
            sim.set_body_force(body + sgn * h * db)
            sim.set_inlet_profile(uin + sgn * h * du)
            vals.append(sim.adjoint_drag(N, T, K, grads=False))
        fd = (vals[0] - vals[1]) / (2.0 * h)
        ad = float((gb * db).sum() + (gu * du).sum())
        errs.append({"adjoint": ad, "fd": fd, "rel_err": abs(ad - fd) / abs(fd)})
    sim.close()
    rec32 = None
    if fp32:
        s32 = api.Simulation(cfg, precision=api.FP32)
        s32.set_body_force(body)
        s32.set_inlet_profile(uin)
        J32, gb32, gu32 = s32.adjoint_drag(N, T, K)
        s32.close()
        rel = []
        for _ in range(directions):
            db = rng.standard_normal(body.shape)
            du = rng.standard_normal(uin.shape)
            d64 = float((gb * db).sum() + (gu * du).sum())
            d32 = float((gb32 * db).sum() + (gu32 * du).sum())
            rel.append(abs(d32 - d64) / abs(d64))
        rec32 = {"J": J32, "rel_err_J": abs(J32 - J) / abs(J), "max_rel_err_vs_fp64_adjoint": max(rel)}
    return {"case": "512x128 D=32 Re=100 U=0.05", "steps": N, "window": T, "checkpoint_every": K, "J": J,
            "J_forward_only": J0, "directions": directions, "rel_step": h,
            "max_rel_err": max(e["rel_err"] for e in errs),
            "median_rel_err": float(np.median([e["rel_err"] for e in errs])),
            "forward_s": t1 - t0, "gradient_s": t2 - t1, "gradient_over_forward": (t2 - t1) / (t1 - t0),
            "grad_body_max": float(np.abs(gb).max()), "grad_uin_max": float(np.abs(gu).max()), "fp32": rec32,
            "checks": errs}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--window", type=int, default=2000)
    ap.add_argument("--checkpoint", type=int, default=100)
    ap.add_argument("--directions", type=int, default=16)
    ap.add_argument("--rel-step", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--fp32", action="store_true",
                    help="also run the adjoint on an FP32 handle (FP32 trajectory, FP64 adjoint) and compare")
    a = ap.parse_args(argv)
    out = check(a.steps, a.window, a.checkpoint, a.directions, a.rel_step, a.seed, a.fp32)
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
