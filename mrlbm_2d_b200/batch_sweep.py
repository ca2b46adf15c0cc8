"""Batched sweep of independent cylinder cases against stepping them one after another.

    python -m mrlbm_2d_b200.batch_sweep [--cases 64] [--steps 20000] [--seq-steps 2000]
                                        [--precision 32] [--trial-steps 50]
    python -m mrlbm_2d_b200.batch_sweep --compare-fp64 20000     # FP32 against FP64 mean drag per case

The cases are config.sweep_cases(n): nx uniform in [256, 1024] (multiples of 32), ny = nx/4,
D = ny/5 at (nx/5, ny/2 + 0.5), Re uniform in [40, 200], U = 0.05, seeded.  The batch is
autotuned (tile shape x schedule: persistent cooperative launches, CUDA-graph replays of
batched split steps, or each case's own step launches on per-case streams captured into one
replayed graph), then advanced `steps` steps; the baseline advances each case alone,
with its own autotuned single-case shape, `seq-steps` steps per case, one launch per step.
Aggregate MLUPS = sum of nodes x steps / device time (CUDA events on the launching
streams).  One JSON line.
"""
import argparse
import json
import time

import numpy as np

from . import api
from .config import sweep_cases


def sweep(cases=64, steps=20000, seq_steps=2000, precision=32, trial_steps=50, seed=4242, sequential=True,
          stream=None):
    """The batched sweep and (optionally) the one-case-at-a-time baseline; returns a dict."""
    import torch
    cfgs = sweep_cases(cases, seed=seed)
    nodes = [c.nx * c.ny for c in cfgs]
    total = float(sum(nodes))
    out = {"cases": cases, "nodes_total": int(total), "precision": precision, "steps": steps,
           "nx_range": [min(c.nx for c in cfgs), max(c.nx for c in cfgs)],
           "Re_range": [round(min(c.Re for c in cfgs), 2), round(max(c.Re for c in cfgs), 2)]}

    b = api.Batch(cfgs, precision=precision)
    t0 = time.perf_counter()
    (tile, sched, spl), ms = b.autotune(trial_steps=trial_steps)
    out["autotune"] = {"tile_shape": tile, "schedule": ["persistent", "graph", "streams"][sched], "steps_per_launch": spl,
                       "trial_ms_per_step": ms, "seconds": time.perf_counter() - t0}
    b.step(spl)                                   # warm-up of the chosen schedule
    bs = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = b.launch_count()
    torch.cuda.synchronize()
    e0.record(bs)
    b.step(steps)
    e1.record(bs)
    e1.synchronize()
    el = e0.elapsed_time(e1) * 1e-3
    st = b.status()
    if st == -4:
        raise RuntimeError("batch grid-barrier timeout")
    # cases whose density went non-positive or NaN (under-resolved low-viscosity cases)
    flagged = [i for i, c in enumerate(b.cases) if c.status() != 0]
    out["unstable_cases"] = [{"case": i, "nx": cfgs[i].nx, "Re": round(cfgs[i].Re, 2),
                              "tau": round(0.5 + 3.0 * cfgs[i].uo * 2.0 * cfgs[i].r_c / cfgs[i].Re, 5)}
                             for i in flagged]
    out["batch"] = {"seconds": el, "ms_per_step": el / steps * 1e3, "mlups": total * steps / el / 1e6,
                    "launches": b.launch_count() - n0}
    drag = []
    for i, c in enumerate(b.cases):
        _, fd, _, _ = c.forces()
        if i not in flagged:
            drag.append(float(fd[-1]))
    out["finite_forces_of_stable_cases"] = bool(np.all(np.isfinite(drag)))
    b.close()
    if not sequential:
        return out
    seq_el = 0.0
    st = stream or torch.cuda.Stream()
    for cfg in cfgs:
        s = api.Simulation(cfg, precision=precision)
        s.set_stream(st.cuda_stream)
        s.autotune(trial_steps=10)
        s.step(3)
        torch.cuda.synchronize()
        e0.record(st)
        s.step(seq_steps)
        e1.record(st)
        e1.synchronize()
        seq_el += e0.elapsed_time(e1) * 1e-3
        s.close()
    out["sequential"] = {"seconds": seq_el, "steps_per_case": seq_steps,
                         "mlups": total * seq_steps / seq_el / 1e6}
    out["speedup"] = out["batch"]["mlups"] / out["sequential"]["mlups"]
    return out


def precision_check(cases=64, steps=20000, seed=4242, trial_steps=10):
    """FP32 against FP64 on every case of the sweep, each precision stepped as one batch: the
    mean drag coefficient over the second half of `steps` steps per case, and its relative
    difference (cases whose density went non-positive in either precision are left out)."""
    cfgs = sweep_cases(cases, seed=seed)
    cd = {}
    for prec in (64, 32):
        b = api.Batch(cfgs, precision=prec)
        b.autotune(trial_steps=trial_steps)
        b.step(steps)
        vals = []
        for cfg, c in zip(cfgs, b.cases):
            _, fd, _, _ = c.forces()
            ok = c.status() == 0 and len(fd) > 1
            norm = 0.5 * cfg.rho_infty * cfg.uo ** 2 * (2.0 * cfg.r_c)
            vals.append(float(fd[len(fd) // 2:].mean() / norm) if ok else float("nan"))
        cd[prec] = np.array(vals)
        b.close()
    good = np.isfinite(cd[64]) & np.isfinite(cd[32])
    rel = np.full(len(cfgs), np.nan)
    rel[good] = np.abs(cd[32][good] - cd[64][good]) / np.abs(cd[64][good])
    worst = int(np.nanargmax(rel))
    return {"cases": cases, "steps": steps, "compared_cases": int(good.sum()),
            "rel_err_Cd_max": float(np.nanmax(rel)), "rel_err_Cd_median": float(np.nanmedian(rel)),
            "cases_above_1e-3": int(np.sum(rel[good] > 1e-3)),
            "worst_case": {"case": worst, "nx": cfgs[worst].nx, "ny": cfgs[worst].ny, "Re": round(cfgs[worst].Re, 2),
                           "Cd_fp64": float(cd[64][worst]), "Cd_fp32": float(cd[32][worst])},
            "Cd_fp64_range": [float(cd[64][good].min()), float(cd[64][good].max())]}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--seq-steps", type=int, default=2000)
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--trial-steps", type=int, default=50)
    ap.add_argument("--seed", type=int, default=4242)
    ap.add_argument("--no-sequential", action="store_true", help="skip the one-case-at-a-time baseline")
    ap.add_argument("--compare-fp64", type=int, default=0, metavar="STEPS",
                    help="instead of timing: FP32 against FP64 mean drag on every case over STEPS steps")
    a = ap.parse_args(argv)
    if a.compare_fp64 > 0:
        out = precision_check(a.cases, a.compare_fp64, a.seed)
        print(json.dumps(out), flush=True)
        return out
    out = sweep(a.cases, a.steps, a.seq_steps, a.precision, a.trial_steps, a.seed, not a.no_sequential)
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
