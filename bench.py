"""Benchmark of the moment-regularized D2Q9 cylinder step (one JSON line on rank 0).

Workload: the 2048 x 512 cylinder case (D = 80 at (320.0, 256.5), Re = 200, U = 0.04,
free-slip walls, seeded-noise start); one bench step = one lattice time step over the whole
grid, forces reduced every step.  Synthetic, seeded inputs only.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--precision 32|64] [--case mid|large|small] [--no-studies]

`value` is the aggregate MLUPS of the headline precision, FP64 (the reference's arithmetic;
--precision 32 selects the FP32 deviation form), each timed step preceded by an L2 flush
outside its CUDA event pair (a 256 MiB write, then a read of the same buffer, so L2 holds none
of the state and the flush's own dirty lines are written back before the step starts); the
FP32 form is timed the same way beside it (`fp32`).  `e2e` is the same metric through the
public C ABI with host buffers, as a restart segment: upload the populations, max(K, 1000)
steps, drain the force history every 100 steps, read the last step's rho/ux/uy back.  The
rest of the benchmark metric is measured in the same run: `precision` (FP32 against FP64 on
the 2048 x 512 case over 100,000 steps: Cd, Cl_rms, St, velocity field), `precision_large`
(16384 x 4096 with FP64 mean/rms field statistics), `adjoint` (gradient of mean drag on
512 x 128: cost over the forward run and the check against central differences) and `batch`
(the 64-case sweep against the same cases stepped one after another).  Under torchrun every
rank runs an independent replica (its own seed) on its own GPU: weak scaling, no collective on
the data path; times are max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_LU = {64: 144, 32: 72}       # one read + one write of 9 populations
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", type=int, choices=[32, 64], default=None)
    ap.add_argument("--case", choices=["mid", "large", "small", "quarter"], default="mid")
    ap.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    ap.add_argument("--soak-seconds", type=float, default=1.0,
                    help="untimed steps before each timed run, so the clock samples see the steady state")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tile", type=int, default=None,
                    help="bulk tile shape (default: chosen by the autotuner before timing)")
    ap.add_argument("--large-steps", type=int, default=30,
                    help="timed steps of the 16384 x 4096 roofline case at N=1 (0: skip)")
    ap.add_argument("--fields", action="store_true",
                    help="with --profile: accumulate the FP64 field statistics in every step")
    ap.add_argument("--profile", action="store_true",
                    help="only run warmup + steps of the case (for ncu); prints nothing else")
    ap.add_argument("--e2e-steps", type=int, default=1000,
                    help="steps of the end-to-end restart segment (at least --steps)")
    ap.add_argument("--no-studies", action="store_true",
                    help="skip the precision, adjoint and batch blocks")
    ap.add_argument("--precision-steps", type=int, default=100000,
                    help="steps of the FP32-vs-FP64 study on the 2048 x 512 case")
    ap.add_argument("--large-precision-steps", type=int, default=2000,
                    help="steps of the FP32-vs-FP64 study with field statistics on 16384 x 4096 (0: skip)")
    ap.add_argument("--adjoint-directions", type=int, default=16)
    ap.add_argument("--batch-steps", type=int, default=2000)
    ap.add_argument("--batch-seq-steps", type=int, default=200)
    ap.add_argument("--batch-precision-steps", type=int, default=40000,
                    help="FP32 against FP64 mean drag on every sweep case over this many steps (0: skip)")
    ap.add_argument("--decomp", choices=["replicas", "slabs"], default="replicas",
                    help="replicas: one independent case per rank (weak scaling); slabs: the 16384 x 4096 "
                         "case split into x-slabs across the ranks with the halo exchange (strong scaling)")
    return ap.parse_args()


class RankGroup:
    """One process per GPU (torchrun env: RANK, WORLD_SIZE, LOCAL_RANK, MASTER_*): the
    barrier and max-over-ranks reductions the timing needs; no collective touches the data
    path (every rank advances its own replica).  backend "nccl" on GPUs, "gloo" on CPU."""

    def __init__(self, backend="nccl"):
        import datetime
        import torch
        import torch.distributed as dist
        self.dist, self.torch = dist, torch
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = torch.device("cuda", self.local) if backend == "nccl" else torch.device("cpu")
        if self.world > 1:
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return float(x)
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def replica_seed(rank):
    """Each rank's replica is the same case with its own noise seed."""
    return 1234 + rank


def make_case(name, seed):
    from mrlbm_2d_b200.config import case_large, case_mid, case_quarter, case_small
    c = {"mid": case_mid, "large": case_large, "small": case_small, "quarter": case_quarter}[name]()
    return c.replace(seed=seed)


def case_desc(name, cfg):
    return {"workload": f"cylinder {name}: {cfg.nx}x{cfg.ny}, D={2 * cfg.r_c:g} at ({cfg.x_c:g},{cfg.y_c:g}), "
                        f"Re={cfg.Re:g}, U={cfg.uo:g}, free-slip walls, zero-gradient outlet, seeded noise",
            "nx": cfg.nx, "ny": cfg.ny, "nodes": cfg.nx * cfg.ny}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 100 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        sm, mx, reasons = [], None, set()
        for t, line in self.lines:
            if t < t0 or t > t1:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_from_profiles(precision, case_name):
    """DRAM bytes per lattice update of the step kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "step_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d.get(f"fp{precision}")
        return float(e["dram_bytes_per_lu"]), e.get("source", "profiles/step_traffic.json")
    except Exception:
        return None, None


def cpu_baseline(case_name, seconds, threads=None):
    """The oracle (reference restatement, OpenMP loops, serial streaming) on the host cores:
    a bounded sample of the same workload, wall-clock MLUPS."""
    import oracle
    cfg = make_case(case_name, 1234)
    n = threads or os.cpu_count() or 1
    oracle.set_threads(n)
    o = oracle.Oracle(cfg.replace(num_threads=n), threads=n)
    o.step(2)                                   # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        o.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 100000:
            break
    nodes = cfg.nx * cfg.ny
    o.close()
    return {"value": nodes * steps / el / 1e6, "unit": "MLUPS", "cores": n, "kind": "port",
            "sample": f"{steps} steps of the {cfg.nx}x{cfg.ny} case ({el:.1f} s wall clock, "
                      f"FP64 C++ restatement of 2d_mrlbm.f90 with its OpenMP loops and serial streaming)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    import oracle
    cfg = make_case(args.case, 1234)
    n = os.cpu_count() or 1
    oracle.set_threads(n)
    o = oracle.Oracle(cfg.replace(num_threads=n), threads=n)
    o.step(min(args.warmup, 3))
    # bounded sample: the timed steps stop after ~90 s of host work whatever --steps asks
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        o.step(1)
        done += 1
        if time.perf_counter() - t0 > 90.0:
            break
    el = time.perf_counter() - t0
    nodes = cfg.nx * cfg.ny
    v = nodes * done / el / 1e6
    line = {"metric": "D2Q9 MLUPS", "value": v, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / done * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": case_desc(args.case, cfg), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": n, "kind": "port",
                             "sample": f"{done} timed steps of the full grid after {min(args.warmup, 3)} "
                                       f"warm-up (FP64 C++ restatement of 2d_mrlbm.f90, OpenMP loops, "
                                       f"serial streaming)"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_profile(args):
    """Minimal launch sequence for profilers: create the case, warmup + steps, nothing else."""
    from mrlbm_2d_b200 import build
    build.build()
    import mrlbm_2d_b200 as m
    cfg = make_case(args.case, 1234)
    sim = m.Simulation(cfg, precision=args.precision or 32)
    if args.tile is not None:
        sim.tile_config = args.tile
    if args.fields:
        sim.field_stats_window(1, 10 ** 9)
    sim.step(args.warmup)
    sim.step(args.steps)
    st = sim.status()
    sim.close()
    return 0 if st == 0 else 1


def run_slabs(args):
    """Strong scaling of one large case: the 16384 x 4096 cylinder split into x-slabs, one per
    rank, with the halo exchange after every step (NCCL send/recv between neighbours, overlapped
    with the step).  At one rank it is the single-domain step.  The state (4.8 GB FP32, 9.7 GB
    FP64 over all ranks) is far above the L2, so steps run back to back without a flush."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = RankGroup("nccl")
    rank, world = ranks.rank, ranks.world
    from mrlbm_2d_b200 import build
    if rank == 0:
        build.build()
    ranks.barrier()
    import mrlbm_2d_b200 as m
    from mrlbm_2d_b200.slabs import DistributedSlabRun
    prec = args.precision or 64
    cfg = make_case("large", 1234)
    if world == 1:
        sim = m.Simulation(cfg, precision=prec)
        sim.set_stream(torch.cuda.current_stream().cuda_stream)
        tile, _ = sim.autotune(trial_steps=5)
        step, bounds = (lambda: sim.step(1)), [(1, cfg.nx)]
    else:
        run = DistributedSlabRun(cfg, precision=prec)
        tile, _ = run.sim.autotune(trial_steps=5)
        step, bounds = (lambda: run.step(1)), run.bounds
    for _ in range(args.warmup):
        step()
    ranks.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ranks.barrier()
    ms = ranks.max(e0.elapsed_time(e1)) / args.steps
    nodes = cfg.nx * cfg.ny
    peak, peak_kind = hbm_peak()
    line = {"metric": "D2Q9 MLUPS", "value": nodes / (ms * 1e-3) / 1e6, "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if prec == 32 else "f64",
            "data": "synthetic (seeded noise init)",
            "config": dict(case_desc("large", cfg), precision=f"fp{prec}", parallelism=f"xslabs{world}",
                           slabs=bounds, tile_shape=tile, l2="state far above the L2; steps back to back"),
            "hbm_gbs_alg_per_gpu": BYTES_PER_LU[prec] * nodes / world / (ms * 1e-3) / 1e9, "peak": peak,
            "peak_kind": peak_kind}
    if world > 1:
        run.close()
    else:
        sim.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    if args.decomp == "slabs":
        return run_slabs(args)

    import numpy as np
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    ranks = RankGroup("nccl")
    rank, world = ranks.rank, ranks.world

    from mrlbm_2d_b200 import build
    if rank == 0:
        build.build()
    ranks.barrier()
    import mrlbm_2d_b200 as m

    cfg = make_case(args.case, replica_seed(rank))
    nodes = cfg.nx * cfg.ny
    dev = torch.cuda.current_device()
    # one non-default stream carries the library's kernels, the L2 flush and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    flush_words = flush.view(torch.int64)

    def flush_l2():
        # 256 MiB (twice the L2) written, then read: every line of the state is evicted, and
        # the dirty lines the write leaves are cleaned here rather than inside the timed step
        flush.zero_()
        flush_words.sum()

    def barrier():
        ranks.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return ranks.max(x)

    def pick_tile(sim, flushed):
        if args.tile is not None:
            sim.tile_config = args.tile
            return args.tile
        best, _ = sim.autotune(trial_steps=10)
        if not flushed:
            return best
        # The library's autotuner times back-to-back steps, where several shapes are within
        # noise of each other; the timed protocol below flushes L2 before every step, which
        # separates them.  Re-time every shape under that protocol and keep the fastest.
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(8)]
        times = {}
        for t in range(m.N_TILE_CONFIGS):
            try:
                sim.tile_config = t
                sim.step(2)
            except m.MrlbmError:
                continue
            for a, b in ev:
                flush_l2()
                a.record(stream)
                sim.step(1)
                b.record(stream)
            torch.cuda.synchronize()
            times[t] = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        sim.forces()
        best = min(times, key=times.get) if times else best
        sim.tile_config = best
        return best

    def time_device(precision, K, W, case_cfg=None, soak_s=1.0, fields=False):
        c = case_cfg or cfg
        sim = m.Simulation(c, precision=precision, device=dev)
        sim.set_stream(stream.cuda_stream)
        if fields:                           # FP64 mean/rms sums of u, v, p in every step
            sim.field_stats_window(1, 2 ** 30)
        sim.step(W)
        tile = pick_tile(sim, flushed=case_cfg is None)
        # untimed soak so clock samples see the steady state
        t_soak, n_soak = time.time(), 0
        while time.time() - t_soak < soak_s and n_soak < 20000:
            sim.step(50)
            n_soak += 50
            torch.cuda.synchronize()
        sim.forces()
        launches0 = sim.launch_count()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
        barrier()
        t_wall0 = time.time()
        for s in range(K):
            flush_l2()
            starts[s].record(stream)
            sim.step(1)
            ends[s].record(stream)
        barrier()
        t_wall1 = time.time()
        launches = sim.launch_count() - launches0
        per = [a.elapsed_time(b) for a, b in zip(starts, ends)]
        total_ms = sum(per)
        # unflushed back-to-back steps (state may stay partly in L2), for reference
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sim.step(K)
        e1.record(stream)
        torch.cuda.synchronize()
        noflush_ms = e0.elapsed_time(e1) / K
        st = sim.status()
        _, fd, fl, _ = sim.forces()
        sim.close()
        assert st == 0, "device error flag set"
        assert np.all(np.isfinite(fd)), "non-finite forces"
        return total_ms, launches, per, noflush_ms, (t_wall0, t_wall1), tile

    def protocol_floor(nbytes, n=30):
        """What the flushed protocol costs around a kernel that does nothing, and around a plain
        device copy of the step's algorithmic bytes (half read, half written): the floor any step
        kernel of this size meets under the same protocol."""
        import statistics as st
        tiny = torch.zeros(1, device="cuda")
        src = torch.empty(nbytes // 2, dtype=torch.uint8, device="cuda")
        dst = torch.empty_like(src)
        out = {}
        for name, fn in (("empty_kernel_us", lambda: tiny.add_(1)), ("copy_us", lambda: dst.copy_(src))):
            ts = []
            for _ in range(n):
                flush_l2()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                ts.append((a, b))
            torch.cuda.synchronize()
            out[name] = st.median([a.elapsed_time(b) * 1e3 for a, b in ts])
        del src, dst
        return out

    def time_e2e(precision, K, tile):
        """Public-API restart segment with host buffers: load the state from pinned host
        memory, K steps, force history drained every 100 steps, rho/ux/uy of the last step
        read back into pinned buffers.  Wall clock, max over ranks."""
        sim = m.Simulation(cfg, precision=precision, device=dev)
        sim.set_stream(stream.cuda_stream)
        sim.tile_config = tile               # the autotuner's choice for this case (untimed setup)
        # pinned host buffers: the initial populations (Fortran order, FP64 as in restart.dat)
        f0 = torch.empty(nodes * 9, dtype=torch.float64).pin_memory().numpy()
        sim.get_state(out=f0)                # host copy of the seeded initial populations
        mac = [torch.empty(nodes, dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
        sim.step(2)
        sim.step(1, macro=True)              # untimed: the macroscopic buffer and that kernel's first use
        sim.forces()
        barrier()
        t0 = time.perf_counter()
        sim.load_state(f0, iter=0)
        nrec = 0
        for s0 in range(0, K, 100):
            n = min(100, K - s0)
            sim.step(n, macro=(s0 + n == K))
            nrec += len(sim.forces()[0])
        sim.macro(out=mac)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        el = max_over_ranks(el)
        sim.close()
        h2d = nodes * 9 * 8 / K
        d2h = (nrec * 4 * 8 + 3 * nodes * 8) / K
        del mac
        return {"value": world * nodes * K / el / 1e6, "unit": "MLUPS", "steps": K,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": f"restart segment through the C ABI: load_state (FP64 populations from pinned host "
                        f"memory) + {K} steps + force records drained every 100 steps + rho/ux/uy of the last "
                        f"step into pinned buffers; wall clock, max over ranks"}

    # FP64 (the reference's arithmetic) is the headline; the FP32 deviation form runs beside it
    precisions = [args.precision] if args.precision else ([64, 32] if _fp32_available(m, cfg) else [64])
    head = precisions[0]
    sampler = ClockSampler(local) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    results = {}
    for prec in precisions:
        total_ms, launches, per, noflush_ms, win, tile = time_device(prec, args.steps, args.warmup,
                                                                     soak_s=args.soak_seconds)
        total_ms = max_over_ranks(total_ms)
        results[prec] = (total_ms, launches, per, noflush_ms, win, tile)
    large = {}
    if world == 1 and args.large_steps > 0 and args.case != "large":
        lcfg = make_case("large", 1234)
        lnodes = lcfg.nx * lcfg.ny
        for prec in precisions:
            t, _, _, nf, lwin, ltile = time_device(prec, args.large_steps, 3, case_cfg=lcfg, soak_s=0.5)
            ms = t / args.large_steps
            large[prec] = {"ms_per_step": ms, "mlups": lnodes / (ms * 1e-3) / 1e6, "tile_shape": ltile,
                           "hbm_gbs_alg": BYTES_PER_LU[prec] * lnodes / (ms * 1e-3) / 1e9,
                           "ms_per_step_unflushed": nf, "window": lwin}
            # the same with the field statistics on: six FP64 running sums read and written per
            # node and step on top of the populations (+96 B per lattice update)
            t, _, _, nf, lwin, ltile = time_device(prec, args.large_steps, 3, case_cfg=lcfg, soak_s=0.3, fields=True)
            ms = t / args.large_steps
            bpl = BYTES_PER_LU[prec] + 96
            large[prec]["with_field_statistics"] = {
                "ms_per_step": ms, "mlups": lnodes / (ms * 1e-3) / 1e6, "tile_shape": ltile,
                "bytes_per_lu": bpl, "hbm_gbs_alg": bpl * lnodes / (ms * 1e-3) / 1e9,
                "ms_per_step_unflushed": nf, "window": lwin}
    floor = {}
    if world == 1:
        for prec in precisions:
            f = protocol_floor(BYTES_PER_LU[prec] * nodes)
            floor[prec] = {"empty_kernel_us": f["empty_kernel_us"], "copy_us": f["copy_us"],
                           "bytes": BYTES_PER_LU[prec] * nodes,
                           "copy_gbs": BYTES_PER_LU[prec] * nodes / (f["copy_us"] * 1e-6) / 1e9}
    if sampler:
        time.sleep(0.3)
        sampler.stop()
    e2e_steps = max(args.steps, args.e2e_steps)
    e2e = {prec: time_e2e(prec, e2e_steps, results[prec][5]) for prec in precisions}

    total_ms, launches, per, noflush_ms, win, tile = results[head]
    ms_step = total_ms / args.steps
    value = world * nodes * args.steps / (total_ms * 1e-3) / 1e6
    peak, peak_kind = hbm_peak()
    avg_launch_s = (total_ms / args.steps) * 1e-3
    achieved = BYTES_PER_LU[head] * nodes / avg_launch_s / 1e9
    tr, tr_src = traffic_from_profiles(head, args.case)
    line = {
        "metric": "D2Q9 MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if head == 32 else "f64", "data": "synthetic (seeded noise init)",
        "config": dict(case_desc(args.case, cfg), precision=f"fp{head}",
                       l2="flushed before every timed step (256 MiB written, then read)",
                       parallelism=f"replicas{world}", tile_shape=tile),
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (tr * nodes) if tr is not None else None,
                     "algorithmic_bytes_per_launch": BYTES_PER_LU[head] * nodes,
                     "traffic_source": tr_src},
        "e2e": e2e[head],
    }
    for prec in precisions:
        t, _, _, nf, _, tl = results[prec]
        gbs = BYTES_PER_LU[prec] * nodes / (t / args.steps * 1e-3) / 1e9
        line[f"fp{prec}"] = {"mlups": world * nodes * args.steps / (t * 1e-3) / 1e6, "ms_per_step": t / args.steps,
                             "tile_shape": tl, "ms_per_step_unflushed": nf, "hbm_gbs_alg": gbs,
                             "bytes_per_lu": BYTES_PER_LU[prec], "frac_of_peak": gbs / peak, "e2e": e2e[prec]}
    if 32 in results and 64 in results:
        line["fp32_over_fp64"] = results[64][0] / results[32][0]
    if floor:
        line["flushed_protocol"] = {
            "note": "the same flush-then-events protocol around an empty torch kernel and around a torch "
                    "device copy of each precision's algorithmic bytes per step: the floor a step of this "
                    "size meets (state under 2x the L2, so the flush is what makes it read HBM)",
            **{f"fp{p}": dict(v, copy_frac_of_peak=v["copy_gbs"] / peak) for p, v in floor.items()}}
    if large:
        lcfg = make_case("large", 1234)
        rl = {"workload": case_desc("large", lcfg)["workload"], "steps": args.large_steps,
              "l2": "flushed before every timed step, 256 MiB written then read (working set 4.8 GB FP32 / 9.7 GB FP64)", "peak": peak,
              "peak_kind": peak_kind, "unit": "GB/s", "bound": "hbm"}
        for prec, v in large.items():
            v = dict(v)
            v.pop("window")
            v["frac"] = v["hbm_gbs_alg"] / peak
            fs = dict(v.pop("with_field_statistics"))
            fs.pop("window")
            fs["frac"] = fs["hbm_gbs_alg"] / peak
            v["with_field_statistics"] = fs
            rl[f"fp{prec}"] = v
        if 32 in large and 64 in large:
            rl["fp32_over_fp64"] = large[64]["ms_per_step"] / large[32]["ms_per_step"]
        line["roofline_large"] = rl
    if sampler:
        wins = [r[4] for r in results.values()] + [v["window"] for v in large.values()] + \
               [v["with_field_statistics"]["window"] for v in large.values()]
        t0 = min(w[0] for w in wins) - 1.2
        t1 = max(w[1] for w in wins)
        line["clocks"] = sampler.summary(t0, t1)
    if world == 1 and not args.no_studies:
        line.update(run_studies(args, peak))
    ranks.barrier()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(args.case, args.cpu_sample_seconds)
        except Exception as ex:                 # reported, never fatal
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def run_studies(args, peak):
    """The rest of the benchmark metric, measured in the same run: FP32 against FP64 on the
    2048 x 512 case (and with field statistics on 16384 x 4096), the adjoint's cost and its check
    against central differences on 512 x 128, and the 64-case batched sweep with its FP32
    against FP64 mean drag per case."""
    out = {}
    from mrlbm_2d_b200 import adjoint_check, batch_sweep, precision_study
    t0 = time.perf_counter()
    try:
        p = precision_study.study("mid", args.precision_steps)
        keep = ("case", "nx", "ny", "steps", "stats_from", "rel_err_Cd", "abs_err_St_spectral",
                "rel_err_Cl_rms", "velocity_rel_l2", "velocity_max_abs_over_U", "drag_history_rel_l2")
        out["precision"] = {k: p[k] for k in keep if k in p}
        if "abs_err_St" in p:
            out["precision"]["abs_err_St_reference_method"] = p["abs_err_St"]
        out["precision"]["St_note"] = (
            "St_spectral: peak of the windowed lift spectrum over the statistics window; the reference's "
            "method (period between the first two local maxima of the raw lift, 2d_statistics.f90:191-212) "
            "is reported as St for each precision and is only meaningful once shedding has saturated")
        for prec in (64, 32):
            r = p[f"fp{prec}"]
            out["precision"][f"fp{prec}"] = {k: r[k] for k in ("Cd", "Cl_rms", "St", "St_spectral", "mlups_wall")
                                             if k in r}
        out["precision"]["targets"] = {"rel_err_Cd": 1e-3, "abs_err_St_spectral": 1e-3}
        out["precision"]["seconds"] = time.perf_counter() - t0
    except Exception as ex:
        out["precision"] = {"error": str(ex)}
    if args.large_precision_steps > 0:
        t0 = time.perf_counter()
        try:
            n = args.large_precision_steps
            p = precision_study.study("large", n, stats_from=n // 2, fields=True, chunk=n)
            keep = ("case", "nx", "ny", "steps", "stats_from", "rel_err_Cd", "velocity_rel_l2", "drag_history_rel_l2",
                    "mean_u_rel_l2", "mean_v_rel_l2", "mean_p_rel_l2", "rms_u_rel_l2", "rms_v_rel_l2", "rms_p_rel_l2",
                    "field_samples")
            out["precision_large"] = {k: p[k] for k in keep if k in p}
            out["precision_large"]["seconds"] = time.perf_counter() - t0
        except Exception as ex:
            out["precision_large"] = {"error": str(ex)}
    t0 = time.perf_counter()
    try:
        a = adjoint_check.check(directions=args.adjoint_directions)
        out["adjoint"] = {k: a[k] for k in ("case", "steps", "window", "checkpoint_every", "J", "directions",
                                            "rel_step", "max_rel_err", "median_rel_err", "forward_s", "gradient_s",
                                            "gradient_over_forward")}
        out["adjoint"]["targets"] = {"max_rel_err": 1e-3, "gradient_over_forward": 4.0}
        out["adjoint"]["seconds"] = time.perf_counter() - t0
    except Exception as ex:
        out["adjoint"] = {"error": str(ex)}
    t0 = time.perf_counter()
    try:
        b = batch_sweep.sweep(64, args.batch_steps, args.batch_seq_steps, 32, trial_steps=20)
        bb = b["batch"]
        gbs = BYTES_PER_LU[32] * bb["mlups"] * 1e6 / 1e9
        out["batch"] = {"cases": b["cases"], "nodes_total": b["nodes_total"], "steps": b["steps"],
                        "autotune": b["autotune"], "mlups": bb["mlups"], "ms_per_step": bb["ms_per_step"],
                        "hbm_gbs_alg": gbs, "frac_of_peak": gbs / peak, "bytes_per_lu": BYTES_PER_LU[32],
                        "sequential_mlups": b["sequential"]["mlups"], "speedup_vs_sequential": b["speedup"],
                        "unstable_cases": len(b["unstable_cases"]), "l2": "working set 554 MB (4.4x the L2), no flush"}
        if args.batch_precision_steps > 0:
            out["batch"]["precision"] = batch_sweep.precision_check(64, args.batch_precision_steps)
            out["batch"]["precision"]["targets"] = {"rel_err_Cd": 1e-3}
        out["batch"]["seconds"] = time.perf_counter() - t0
    except Exception as ex:
        out["batch"] = {"error": str(ex)}
    return out


def _fp32_available(m, cfg):
    try:
        s = m.Simulation(cfg.replace(nx=64, ny=32, x_c=20.0, y_c=16.5, r_c=4.0), precision=32)
        s.step(1)
        s.close()
        return True
    except Exception:
        return False


if __name__ == "__main__":
    sys.exit(main())
