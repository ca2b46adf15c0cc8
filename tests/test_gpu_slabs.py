"""x-slabs of one domain: stepped together with their halo exchange, each slab's populations
equal the matching columns of the single-domain run bit for bit, and the force records too."""
import numpy as np
import pytest

from cases import CASES
from mrlbm_2d_b200.slabs import cylinder_columns, partition

pytestmark = pytest.mark.gpu


def _single(mrlbm, cfg, prec, steps):
    s = mrlbm.Simulation(cfg, precision=prec)
    s.step(steps)
    out = (s.get_state(), s.forces())
    s.close()
    return out


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("parts,tiles", [(2, (1, 1)), (3, (18, 27, 22)), (4, (3, 16, 10, 0))])
def test_slabs_match_single_domain(mrlbm, prec, parts, tiles):
    cfg = CASES["benchmark_small_400x100"]()
    bounds = partition(400, parts, cylinder_columns(cfg))
    sims = [mrlbm.Simulation(cfg, precision=prec, slab=b) for b in bounds]
    for s, t in zip(sims, tiles):
        try:
            s.tile_config = t
        except mrlbm.MrlbmError:
            pass
    mrlbm.slabs_step(sims, 17)
    mrlbm.slabs_step(sims, 23)
    f_ref, (it, fd, fl, rin) = _single(mrlbm, cfg, prec, 40)
    f = np.concatenate([s.get_state() for s in sims], axis=0)
    assert f.shape == f_ref.shape
    assert np.array_equal(f, f_ref)
    recs = [s.forces() for s in sims]
    for r in recs:
        assert np.array_equal(r[0], it)
    assert np.array_equal(sum(r[1] for r in recs), fd) and np.array_equal(sum(r[2] for r in recs), fl)
    assert np.array_equal(sum(r[3] for r in recs), rin)
    for s in sims:
        assert s.status() == 0
        s.close()


def test_halo_pack_unpack_exchange_in_torch_buffers(mrlbm):
    """The rank-to-rank path without the transport: pack each face into a torch tensor, hand it
    to the neighbour, unpack; same bits as the single-domain run."""
    import torch
    cfg = CASES["freeslip_label15"]()
    bounds = partition(cfg.nx, 2, cylinder_columns(cfg))
    stream = torch.cuda.Stream()
    sims = [mrlbm.Simulation(cfg, precision=64, slab=b) for b in bounds]
    for s in sims:
        s.set_stream(stream.cuda_stream)
    n, e = sims[0].halo_size()
    assert n == 3 * cfg.ny and e == 8
    buf = {(r, side): torch.empty(n, dtype=torch.float64, device="cuda") for r in range(2) for side in range(2)}
    with torch.cuda.stream(stream):
        for _ in range(30):
            for s in sims:
                s.step(1)
            sims[0].halo_pack(1, buf[(0, 1)].data_ptr())
            sims[1].halo_pack(0, buf[(1, 0)].data_ptr())
            sims[1].halo_unpack(0, buf[(0, 1)].data_ptr())
            sims[0].halo_unpack(1, buf[(1, 0)].data_ptr())
    torch.cuda.synchronize()
    f_ref, _ = _single(mrlbm, cfg, 64, 30)
    f = np.concatenate([s.get_state() for s in sims], axis=0)
    assert np.array_equal(f, f_ref)
    for s in sims:
        s.close()


@pytest.mark.parametrize("prec", [64, 32])
def test_faces_first_exchange_overlapping_the_step(mrlbm, prec):
    """The overlapped order through torch buffers: face kernels, then on a second stream the
    faces of the next level packed and unpacked into the neighbour's next level, while the
    step kernels run on the first stream.  Same bits as the single-domain run."""
    import torch
    cfg = CASES["benchmark_small_400x100"]()
    bounds = partition(cfg.nx, 2, cylinder_columns(cfg))
    main, side = torch.cuda.Stream(), torch.cuda.Stream()
    sims = [mrlbm.Simulation(cfg, precision=prec, slab=b) for b in bounds]
    for s in sims:
        s.set_stream(main.cuda_stream)
    n, e = sims[0].halo_size()
    dt = torch.float64 if e == 8 else torch.float32
    buf = {(r, side_): torch.empty(n, dtype=dt, device="cuda") for r in range(2) for side_ in range(2)}
    for _ in range(30):
        for s in sims:
            s.step_faces()
        side.wait_stream(main)
        for s in sims:
            s.set_stream(side.cuda_stream)
        sims[0].halo_pack_next(1, buf[(0, 1)].data_ptr())
        sims[1].halo_pack_next(0, buf[(1, 0)].data_ptr())
        sims[1].halo_unpack_next(0, buf[(0, 1)].data_ptr())
        sims[0].halo_unpack_next(1, buf[(1, 0)].data_ptr())
        for s in sims:
            s.set_stream(main.cuda_stream)
            s.step(1)
        main.wait_stream(side)
    torch.cuda.synchronize()
    f_ref, _ = _single(mrlbm, cfg, prec, 30)
    f = np.concatenate([s.get_state() for s in sims], axis=0)
    assert np.array_equal(f, f_ref)
    for s in sims:
        assert s.status() == 0
        s.close()


def test_step_faces_is_a_no_op_without_halo(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    s = mrlbm.Simulation(cfg, precision=64)
    f0, it0 = s.get_state(), s.iter
    s.step_faces()
    assert np.array_equal(s.get_state(), f0) and s.iter == it0
    s.close()


def test_slab_cutting_the_cylinder_is_rejected(mrlbm):
    cfg = CASES["benchmark_small_400x100"]()
    lo, hi = cylinder_columns(cfg)
    with pytest.raises(mrlbm.MrlbmError) as e:
        mrlbm.Simulation(cfg, slab=(1, (lo + hi) // 2))
    assert e.value.code == 3


RANK_WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import datetime
import numpy as np
import torch, torch.distributed as dist
from cases import CASES
from mrlbm_2d_b200.slabs import DistributedSlabRun
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
torch.cuda.set_device(0)
run = DistributedSlabRun(CASES["benchmark_small_400x100"](), precision={prec}, device=0)
run.step(25)
it, fd, fl, rin = run.forces()
np.save(os.path.join({out!r}, "f%d.npy" % run.rank), run.sim.get_state())
if run.rank == 0:
    np.save(os.path.join({out!r}, "forces.npy"), np.stack([fd, fl, rin]))
print(json.dumps({{"rank": run.rank, "bounds": run.bounds[run.rank], "status": run.sim.status()}}), flush=True)
run.close()
dist.destroy_process_group()
"""


@pytest.mark.parametrize("prec", [64, 32])
def test_distributed_slab_run_two_ranks_on_one_gpu(mrlbm, prec, tmp_path):
    """DistributedSlabRun end to end: two processes, one slab each, sharing the GPU, with the
    faces swapped over a gloo group through pinned host buffers (the kernels of the two ranks
    never wait on each other; the host does).  Same bits as the single-domain run."""
    import json
    import os
    from test_cpu_multirank import _launch
    here = os.path.dirname(os.path.abspath(__file__))
    code = RANK_WORKER.format(root=os.path.dirname(here), tests=here, prec=prec, out=str(tmp_path))
    outs = _launch(code, world=2, timeout=300)
    recs = sorted((json.loads(o.strip().splitlines()[-1]) for o in outs), key=lambda r: r["rank"])
    assert [r["status"] for r in recs] == [0, 0]
    f = np.concatenate([np.load(tmp_path / f"f{r}.npy") for r in range(2)], axis=0)
    f_ref, (it, fd, fl, rin) = _single(mrlbm, CASES["benchmark_small_400x100"](), prec, 25)
    assert np.array_equal(f, f_ref)
    got = np.load(tmp_path / "forces.npy")
    assert np.array_equal(got[0], fd) and np.array_equal(got[1], fl) and np.array_equal(got[2], rin)
