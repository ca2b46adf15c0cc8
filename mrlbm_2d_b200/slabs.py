"""One domain split into x-slabs: the column partition, and the halo exchange of one slab per
rank over torch.distributed.

The step of a slab is the single-domain step restricted to its columns (mrlbm_create_slab);
after every step each slab sends the populations that cross its faces (3 x ny values per face)
to its neighbours, which is the one exchange the decomposition needs.  Within one process,
`mrlbm_2d_b200.slabs_step` does this with device-to-device copies; across processes (one GPU
per rank) `SlabExchange` packs the faces into tensors, swaps them with the neighbouring ranks
(NCCL send/recv on GPUs; gloo through pinned host buffers where several ranks share one GPU,
and on CPU for the host-logic tests) and unpacks them.

    run = DistributedSlabRun(cfg, precision=FP32)        # under torchrun, one rank per GPU
    run.step(1000)
    it, fd, fl, rin = run.forces()                        # summed over ranks (one has the cylinder)
"""
import numpy as np

from . import api


def cylinder_columns(cfg):
    """Global columns the cylinder, its wall nodes and their bilinear stencils occupy (a host-
    only handle builds the geometry); None without a cylinder."""
    s = api.Simulation(cfg, precision=api.FP64, device=-1)
    try:
        if s.nbct == 0:
            return None
        nodes = s.boundary_nodes()
        cols = [int(v) for v in nodes["bou_i"]]
        st = nodes["stencil"]                         # per node: i_p2(4), j_p2(4), i_p3, j_p3, i_p4, j_p4
        cols += [int(v) for v in st[:, [0, 1, 2, 3, 8, 9, 10, 11, 16, 17, 18, 19]].ravel()]
        solid = np.nonzero(s.node_classes()["issolid"].any(axis=1))[0]
        if solid.size:
            cols += [int(solid.min()) + 1, int(solid.max()) + 1]
        return min(cols), max(cols)
    finally:
        s.close()


def partition(nx, parts, keep=None, min_width=4):
    """Split columns 1..nx into `parts` adjacent slabs of nearly equal width; a boundary that would
    cut the column range `keep` (with one column of margin) moves just outside it."""
    if parts < 1 or nx < parts * min_width:
        raise ValueError("too many slabs for the domain")
    edges = [1 + (nx * p) // parts for p in range(parts + 1)]
    edges[-1] = nx + 1
    if keep is not None:
        lo, hi = keep[0] - 1, keep[1] + 1
        for p in range(1, parts):
            if lo <= edges[p] <= hi + 1:
                left, right = lo, hi + 1
                edges[p] = left if abs(edges[p] - left) <= abs(right - edges[p]) else right
    for p in range(parts):
        if edges[p + 1] - edges[p] < min_width:
            raise ValueError("cannot partition around the cylinder with this many slabs")
    return [(edges[p], edges[p + 1] - 1) for p in range(parts)]


def _host_transport(group):
    import torch.distributed as dist
    return dist.get_backend(group) == "gloo"


class SlabExchange:
    """Halo swap of one slab with its left and right neighbours (ranks rank-1, rank+1) over
    torch.distributed.  pack(side, tensor) / unpack(side, tensor) move a face between the
    slab's state and a flat tensor of n_values elements (side 0 left, 1 right).

    With NCCL the faces travel device to device.  A gloo group moves host tensors only, so
    device faces are staged through pinned host buffers (one copy each way per face)."""

    def __init__(self, rank, world, pack, unpack, n_values, dtype, device, group=None):
        import torch
        self.rank, self.world = rank, world
        self.left = rank - 1 if rank > 0 else None
        self.right = rank + 1 if rank + 1 < world else None
        self.pack, self.unpack = pack, unpack
        self.group = group
        device = torch.device(device)
        mk = lambda: torch.empty(n_values, dtype=dtype, device=device)
        self.send = {0: mk(), 1: mk()}
        self.recv = {0: mk(), 1: mk()}
        self.staged = device.type == "cuda" and _host_transport(group)
        if self.staged:
            mh = lambda: torch.empty(n_values, dtype=dtype, pin_memory=True)
            self.send_h = {0: mh(), 1: mh()}
            self.recv_h = {0: mh(), 1: mh()}

    def exchange(self):
        import torch
        import torch.distributed as dist
        sides = [(side, peer) for side, peer in ((0, self.left), (1, self.right)) if peer is not None]
        for side, _ in sides:
            self.pack(side, self.send[side])
        send, recv = self.send, self.recv
        if self.staged:
            for side, _ in sides:
                self.send_h[side].copy_(self.send[side])      # ordered after the pack on this stream
            torch.cuda.current_stream().synchronize()
            send, recv = self.send_h, self.recv_h
        ops = []
        for side, peer in sides:
            ops.append(dist.P2POp(dist.isend, send[side], peer, self.group))
            ops.append(dist.P2POp(dist.irecv, recv[side], peer, self.group))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for side, _ in sides:
            if self.staged:
                self.recv[side].copy_(self.recv_h[side])
            self.unpack(side, self.recv[side])


class DistributedSlabRun:
    """One x-slab of `cfg` per rank (torch.distributed initialised, one GPU per rank).

    Each step overlaps the exchange with the step: the face kernel writes the halo-face
    columns of the next level, a second stream sends them (and receives the neighbours') while
    the step kernel computes the whole slab, and the next step waits for that stream."""

    def __init__(self, cfg, precision=api.FP32, bounds=None, device=None):
        import torch
        import torch.distributed as dist
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        dev = torch.cuda.current_device() if device is None else device
        if bounds is None:
            info = api.Simulation(cfg, precision=api.FP64, device=-1)
            nx = info.nx
            info.close()
            bounds = partition(nx, self.world, cylinder_columns(cfg))
        self.bounds = bounds
        self.sim = api.Simulation(cfg, precision=precision, device=dev, slab=bounds[self.rank])
        self.stream = torch.cuda.current_stream(dev)
        self.side = torch.cuda.Stream(dev)
        self.sim.set_stream(self.stream.cuda_stream)
        n, e = self.sim.halo_size()
        dtype = torch.float64 if e == 8 else torch.float32
        # the side stream packs and unpacks: point the handle at it around those copies
        def on_side(fn):
            def run(side, t):
                self.sim.set_stream(self.side.cuda_stream)
                try:
                    fn(side, t.data_ptr())
                finally:
                    self.sim.set_stream(self.stream.cuda_stream)
            return run
        self.ex = SlabExchange(self.rank, self.world, on_side(self.sim.halo_pack_next),
                               on_side(self.sim.halo_unpack_next), n, dtype, torch.device("cuda", dev))

    def step(self, n=1):
        import torch
        for _ in range(int(n)):
            self.sim.step_faces()
            self.side.wait_stream(self.stream)            # faces written; previous step done
            with torch.cuda.stream(self.side):
                self.ex.exchange()
            self.sim.step(1)
            self.stream.wait_stream(self.side)            # ghost columns in before the next step

    def forces(self):
        """Force history summed over the slabs (iter, F_drag, F_lift, sum rho(1,:))."""
        import torch
        import torch.distributed as dist
        it, fd, fl, rin = self.sim.forces()
        dev = "cpu" if _host_transport(None) else "cuda"
        t = torch.tensor(np.stack([fd, fl, rin]), dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        a = t.cpu().numpy()
        return it, a[0], a[1], a[2]

    def close(self):
        self.sim.close()
