"""One periodic field split over ranks along y, one slab per rank.

The reference decomposes its field over MPI ranks (procDim, Main.cpp:21-30;
segment(), FlowField.cpp:278-288), gives every rank its padded block of
nc_seg + 6 cells per direction and refreshes the three ghost layers with
HaloTransfer before each step (update.cpp:894-1054).  Here the split is along
y only (procDim = {P, 1, 1}): x and z stay periodic inside each slab, so the
halo is the y exchange alone -- three planes of the five components to each of
the two neighbours, sent from the library's halo buffers with NCCL
send/receive (``torch.distributed``, one process per GPU), or with a device
copy when all slabs live in one process.  As in the reference's Evolve loop
(update.cpp:106-108, 130-146), the halo is exchanged once after the upload and
after every step, so the ghost planes are current whenever the diagnostics or
the next step read them.  The time step is the minimum over
ranks, and the diagnostics merge every rank's part (gks_stats_reduce), as the
reference's MPI_Allreduce / MPI_Reduce do (update.cpp:714-762, 1057-1079).
"""

from __future__ import annotations

import numpy as np

import gks_b200 as gks


def slab_planes(nc: int, nranks: int, rank: int) -> tuple:
    """(ny, y0): interior planes and first global plane of `rank`'s slab
    (segment(): sta[0] = procId * nc_segy)."""
    if nranks < 1 or nc % nranks:
        raise ValueError(f"{nc} planes do not split evenly over {nranks} ranks")
    ny = nc // nranks
    if ny < 3:
        raise ValueError(f"slabs of {ny} planes cannot hold the 3-plane halo")
    return ny, rank * ny


def split_block(W: np.ndarray, nranks: int, rank: int) -> np.ndarray:
    """The padded block of `rank`'s slab cut from the whole field's padded block
    W (5, nt, nt, nt) (ghosts included): its planes y0 .. y0 + ny + 5
    (segmentFill, FlowField.cpp:290-303)."""
    nc = W.shape[1] - 6
    ny, y0 = slab_planes(nc, nranks, rank)
    return np.ascontiguousarray(W[:, y0:y0 + ny + 6])


def merge_blocks(blocks) -> np.ndarray:
    """The whole field's padded block from every rank's slab block (rank
    order): interior planes from their owners, y ghosts as the periodic image."""
    nranks = len(blocks)
    nt = blocks[0].shape[2]
    nc = nt - 6
    W = np.empty((5, nt, nt, nt))
    for r, b in enumerate(blocks):
        ny, y0 = slab_planes(nc, nranks, r)
        W[:, 3 + y0:3 + y0 + ny] = b[:, 3:3 + ny]
    W[:, :3] = W[:, nc:nc + 3]
    W[:, nc + 3:] = W[:, 3:6]
    return W


def exchange_halo(bufs, rank: int, nranks: int, group=None):
    """The y exchange of HaloTransfer (update.cpp:899-954) on the four halo
    buffers of a slab as torch tensors (send south, send north, receive south,
    receive north): the south planes go to the south neighbour (rank - 1),
    whose north ghosts they fill, the north planes to rank + 1; the ring is
    periodic.  NCCL for CUDA tensors, gloo for CPU tensors; one rank copies in
    place."""
    send_s, send_n, recv_s, recv_n = bufs
    if nranks == 1:
        recv_n.copy_(send_s)
        recv_s.copy_(send_n)
        return
    import torch.distributed as dist

    south, north = (rank - 1) % nranks, (rank + 1) % nranks
    # to one peer, the sends and receives match in the order they are posted:
    # every rank posts (south planes, north planes) and receives (north ghosts,
    # south ghosts), so with two ranks (south == north) they still pair up
    ops = [dist.P2POp(dist.isend, send_s, south, group), dist.P2POp(dist.irecv, recv_n, north, group),
           dist.P2POp(dist.isend, send_n, north, group), dist.P2POp(dist.irecv, recv_s, south, group)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()


def min_over_ranks(x: float, device, group=None) -> float:
    """The smallest of every rank's x (the field's dt from the slabs' dts:
    MPI_Allreduce of the maximum wave speed in the reference)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


def gather_parts(part: np.ndarray, device, group=None) -> np.ndarray:
    """Every rank's statistics part (gks_stats_part), in rank order, on every rank."""
    import torch
    import torch.distributed as dist

    t = torch.from_numpy(np.ascontiguousarray(part, dtype=np.float64)).to(device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(parts, t, group=group)
    return torch.stack(parts).cpu().numpy()


class _DeviceArray:
    """A device allocation of the library as a 1-D float64 array for torch."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def halo_tensors(solver: "gks.Solver", device):
    """The slab's four halo buffers as torch tensors sharing its device memory."""
    import torch

    ptrs, n = solver.halo_buffers()
    return [torch.as_tensor(_DeviceArray(p, n), device=device) for p in ptrs]


class SlabField:
    """This rank's slab of a periodic field split over the ranks of `group`
    along y (torch.distributed initialised, NCCL, one GPU per rank).  The
    library and the exchange share one stream, so the steps and the NCCL halo
    exchange are ordered on the GPU without host synchronisation."""

    def __init__(self, phys: "gks.Phys", precision: int = gks.FP64, flags: int = 0, group=None):
        import torch
        import torch.distributed as dist

        self.group = group
        self.rank = dist.get_rank(group)
        self.nranks = dist.get_world_size(group)
        self.phys = phys
        self.ny, self.y0 = slab_planes(phys.nc, self.nranks, self.rank)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.device)
        self.solver = gks.Solver(phys, precision, flags, device=self.device.index, slab=(self.ny, self.y0))
        self.solver.set_stream(self.stream.cuda_stream)
        self.bufs = halo_tensors(self.solver, self.device)

    def close(self):
        self.solver.close()

    def upload(self, block: np.ndarray):
        """This rank's padded slab block (5, ny + 6, nt, nt) (split_block);
        its y ghosts are then exchanged."""
        self.solver.upload(block)
        self.exchange()

    def download(self) -> np.ndarray:
        return self.solver.download()

    def exchange(self):
        import torch

        self.solver.halo_pack()
        with torch.cuda.stream(self.stream):
            exchange_halo(self.bufs, self.rank, self.nranks, self.group)
        self.solver.halo_unpack()

    def timestep(self, cfl: float) -> float:
        """dt of the whole field: the minimum of the slabs' (update.cpp:1057-1079
        with the maximum wave speed taken over every rank)."""
        import torch

        with torch.cuda.stream(self.stream):
            dt = min_over_ranks(self.solver.timestep(cfl), self.device, self.group)
        self.solver.set_dt(dt)
        return dt

    def step(self, nsteps: int = 1):
        """nsteps steps, each followed by the halo exchange."""
        for _ in range(nsteps):
            self.solver.step(1)
            self.exchange()

    def sync(self):
        self.solver.sync()

    def stats(self) -> dict:
        """The whole field's diagnostics on every rank (parts merged in rank order)."""
        import torch

        with torch.cuda.stream(self.stream):
            parts = gather_parts(self.solver.stats_part(), self.device, self.group)
        return gks.stats_reduce(parts, self.phys)


class LocalSlabs:
    """Every slab of one field in this process, on the current GPU: the
    exchange is a device copy between the slabs' halo buffers.  The same
    library calls and data movement as SlabField on P ranks, without a
    process group (a single-GPU run of the decomposition, and its test)."""

    def __init__(self, phys: "gks.Phys", nranks: int, precision: int = gks.FP64, flags: int = 0):
        import torch

        self.phys = phys
        self.nranks = nranks
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.Stream(device=self.device)
        self.solvers = []
        for r in range(nranks):
            s = gks.Solver(phys, precision, flags, slab=slab_planes(phys.nc, nranks, r))
            s.set_stream(self.stream.cuda_stream)
            self.solvers.append(s)
        self.bufs = [halo_tensors(s, self.device) for s in self.solvers]

    def close(self):
        for s in self.solvers:
            s.close()

    def upload(self, W: np.ndarray):
        """The whole field's padded block (5, nt, nt, nt)."""
        for r, s in enumerate(self.solvers):
            s.upload(split_block(W, self.nranks, r))
        self.exchange()

    def download(self) -> np.ndarray:
        return merge_blocks([s.download() for s in self.solvers])

    def exchange(self):
        import torch

        for s in self.solvers:
            s.halo_pack()
        with torch.cuda.stream(self.stream):
            for r in range(self.nranks):
                south, north = (r - 1) % self.nranks, (r + 1) % self.nranks
                self.bufs[r][3].copy_(self.bufs[north][0])  # north ghosts <- the north slab's south planes
                self.bufs[r][2].copy_(self.bufs[south][1])  # south ghosts <- the south slab's north planes
        for s in self.solvers:
            s.halo_unpack()

    def timestep(self, cfl: float) -> float:
        dt = min(s.timestep(cfl) for s in self.solvers)
        for s in self.solvers:
            s.set_dt(dt)
        return dt

    def step(self, nsteps: int = 1):
        for _ in range(nsteps):
            for s in self.solvers:
                s.step(1)
            self.exchange()

    def sync(self):
        for s in self.solvers:
            s.sync()

    def stats(self) -> dict:
        return gks.stats_reduce(np.stack([s.stats_part() for s in self.solvers]), self.phys)
