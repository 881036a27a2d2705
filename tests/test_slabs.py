"""A domain decomposed into z-slabs (hyqmom.slabs): the owned layers of
every slab equal the single-domain step bit for bit.

* world size 2 and 3 with the gloo backend on the CPU: each rank steps its
  slab with the oracle (the reference's serial step restated, split at the
  CFL reduction), the ranks exchange ghost layers and all-reduce the max
  wave speed through torch.distributed -- the same protocol code the GPU
  ranks run over NCCL;
* on one GPU: two and three slab contexts stepped in turn, the exchange and
  the reduction done between them on the device (no kernel waits on another).
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle_lib as ol
from hyqmom import ic, slabs


def crossing(Nz=12, nnmax=3):
    return ic.with_jets(ic.default_params(Nx=10, Ny=9, Nz=Nz, Ma=1.0, Kn=0.01, CFL=0.5, tmax=10.0, nnmax=nnmax), "crossing")


class OracleSlab:
    """A slab stepped by the oracle on the CPU (test engine)."""

    def __init__(self, p, nranks, rank):
        import torch
        self.torch = torch
        self.layout = slabs.local_layout(p["Nz"], nranks, rank)
        k0, k1, lo, hi = self.layout
        self.M = np.asfortranarray(ic.initial_state(p)[:, :, k0 - lo:k1 + hi, :])
        self.pp = dict(slabs.slab_params(p, nranks, rank), **ic.grid_spacing(p))
        self.t = 0.0
        self.Nx, self.Ny = p["Nx"], p["Ny"]

    def begin(self, pair):
        self.work, v = ol.step_begin(self.M, self.pp)
        pair.copy_(self.torch.tensor(slabs.vmax_pair(v), dtype=self.torch.float64))

    def end(self, pair):
        _, self.t = ol.step_end(self.work, self.M, slabs.vmax_from_pair(pair.tolist()), self.t)

    def get_layers(self, kl, nk):
        a = self.M[:, :, kl:kl + nk, :].reshape(-1, 35, order="F").T
        return self.torch.tensor(np.ascontiguousarray(a))

    def set_layers(self, kl, nk, buf):
        a = buf.numpy().T.reshape(self.Nx, self.Ny, nk, 35, order="F")
        self.M[:, :, kl:kl + nk, :] = a


def _rank(rank, world, port, nsteps, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = crossing()
        eng = OracleSlab(p, world, rank)
        for _ in range(nsteps):
            slabs.step(eng, rank, world, eng.layout, dist, lambda shape: torch.zeros(shape, dtype=torch.float64))
        k0, k1, lo, hi = eng.layout
        q.put((rank, k0, np.array(eng.M[:, :, lo:lo + (k1 - k0), :]), eng.t))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition():
    assert slabs.partition(12, 3) == [(0, 4), (4, 8), (8, 12)]
    assert slabs.partition(13, 3) == [(0, 5), (5, 9), (9, 13)]
    with pytest.raises(ValueError):
        slabs.partition(5, 3)
    assert slabs.local_layout(12, 3, 0) == (0, 4, 0, 2)
    assert slabs.local_layout(12, 3, 1) == (4, 8, 2, 2)
    assert slabs.vmax_from_pair(slabs.vmax_pair(float("nan"))) != slabs.vmax_from_pair(slabs.vmax_pair(float("nan")))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_slabs_equal_single_domain(world):
    nsteps = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nsteps, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    got = [q.get(timeout=600) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    p = crossing()
    M = np.asfortranarray(ic.initial_state(p))
    pp = dict(p, **ic.grid_spacing(p))
    t = 0.0
    for _ in range(nsteps):
        _, t, _ = ol.step(M, pp, t)
    for rank, k0, own, tr in got:
        assert tr == t
        assert np.array_equal(own, M[:, :, k0:k0 + own.shape[2], :]), rank


def _rank_leaves(rank, world, port, q):
    """Rank 1 steps once and leaves (between steps, nothing in flight); rank
    0 goes on and its next collective must end with an error, not hang."""
    import datetime
    import time
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    p = crossing()
    eng = OracleSlab(p, world, rank)
    buf = lambda shape: torch.zeros(shape, dtype=torch.float64)  # noqa: E731
    slabs.step(eng, rank, world, eng.layout, dist, buf)
    def put(x):  # flushed before the process ends without clean-up
        q.put(x)
        q.close()
        q.join_thread()

    if rank == 1:
        put((rank, "left"))
        os._exit(0)
    t0 = time.time()
    try:
        slabs.step(eng, rank, world, eng.layout, dist, buf)
        put((rank, "no error"))
    except Exception as e:  # the gloo timeout or the closed connection
        put((rank, f"error after {time.time() - t0:.1f} s: {type(e).__name__}"))
    os._exit(0)


def test_a_rank_that_leaves_ends_the_next_step_with_an_error():
    """Failure detection on the host: a slab rank that exits between steps
    makes the other rank's next step raise within the process group's
    timeout instead of waiting for ever (no GPU involved)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_leaves, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for pr in procs:
        pr.join(timeout=60)
    print(got)
    assert got[1] == "left"
    assert got[0].startswith("error after"), got[0]
    assert float(got[0].split()[2]) < 60.0


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs", [2, 3])
def test_gpu_slabs_equal_single_domain(nslabs):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hyqmom.runner import Solver
    p = crossing(Nz=12, nnmax=20)
    nsteps = 6
    engines = [slabs.GpuSlab(p, nslabs, r) for r in range(nslabs)]
    try:
        for e in engines:
            e.set_initial_condition()
        for _ in range(nsteps):
            pairs = [torch.zeros(2, dtype=torch.float64, device="cuda") for _ in engines]
            for e, pr in zip(engines, pairs):
                e.begin(pr)
            g = torch.stack(pairs).max(dim=0).values
            for e in engines:
                e.end(g)
            # ghost exchange between neighbouring slabs (as slabs.step does
            # between ranks)
            for r in range(nslabs - 1):
                a, b = engines[r], engines[r + 1]
                k0a, k1a, loa, hia = a.layout
                k0b, k1b, lob, hib = b.layout
                up = a.get_layers(loa + (k1a - k0a) - slabs.GHOST, slabs.GHOST)
                down = b.get_layers(lob, slabs.GHOST)
                b.set_layers(0, slabs.GHOST, up)
                a.set_layers(loa + (k1a - k0a), slabs.GHOST, down)
        owned = [e.owned_state() for e in engines]
        stats = [e.stats() for e in engines]
    finally:
        for e in engines:
            e.close()
    s = Solver(p)
    try:
        s.set_state_ic()
        s.advance(nsteps)
        M, st = s.get_state(), s.stats()
    finally:
        s.close()
    k = 0
    for o, sti in zip(owned, stats):
        assert np.array_equal(o, M[:, :, k:k + o.shape[2], :])
        assert sti["t"] == st["t"] and sti["nn"] == nsteps
        k += o.shape[2]
    assert k == p["Nz"]
