"""One domain decomposed into z-slabs over ranks, one GPU per rank.

Replaces the rank-local parts of the reference's MPI step: the Cartesian
split (src/mpi/setup_mpi_cartesian_3d.jl:45-70), the halo exchange
(src/mpi/halo_exchange_3d.jl:26-122), the recomputed halo fluxes and speeds
(src/mpi/compute_halo_fluxes_and_wavespeeds_3d.jl:34-132) and the dt
all-reduce (src/simulation_runner.jl:403).

The split is along z (the slowest index of the moment-major layout, so a
slab and its boundary layers are contiguous blocks of every moment plane,
and each slab has at most two neighbours; Nz = 1 grids are not split).  Each
slab holds GHOST = 2 layers of its neighbours on each side that has one.
Per step:

1. phase [A] on every local layer, ghosts included.  The ghosts hold the
   neighbour's pre-step layers, so their closures, fluxes and speeds are the
   neighbour's own, bit for bit (the reference instead re-realizes the
   exchanged, already realized moments, which is why its multi-rank results
   differ from one rank's within its MPI tolerance, test/test_mpi.jl:35-36);
2. the max |speed| over the slabs (MAX all-reduce of {max over non-NaN,
   NaN flag}, so a NaN anywhere gives NaN as the serial code's `maximum`);
3. dt, the HLL sweeps, phases [E]+[F].  Two ghost layers keep every owned
   layer two layers from the local line ends, where the serial copy rules of
   pas_HLL act, so only ghosts see them;
4. the ghost exchange: each slab sends its two lowest owned layers down and
   its two highest up (batched point-to-point, NCCL between GPUs).

The owned layers of all slabs then equal the single-domain step bit for bit.
`engine` objects provide begin() -> local vmax pair, end(pair),
get_layers(k0, nk) and set_layers(k0, nk, buf) on the slab's local layers;
GpuSlab is the library's, the tests add one on the CPU.
"""
import numpy as np

GHOST = 2


def partition(Nz, nranks):
    """Owned z-ranges [k0, k1) of the ranks, as even as possible; each slab
    needs at least GHOST layers (its neighbours' ghosts)."""
    if Nz < GHOST * nranks:
        raise ValueError(f"Nz = {Nz} is too small for {nranks} z-slabs of at least {GHOST} layers")
    base, extra = divmod(Nz, nranks)
    out, k = [], 0
    for r in range(nranks):
        n = base + (1 if r < extra else 0)
        out.append((k, k + n))
        k += n
    return out


def local_layout(Nz, nranks, rank):
    """(k0, k1, lo, hi): the owned global range and the ghost layers below
    and above; the slab's local layers are global [k0 - lo, k1 + hi)."""
    k0, k1 = partition(Nz, nranks)[rank]
    lo = GHOST if rank > 0 else 0
    hi = GHOST if rank < nranks - 1 else 0
    return k0, k1, lo, hi


def slab_params(p, nranks, rank):
    """The local parameter dict of a slab (its z-extent covers the local
    layers; the step uses the global spacing through hyq_set_spacing)."""
    k0, k1, lo, hi = local_layout(p["Nz"], nranks, rank)
    q = dict(p)
    q["Nz"] = (k1 + hi) - (k0 - lo)
    return q


def vmax_pair(v):
    """{max over non-NaN, NaN flag} of a local max |speed|."""
    return (0.0, 1.0) if v != v else (float(v), 0.0)


def vmax_from_pair(pair):
    return float("nan") if pair[1] > 0 else float(pair[0])


def step(engine, rank, nranks, layout, dist, make_buffer, group=None):
    """One step of a slab: phase [A], the MAX all-reduce, the rest of the
    step, the ghost exchange.  make_buffer(shape) returns a tensor on the
    engine's device (the communication buffers)."""
    import torch
    k0, k1, lo, hi = layout
    pair = make_buffer((2,))
    engine.begin(pair)
    if dist is not None and nranks > 1:
        dist.all_reduce(pair, op=dist.ReduceOp.MAX, group=group)
    engine.end(pair)
    if dist is None or nranks == 1:
        return
    own = k1 - k0
    ops, recv = [], []
    if rank > 0:
        send_lo = engine.get_layers(lo, GHOST)
        buf = torch.empty_like(send_lo)
        ops += [dist.P2POp(dist.isend, send_lo, rank - 1, group), dist.P2POp(dist.irecv, buf, rank - 1, group)]
        recv.append((0, buf))
    if rank < nranks - 1:
        send_hi = engine.get_layers(lo + own - GHOST, GHOST)
        buf = torch.empty_like(send_hi)
        ops += [dist.P2POp(dist.isend, send_hi, rank + 1, group), dist.P2POp(dist.irecv, buf, rank + 1, group)]
        recv.append((lo + own, buf))
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    for kl, buf in recv:
        engine.set_layers(kl, GHOST, buf)


class GpuSlab:
    """A slab on this rank's GPU: a library context over the local layers."""

    def __init__(self, p, nranks, rank, device=0, mode="plain"):
        import torch
        from . import ic
        from .runner import Solver
        self.torch = torch
        self.layout = local_layout(p["Nz"], nranks, rank)
        k0, k1, lo, hi = self.layout
        self.params = slab_params(p, nranks, rank)
        self.solver = Solver(self.params, device=device, mode=mode)
        g = ic.grid_spacing(p)
        self.solver._chk(self.solver._lib.hyq_set_spacing(self.solver._h, g["dx"], g["dy"], g["dz"]))
        self.Nx, self.Ny = p["Nx"], p["Ny"]
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.ExternalStream(self.solver.stream, device=self.device)
        self.global_params = p

    def set_initial_condition(self):
        """The slab's layers of the global initial condition, generated on the
        device from the global tables (the z-centres of the local layers)."""
        from . import ic
        k0, k1, lo, hi = self.layout
        xm, ym, zm, dx, dy, dz, bg, regions, moments = ic.ic_tables(self.global_params)
        zl = np.ascontiguousarray(zm[k0 - lo:k1 + hi])
        off = k0 - lo
        # index boxes (the runner's built-in cubes) move to local z-indices
        regions = [(kind, every, rlo, rhi, (i0, i1, j0, j1, kk0 - off, kk1 - off)) if kind == 1 else (kind, every, rlo, rhi, idx)
                   for kind, every, rlo, rhi, idx in regions for (i0, i1, j0, j1, kk0, kk1) in [idx]]
        tables = (xm, ym, zl, dx, dy, dz, bg, regions, moments)
        self.solver.set_state_ic(dict(self.global_params), tables=tables)

    def begin(self, pair):
        lib = self.solver._lib
        self.solver._chk(lib.hyq_step_begin(self.solver._h, pair.data_ptr()))
        self.solver.synchronize()

    def end(self, pair):
        self.torch.cuda.current_stream(self.device).synchronize()
        self.solver._chk(self.solver._lib.hyq_step_end(self.solver._h, pair.data_ptr()))
        self.solver.synchronize()

    def get_layers(self, kl, nk):
        buf = self.torch.empty((35, nk * self.Nx * self.Ny), dtype=self.torch.float64, device=self.device)
        self.solver._chk(self.solver._lib.hyq_copy_layers(self.solver._h, kl, nk, buf.data_ptr(), 0))
        self.solver.synchronize()
        return buf

    def set_layers(self, kl, nk, buf):
        self.torch.cuda.current_stream(self.device).synchronize()
        self.solver._chk(self.solver._lib.hyq_copy_layers(self.solver._h, kl, nk, buf.data_ptr(), 1))
        self.solver.synchronize()

    def owned_state(self):
        """(Nx, Ny, own, 35) of the owned layers (host)."""
        k0, k1, lo, hi = self.layout
        return self.solver.get_state()[:, :, lo:lo + (k1 - k0), :]

    def stats(self):
        return self.solver.stats()

    def close(self):
        self.solver.close()
