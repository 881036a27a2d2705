"""The wave-speed network of the learned path (HYQ_MODE_LEARNED).

A 35 -> 128 -> 128 -> 128 -> 6 MLP with SiLU maps a cell's standardized
moments (M2CS4_35's S of the realized moments) to the six extreme eigenvalues
of its x, y and z flux Jacobians, standardized as (lam - u_a) / sqrt(C_aa).
The step uses the prediction only to seed the certified characteristic-
polynomial solve of each Jacobian (hyq_charpoly.cuh): the network decides
where the root search starts, never what the speeds are.

Everything that computes runs in libhyqmom_b200.so: training inputs and
targets (hyq_net_features, hyq_cells_wavespeed_targets), the BF16 tcgen05
forward/backward kernels (hyq_net_train_batch), Adam (hyq_net_adam) and the
inference kernel the step launches.  PyTorch only holds device buffers.

Training data (seeded): the realized moments of plain-path crossing-jet runs
at Ma in {0, 0.5, 1, 2} x Kn in {1e-3, 1e-2, 1e-1, 1}, plus realizable
moments of random Gaussian mixtures (2-4 components, Dirichlet(1) weights,
means N(0, Ma^2), Wishart(5) covariances), all in FP64.
"""
import ctypes
import os

import numpy as np

from . import _lib

NIN, NH, NOUT = 35, 128, 6
P_W1 = 0
P_B1 = P_W1 + NH * NIN
P_W2 = P_B1 + NH
P_B2 = P_W2 + NH * NH
P_W3 = P_B2 + NH
P_B3 = P_W3 + NH * NH
P_W4 = P_B3 + NH
P_B4 = P_W4 + NOUT * NH
NPARAM = P_B4 + NOUT
assert NPARAM == _lib.NET_PARAMS

WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wavenet_weights.npz")


class WaveNet:
    """FP32 parameters (the C-ABI order) and the seed margin."""

    def __init__(self, params, margin=0.05, meta=None):
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        assert self.params.size == NPARAM
        self.margin = float(margin)
        self.meta = dict(meta or {})

    def save(self, path=WEIGHTS_PATH):
        np.savez(path, params=self.params, margin=np.float64(self.margin),
                 meta=np.array(repr(self.meta)))

    @classmethod
    def load(cls, path=WEIGHTS_PATH):
        z = np.load(path, allow_pickle=False)
        meta = {}
        if "meta" in z.files:
            try:
                import ast
                meta = ast.literal_eval(str(z["meta"]))
            except (ValueError, SyntaxError):
                meta = {}
        return cls(z["params"], float(z["margin"]), meta)

    def layers(self):
        """(W1, b1, W2, b2, W3, b3, W4, b4) as FP32 arrays (W: out x in)."""
        p = self.params
        return (p[P_W1:P_B1].reshape(NH, NIN), p[P_B1:P_W2], p[P_W2:P_B2].reshape(NH, NH), p[P_B2:P_W3],
                p[P_W3:P_B3].reshape(NH, NH), p[P_B3:P_W4], p[P_W4:P_B4].reshape(NOUT, NH), p[P_B4:NPARAM])


def load_default():
    """The packaged, trained network (raises if it is missing)."""
    if not os.path.exists(WEIGHTS_PATH):
        raise _lib.HyqError(f"no trained wave-speed network at {WEIGHTS_PATH}; train one with hyqmom.wavenet.train()")
    return WaveNet.load(WEIGHTS_PATH)


def init_params(seed=0):
    """He-style initialisation (uniform, fan-in), zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    for w0, w1, fan in ((P_W1, P_B1, NIN), (P_W2, P_B2, NH), (P_W3, P_B3, NH), (P_W4, P_B4, NH)):
        lim = np.sqrt(6.0 / fan) * (0.5 if w0 == P_W4 else 1.0)
        p[w0:w1] = rng.uniform(-lim, lim, w1 - w0)
    return p


# ----------------------------------------------------------- host reference
def bf16(x):
    """Round to BF16 (nearest even) and back, as the device does."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def reference_forward(params, S, emulate=True):
    """Host forward pass in FP64 on inputs S (n x 35).  emulate: round the
    weights, inputs and activations to BF16 where the device kernels do."""
    net = WaveNet(params)
    W1, b1, W2, b2, W3, b3, W4, b4 = [np.asarray(a, np.float64) for a in net.layers()]
    r = (lambda a: bf16(a).astype(np.float64)) if emulate else (lambda a: np.asarray(a, np.float64))
    W1, W2, W3, W4 = r(W1), r(W2), r(W3), r(W4)
    h = r(S)
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        h = r(_silu(h @ W.T + b))
    return h @ W4.T + b4


def reference_gradients(params, S, T, dscale, emulate=True):
    """Host FP64 backward pass of 0.5 * dscale * sum((y - T)^2) with the
    device's BF16 roundings (emulate): returns (gradient vector, sum of
    squared errors)."""
    net = WaveNet(params)
    W1, b1, W2, b2, W3, b3, W4, b4 = [np.asarray(a, np.float64) for a in net.layers()]
    r = (lambda a: bf16(a).astype(np.float64)) if emulate else (lambda a: np.asarray(a, np.float64))
    W1, W2, W3, W4 = r(W1), r(W2), r(W3), r(W4)
    x = r(S)
    hs, ds = [x], []
    h = x
    for W, b in ((W1, b1), (W2, b2), (W3, b3)):
        z = h @ W.T + b
        h = r(_silu(z))
        hs.append(h)
        ds.append(r(_dsilu(z)))
    y = h @ W4.T + b4
    e = y - T
    sse = float(np.sum(e * e))
    g = r(dscale * e)
    grads = np.zeros(NPARAM)
    grads[P_W4:P_B4] = (g.T @ hs[3]).ravel()
    grads[P_B4:NPARAM] = g.sum(0)
    dh = g @ W4
    for l, (W, w0, b0) in reversed(list(enumerate(((W1, P_W1, P_B1), (W2, P_W2, P_B2), (W3, P_W3, P_B3))))):
        dz = r(dh * ds[l])
        grads[w0:b0] = (dz.T @ hs[l]).ravel()
        grads[b0:b0 + NH] = dz.sum(0)
        dh = dz @ W
    return grads, sse


# ----------------------------------------------------------- device helpers
def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _chk(rc):
    if rc != 0:
        raise _lib.HyqError(f"{_lib.ERRORS.get(rc, rc)}: {_lib.load().hyq_last_error(None).decode()}")


def targets(M, flag2D=0, Ma=1.0, positivity=True):
    """(T, Mr): device training targets [n, 8] (6 used) and realized moments
    [35, n] of the moments M (torch float64 [35, n], moment-major)."""
    import torch
    lib = _lib.load()
    n = M.shape[1]
    T = torch.empty((n, 8), dtype=torch.float32, device=M.device)
    Mr = torch.empty_like(M)
    _chk(lib.hyq_cells_wavespeed_targets(_ptr(M), n, int(flag2D), float(Ma), int(bool(positivity)), _ptr(T), _ptr(Mr), _stream(torch)))
    return T, Mr


def features(Mr):
    """Device input tiles (uint8 [ntiles, tile_bytes]) of the moments Mr [35, n]."""
    import torch
    lib = _lib.load()
    n = Mr.shape[1]
    nt = (n + 127) // 128
    X = torch.empty((nt, int(lib.hyq_net_tile_bytes())), dtype=torch.uint8, device=Mr.device)
    _chk(lib.hyq_net_features(_ptr(Mr), n, _ptr(X), _stream(torch)))
    return X


def pack(w):
    """Device BF16 weight image of the FP32 parameters w (torch, device)."""
    import torch
    lib = _lib.load()
    img = torch.zeros(int(lib.hyq_net_image_bytes()), dtype=torch.uint8, device=w.device)
    _chk(lib.hyq_net_pack(_ptr(w), _ptr(img), _stream(torch)))
    return img


def forward(image, M):
    """Network outputs [6, n] (torch float32) of the moments M [35, n] through
    the inference kernel the step uses (features computed inline)."""
    import torch
    lib = _lib.load()
    n = M.shape[1]
    out = torch.empty((6, n), dtype=torch.float32, device=M.device)
    err = torch.zeros(1, dtype=torch.int32, device=M.device)
    _chk(lib.hyq_net_forward(_ptr(image), _ptr(M), n, _ptr(out), _ptr(err), _stream(torch)))
    torch.cuda.synchronize()
    if int(err.item()):
        raise _lib.HyqError("HYQ_ETIMEOUT: the network kernel gave up waiting for its tensor-core operations")
    return out


class Trainer:
    """Adam on the device through the library's training kernels."""

    def __init__(self, params, nparts=None, lr=2e-3, betas=(0.9, 0.999), eps=1e-8, wd=0.0):
        import torch
        self.torch = torch
        self.lib = _lib.load()
        dev = torch.device("cuda")
        self.w = torch.tensor(np.asarray(params, np.float32), device=dev)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        props = torch.cuda.get_device_properties(dev)
        self.nparts = int(nparts or props.multi_processor_count)
        self.partial = torch.zeros((self.nparts, NPARAM), dtype=torch.float32, device=dev)
        self.scratch = torch.empty(int(self.lib.hyq_net_scratch_bytes(self.nparts)), dtype=torch.uint8, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.image = pack(self.w)
        self.lr, self.betas, self.eps, self.wd = lr, betas, eps, wd
        self.step_count = 0

    def gradients(self, X, T, n, tiles, rows):
        """Summed gradient of the batch `tiles` (torch int32 on the device) of
        0.5 * dscale * SSE with dscale = 2 / (rows * 6); returns (grad, sse)."""
        torch = self.torch
        g = torch.empty_like(self.w)
        self.loss.zero_()
        nparts = min(self.nparts, int(tiles.numel()))
        _chk(self.lib.hyq_net_train_batch(_ptr(self.image), _ptr(X), _ptr(T), int(n), _ptr(tiles), int(tiles.numel()),
                                           float(2.0 / (rows * 6)), _ptr(self.scratch), _ptr(self.partial), nparts, _ptr(self.loss),
                                           _ptr(self.err), _stream(torch)))
        _chk(self.lib.hyq_net_adam(_ptr(self.w), _ptr(self.m), _ptr(self.v), _ptr(self.partial), nparts, 0.0, 0.9, 0.999, 1e-8, 0.0,
                                   1, _ptr(g), _stream(torch)))
        torch.cuda.synchronize()
        if int(self.err.item()):
            raise _lib.HyqError("HYQ_ETIMEOUT in the training kernel")
        return g, float(self.loss.item())

    def step(self, X, T, n, tiles, rows, lr=None):
        """One Adam step on a batch (no host synchronisation)."""
        torch = self.torch
        self.step_count += 1
        nparts = min(self.nparts, int(tiles.numel()))
        _chk(self.lib.hyq_net_train_batch(_ptr(self.image), _ptr(X), _ptr(T), int(n), _ptr(tiles), int(tiles.numel()),
                                           float(2.0 / (rows * 6)), _ptr(self.scratch), _ptr(self.partial), nparts, _ptr(self.loss),
                                           _ptr(self.err), _stream(torch)))
        _chk(self.lib.hyq_net_adam(_ptr(self.w), _ptr(self.m), _ptr(self.v), _ptr(self.partial), nparts,
                                   float(self.lr if lr is None else lr), float(self.betas[0]), float(self.betas[1]),
                                   float(self.eps), float(self.wd), self.step_count, None, _stream(torch)))
        _chk(self.lib.hyq_net_pack(_ptr(self.w), _ptr(self.image), _stream(torch)))

    def check(self):
        self.torch.cuda.synchronize()
        if int(self.err.item()):
            raise _lib.HyqError("HYQ_ETIMEOUT in the training kernel")

    def params(self):
        return self.w.detach().cpu().numpy().copy()


# ----------------------------------------------------------- training data
def gaussian_raw_moments(mu, cov):
    """Raw moments up to order 4 of 3-D Gaussians (mu [n,3], cov [n,3,3]) in
    the 35-moment order, by the Gaussian recursion
    E[x_i f] = mu_i E[f] + sum_j cov_ij E[d f / d x_j]."""
    n = mu.shape[0]
    memo = {(0, 0, 0): np.ones(n)}

    def m(a, b, c):
        key = (a, b, c)
        if key in memo:
            return memo[key]
        if a > 0:
            i, e = 0, (a - 1, b, c)
        elif b > 0:
            i, e = 1, (a, b - 1, c)
        else:
            i, e = 2, (a, b, c - 1)
        val = mu[:, i] * m(*e)
        for j in range(3):
            if e[j] > 0:
                d = list(e)
                d[j] -= 1
                val = val + cov[:, i, j] * e[j] * m(*d)
        memo[key] = val
        return val

    return np.stack([m(*ijk) for ijk in MOMENT_ORDER], axis=0)


# (i, j, k) exponents of the 35 moments (src/utils/moment_idx.jl:73-76)
MOMENT_ORDER = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 0, 0), (4, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0), (3, 1, 0), (0, 2, 0),
                (1, 2, 0), (2, 2, 0), (0, 3, 0), (1, 3, 0), (0, 4, 0), (0, 0, 1), (1, 0, 1), (2, 0, 1), (3, 0, 1), (0, 0, 2),
                (1, 0, 2), (2, 0, 2), (0, 0, 3), (1, 0, 3), (0, 0, 4), (0, 1, 1), (1, 1, 1), (2, 1, 1), (0, 2, 1), (1, 2, 1),
                (0, 3, 1), (0, 1, 2), (1, 1, 2), (0, 1, 3), (0, 2, 2)]


def mixture_moments(n, rng, Ma=1.0):
    """Raw moments [35, n] of n random Gaussian mixtures: 2-4 components,
    weights Dirichlet(1), means N(0, Ma^2), covariances Wishart(5 dof, I/5),
    density 1."""
    out = np.zeros((35, n))
    K = rng.integers(2, 5, size=n)
    for k in range(4):
        use = K > k
        w = np.zeros(n)
        w[use] = 1.0
        if k == 0:
            wts = rng.dirichlet(np.ones(4), size=n)
        cnt = use.sum()
        if cnt == 0:
            continue
        mu = rng.normal(0.0, max(Ma, 1e-3), size=(n, 3))
        A = rng.normal(size=(n, 3, 5)) / np.sqrt(5.0)
        cov = A @ np.transpose(A, (0, 2, 1))
        wk = np.where(use, wts[:, k], 0.0)
        out += wk[None, :] * gaussian_raw_moments(mu, cov)
    return out / out[0][None, :]


def crossing_run_states(Ma, Kn, grid=(48, 48, 24), steps=120, every=8, device=0):
    """Moment states [35, n] of a plain-path crossing-jets run (CFL 0.5),
    sampled every `every` steps after the first."""
    from . import ic
    from .runner import Solver
    p = ic.with_jets(ic.default_params(Nx=grid[0], Ny=grid[1], Nz=grid[2], Ma=Ma, Kn=Kn, CFL=0.5, tmax=1e9, nnmax=100000),
                     "crossing")
    s = Solver(p, device=device)
    out = []
    try:
        s.set_state(ic.initial_state(p))
        for k in range(every, steps + 1, every):
            s.advance(every)
            if s.stats()["status"]:
                break
            out.append(s.get_state().reshape(-1, 35, order="F").T.copy())
    finally:
        s.close()
    return np.concatenate(out, axis=1) if out else np.zeros((35, 0))


def build_dataset(seed=0, grid=(48, 48, 24), steps=120, every=6, n_mix=2_400_000, Mas=(0.0, 0.5, 1.0, 2.0),
                  Kns=(1e-3, 1e-2, 1e-1, 1.0), device=0, log=print):
    """Training set on the device: (X tiles, T [n, 8], n).  Rows whose target
    is not finite are dropped; rows are shuffled (seeded)."""
    import torch
    rng = np.random.default_rng(seed)
    parts = []
    for Ma in Mas:
        for Kn in Kns:
            S = crossing_run_states(Ma, Kn, grid=grid, steps=steps, every=every, device=device)
            parts.append((S, Ma))
            log(f"crossing Ma={Ma} Kn={Kn}: {S.shape[1]} states")
    for q, Ma in enumerate(Mas):
        parts.append((mixture_moments(n_mix // len(Mas), rng, Ma=Ma), Ma))
    Ms, Ts = [], []
    for S, Ma in parts:
        if S.shape[1] == 0:
            continue
        M = torch.tensor(S, dtype=torch.float64, device="cuda")
        T, Mr = targets(M, Ma=Ma)
        ok = torch.isfinite(T[:, :6]).all(dim=1) & torch.isfinite(Mr).all(dim=0)
        Ms.append(Mr[:, ok])
        Ts.append(T[ok])
        del M
    Mr = torch.cat(Ms, dim=1)
    T = torch.cat(Ts, dim=0)
    perm = torch.tensor(rng.permutation(Mr.shape[1]), device="cuda")
    Mr = Mr[:, perm].contiguous()
    T = T[perm].contiguous()
    X = features(Mr)
    return X, T, Mr


def train(out=WEIGHTS_PATH, seed=0, epochs=6, batch_tiles=64, lr=2e-3, val_frac=0.05, data=None, log=print, **data_kw):
    """Train the network on the device; returns (WaveNet, report)."""
    import time
    import torch
    t0 = time.time()
    X, T, Mr = data if data is not None else build_dataset(seed=seed, log=log, **data_kw)
    n = T.shape[0]
    ntiles = (n + 127) // 128
    nval = max(1, int(ntiles * val_frac))
    val_tiles, train_tiles = np.arange(ntiles - nval, ntiles), np.arange(0, ntiles - nval)
    tr = Trainer(init_params(seed), lr=lr)
    rng = np.random.default_rng(seed + 1)
    steps_per_epoch = max(1, len(train_tiles) // batch_tiles)
    total = epochs * steps_per_epoch
    history = []
    for ep in range(epochs):
        order = rng.permutation(train_tiles).astype(np.int32)
        ord_dev = torch.tensor(order, device="cuda")
        for s in range(steps_per_epoch):
            k = ep * steps_per_epoch + s
            lr_k = lr * 0.5 * (1.0 + np.cos(np.pi * k / total))
            tiles = ord_dev[s * batch_tiles:(s + 1) * batch_tiles]
            tr.step(X, T, n, tiles, rows=tiles.numel() * 128, lr=lr_k)
        tr.check()
        vl = evaluate(tr.image, Mr, T, val_tiles)
        history.append({"epoch": ep + 1, "val_rmse": vl["rmse"]})
        log(f"epoch {ep + 1}: val rmse {vl['rmse']:.4f} ({time.time() - t0:.1f} s)")
    rep = evaluate(tr.image, Mr, T, val_tiles)
    # the seeds move outward by twice the median error (normalised units): a
    # seed that still lands inside the spectrum is rejected by the solve's
    # sign test and costs one evaluation, one placed far outside costs Newton
    # steps, so a tight margin wins (host sweep on crossing-jet states)
    margin = float(min(0.05, max(0.005, 2.0 * rep["median_abs"])))
    net = WaveNet(tr.params(), margin=margin,
                  meta={"rows": int(n), "epochs": epochs, "batch_rows": batch_tiles * 128, "lr": lr, "seed": seed,
                        "val_rmse": rep["rmse"], "val_q99_abs": rep["q99_abs"], "history": history,
                        "train_seconds": round(time.time() - t0, 1)})
    if out:
        net.save(out)
    return net, rep


def evaluate(image, Mr, T, tiles):
    """Validation error of the network on the rows of `tiles` (inference
    kernel, features computed inline from Mr)."""
    import torch
    rows = torch.tensor(np.concatenate([np.arange(t * 128, t * 128 + 128) for t in tiles]), device="cuda")
    rows = rows[rows < T.shape[0]]
    M = Mr[:, rows].contiguous()
    y = forward(image, M).T
    e = (y - T[rows, :6]).abs()
    return {"rmse": float(torch.sqrt((e * e).mean()).item()), "q99_abs": float(torch.quantile(e.flatten()[:1_000_000], 0.99).item()),
            "median_abs": float(e.median().item()), "rows": int(rows.numel())}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the wave-speed network on the GPU")
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n-mix", type=int, default=2_400_000)
    args = ap.parse_args()
    net, rep = train(out=args.out, epochs=args.epochs, seed=args.seed, n_mix=args.n_mix)
    print(json.dumps({"report": rep, "margin": net.margin, "meta": net.meta}))
