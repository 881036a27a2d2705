"""Cell states chosen to take the rare branches of the reference's closure,
realizability and eigenvalue code (test data; FP64, seeded):

* developed crossing-jet cells (oracle run, Kn = 0.01), which take the
  flag220 repeats, the complex-eigenvalue corrections and the fast-math NaN
  of the Cardano roots;
* degenerate Gaussians (rank-1 and rank-2 covariances, |correlation| = 1 or
  a singular correlation matrix): the faces case of realizable_3D and
  edge_corner_correction;
* near-degenerate two-component mixtures (|correlation| -> 1);
* rank-1 Gaussians whose cross covariances are divided by 0.9999: their
  correlations sit at a corner of the elliptope scaled out by 1 / 0.9999,
  so realizability_S2's 0.9999 contraction lands S2 on the boundary and
  realizable_3D takes its S2 <= S2min faces case (a non-realizable input
  such as the x+y+z-2M update can produce);
* states with a negative variance along x, y or z (what the x+y+z-2M update
  can leave behind): eigenvalues6z's re-realization when the z function
  runs on them directly (phase [A] realizes them first).
"""
import numpy as np

import oracle_lib as ol
from hyqmom import ic, wavenet


def _gauss(w, mu, C):
    return w * wavenet.gaussian_raw_moments(np.asarray(mu, float)[None, :], np.asarray(C, float)[None, :, :])[:, 0]


def branch_states(seed=11, n_flow=240):
    rng = np.random.default_rng(seed)
    out = []
    # developed flow
    p = ic.with_jets(ic.default_params(Nx=12, Ny=12, Nz=12, Ma=1.0, Kn=0.01, CFL=0.5, tmax=10.0, nnmax=100), "crossing")
    M = np.asfortranarray(ic.initial_state(p))
    pp = dict(p, **ic.grid_spacing(p))
    t = 0.0
    for _ in range(16):
        _, t, _ = ol.step(M, pp, t)
    cells = np.array(M).reshape(-1, 35, order="F")
    out.append(cells[rng.choice(len(cells), n_flow, replace=False)])
    # degenerate Gaussians
    for _ in range(24):
        mu = rng.normal(0, 1, 3)
        a = rng.normal(size=3)
        C1 = np.outer(a, a) + 1e-14 * np.eye(3)            # rank 1: |corr| = 1 pairwise
        B = rng.normal(size=(3, 2))
        C2 = B @ B.T                                         # rank 2: singular correlation
        out.append(_gauss(1.0, mu, C1)[None, :])
        out.append(_gauss(1.0, mu, C2)[None, :])
    # near-degenerate mixtures
    for _ in range(48):
        mu = rng.normal(0, 0.7, (2, 3))
        a = rng.normal(size=3)
        eps = 10 ** rng.uniform(-9, -3)
        C = [np.outer(a, a) + eps * np.eye(3), np.outer(a + 0.05 * rng.normal(size=3), a) + eps * np.eye(3)]
        C[1] = 0.5 * (C[1] + C[1].T) + eps * np.eye(3)
        w = rng.dirichlet([1.0, 1.0])
        out.append((_gauss(w[0], mu[0], C[0]) + _gauss(w[1], mu[1], C[1]))[None, :])
    # corners of the elliptope scaled out by 1 / 0.9999
    for _ in range(24):
        v = rng.choice([-1.0, 1.0], 3)
        sd = np.exp(rng.uniform(-0.5, 0.5, 3))
        mu = rng.normal(0, 1, 3)
        C = np.outer(v * sd, v * sd)
        m = _gauss(1.0, mu, C).copy()
        for idx, (i, j) in ((6, (0, 1)), (16, (0, 2)), (25, (1, 2))):
            m[idx] = C[i, j] / 0.9999 + mu[i] * mu[j]
        out.append(m[None, :])
    # negative variance along one axis
    for q in range(24):
        mu = rng.normal(0, 1, 3)
        A = rng.normal(size=(3, 3))
        m = _gauss(1.0, mu, A @ A.T / 3 + 0.1 * np.eye(3))
        i1, i2 = [(1, 2), (5, 9), (15, 19)][q % 3]
        m = m.copy()
        m[i2] = m[i1] ** 2 / m[0] - 0.05 * (1 + rng.random())
        out.append(m[None, :])
    return np.concatenate(out, axis=0)


def negative_variance_rows(states):
    """Rows of `states` with a negative variance along some axis."""
    m0 = states[:, 0]
    var = [states[:, i2] / m0 - (states[:, i1] / m0) ** 2 for i1, i2 in ((1, 2), (5, 9), (15, 19))]
    return np.where((var[0] < 0) | (var[1] < 0) | (var[2] < 0))[0]
