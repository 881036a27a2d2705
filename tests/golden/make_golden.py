"""Generate the committed golden fixtures under tests/golden/.

Run once in a checkout that has the reference mounted (default
/root/reference, override with HYQMOM_REFERENCE):

    python tests/golden/make_golden.py

It writes three kinds of fixtures, all numbers only:

* ``autogen.npz``  -- seeded random inputs and the outputs of the reference's
  own generated closed forms (``src/autogen/*.jl``), evaluated through the
  fixture-time translator in ``julia_autogen.py``.
* ``matlab_unit.npz`` -- the MATLAB v5 unit goldens the reference's
  ``test/test_golden_files.jl`` compares against
  (``legacy/3D_MATLAB/tests/goldenfiles/*.mat``), flattened.
* ``mpi_1rank_{small,medium}.npz`` -- the end-to-end Nz=1 goldens of
  ``test/goldenfiles/mpi_1rank_*.bin`` (header + (Np,Np,35) array), which the
  reference's ``test/test_mpi.jl:114-141`` reads.

Nothing at test time reads the reference; tests only read these files.
"""
import os
import sys

import numpy as np
import scipy.io as sio

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import julia_autogen as ja  # noqa: E402

REF = ja.REF_ROOT


def std_moments(rng, n_samples=9, dim=3, corr=0.6):
    """Standardized moments S_ijk (i+j+k <= 5) of a random weighted sample."""
    P = rng.normal(size=(dim, n_samples))
    if dim >= 2:
        P[1] += corr * rng.normal() * P[0]
    if dim >= 3:
        P[2] += corr * rng.normal() * P[1]
    w = rng.random(n_samples)
    w /= w.sum()
    mu = P @ w
    P = P - mu[:, None]
    sd = np.sqrt((P ** 2) @ w)
    P = P / sd[:, None]
    if dim == 3:
        return lambda i, j, k: float(np.sum(w * P[0] ** i * P[1] ** j * P[2] ** k))
    return lambda i, j: float(np.sum(w * P[0] ** i * P[1] ** j))


S28_NAMES = ['300', '400', '110', '210', '310', '120', '220', '030', '130', '040', '101', '201', '301', '102', '202',
             '003', '103', '004', '011', '111', '211', '021', '121', '031', '012', '112', '013', '022']


def autogen_fixtures(rng, n=64):
    out = {}
    # delta2star3D, lower_bound_S220, bound_minor1 on realizable and perturbed states
    d2 = ja.get('delta2star3D')
    lb = ja.get('lower_bound_S220')
    bm = ja.get('bound_minor1')
    A, E, LB, BM = [], [], [], []
    for t in range(n):
        S = std_moments(rng)
        a = np.array([S(*map(int, nm)) for nm in S28_NAMES])
        if t % 2:
            a = a + 0.05 * rng.normal(size=28)
        A.append(a)
        E.append(np.asarray(d2(*a), dtype=float))
        g = dict(zip(S28_NAMES, a))
        LB.append(np.asarray(lb(g['011'], g['012'], g['021'], g['101'], g['102'], g['110'], g['111'], g['120'], g['201'], g['210'])))
        BM.append(np.asarray(bm(g['003'], g['011'], g['012'], g['021'], g['030'], g['101'], g['102'], g['110'], g['111'],
                                g['120'], g['201'], g['210'], g['300'])))
    out['d2_in'] = np.array(A)
    out['d2_E'] = np.array(E)
    out['lb_S220'] = np.array(LB)
    out['bound_minor1'] = np.array(BM)

    # jacobian6 on 2-D raw moments of random samples (x = flux direction)
    jac = ja.get('jacobian6')
    keys = [(0, 0), (0, 1), (0, 2), (0, 3), (0, 4), (1, 0), (1, 1), (1, 2), (1, 3), (2, 0), (2, 1), (2, 2), (3, 0), (3, 1), (4, 0)]
    Jin, Jout = [], []
    for t in range(n):
        X = rng.normal(rng.normal(), 0.3 + rng.random(), 7)
        Y = rng.normal(rng.normal(), 0.3 + rng.random(), 7) + 0.4 * rng.normal() * X
        w = rng.random(7)
        w *= (0.01 + 2 * rng.random()) / w.sum()
        m = np.array([np.sum(w * X ** a * Y ** b) for (a, b) in keys])
        Jin.append(m)
        Jout.append(np.asarray(jac(*m), dtype=float))
    out['jac_in'] = np.array(Jin)
    out['jac_J'] = np.array(Jout)

    # delta2starchol_L3 and rootsR on 2-D standardized states (realizable and not)
    L3f = ja.get('delta2starchol_L3')
    rr = ja.get('rootsR')
    Lin, Lout, Rin, Rre, Rim = [], [], [], [], []
    for t in range(n):
        S = std_moments(rng, dim=2)
        s = {k: S(*k) for k in [(3, 0), (4, 0), (1, 1), (2, 1), (3, 1), (1, 2), (2, 2), (0, 3), (1, 3), (0, 4)]}
        if t % 2:
            for k in s:
                if k not in [(4, 0), (0, 4)]:
                    s[k] += 0.2 * rng.normal()
            s[(1, 1)] = np.tanh(s[(1, 1)])
        a = [s[(0, 3)], s[(0, 4)], s[(1, 1)], s[(1, 2)], s[(1, 3)], s[(2, 1)], s[(2, 2)], s[(3, 0)], s[(3, 1)], s[(4, 0)]]
        Lin.append(a)
        Lout.append(L3f(*a))
        H20 = s[(4, 0)] - s[(3, 0)] ** 2 - 1
        H02 = s[(0, 4)] - s[(0, 3)] ** 2 - 1
        b = [1 - s[(1, 1)] ** 2, H02, H20, s[(0, 3)], s[(1, 1)], s[(1, 2)], s[(1, 3)], s[(2, 1)], s[(3, 0)], s[(3, 1)]]
        R = np.asarray(rr(*b), dtype=complex)
        Rin.append(b)
        Rre.append(R.real)
        Rim.append(R.imag)
    # extra rootsR cases chosen to have one real root (finite Cardano output)
    k = 0
    while k < n:
        s30, s11, s21, s31, s12, s03, s13 = rng.normal(size=7) * 0.7
        s11 = np.tanh(s11)
        H20, H02 = rng.random(2) * 2 + 0.01
        b = [1 - s11 ** 2, H02, H20, s03, s11, s12, s13, s21, s30, s31]
        R = np.asarray(rr(*b), dtype=complex)
        if np.all(np.isfinite(R)):
            Rin.append(b)
            Rre.append(R.real)
            Rim.append(R.imag)
            k += 1
    out['L3_in'] = np.array(Lin)
    out['L3_out'] = np.array(Lout)
    out['rootsR_in'] = np.array(Rin)
    out['rootsR_re'] = np.array(Rre)
    out['rootsR_im'] = np.array(Rim)

    rxy = ja.get('rootsR_X_Y')
    Xin, Xre, Xim = [], [], []
    k = 0
    while k < 2 * n:
        a = rng.normal(size=9)
        a[0] = abs(a[0]) + 0.05
        a[1] = abs(a[1]) + 0.05
        a[7] = abs(a[7]) + 0.05
        R = np.asarray(rxy(*a), dtype=complex)
        if k < n and not np.all(np.isfinite(R)):
            continue
        Xin.append(a)
        Xre.append(R.real)
        Xim.append(R.imag)
        k += 1
    out['rXY_in'] = np.array(Xin)
    out['rXY_re'] = np.array(Xre)
    out['rXY_im'] = np.array(Xim)

    # moment conversions
    m4c = ja.get('M4toC4_3D')
    c4m = ja.get('C4toM4_3D')
    c5m = ja.get('C5toM5_3D')
    s4c = ja.get('S4toC4_3D_r')
    E35 = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 0, 0), (4, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0), (3, 1, 0), (0, 2, 0), (1, 2, 0),
           (2, 2, 0), (0, 3, 0), (1, 3, 0), (0, 4, 0), (0, 0, 1), (1, 0, 1), (2, 0, 1), (3, 0, 1), (0, 0, 2), (1, 0, 2), (2, 0, 2),
           (0, 0, 3), (1, 0, 3), (0, 0, 4), (0, 1, 1), (1, 1, 1), (2, 1, 1), (0, 2, 1), (1, 2, 1), (0, 3, 1), (0, 1, 2), (1, 1, 2),
           (0, 1, 3), (0, 2, 2)]
    Min, Cout, C5in, M5out, S4in, S4C2, S4out, C4in, C4out = [], [], [], [], [], [], [], [], []
    for t in range(n):
        P = rng.normal(size=(3, 11)) + rng.normal(size=(3, 1))
        w = rng.random(11)
        w *= (0.05 + rng.random()) / w.sum()
        raw = lambda i, j, k: float(np.sum(w * P[0] ** i * P[1] ** j * P[2] ** k))  # noqa: E731
        M = [raw(*e) for e in E35]
        Min.append(M)
        C = np.asarray(m4c(*M))
        Cout.append([C[e] for e in E35])
        # central moments of the same sample up to order 5
        M0 = raw(0, 0, 0)
        mu = P @ w / M0
        Q = P - mu[:, None]
        cen = lambda i, j, k: float(np.sum(w * Q[0] ** i * Q[1] ** j * Q[2] ** k) / M0)  # noqa: E731
        names5 = ['200', '110', '101', '020', '011', '002', '300', '210', '201', '120', '111', '102', '030', '021', '012',
                  '003', '400', '310', '301', '220', '211', '202', '130', '121', '112', '103', '040', '031', '022', '013',
                  '004', '500', '410', '320', '230', '140', '401', '302', '203', '104', '311', '221', '131', '212', '113',
                  '122', '050', '041', '032', '023', '014', '005']
        cv = [cen(*map(int, nm)) for nm in names5]
        args = [M0, mu[0], mu[1], mu[2]] + cv
        C5in.append(args)
        M5 = np.asarray(c5m(*args))
        M5out.append(M5.reshape(-1, order='F'))
        C4args = args[:35]
        C4in.append(C4args)
        C4out.append(np.asarray(c4m(*C4args)).reshape(-1, order='F'))
        # S4toC4_3D_r: covariance + arbitrary 3rd/4th-order standardized values
        G = rng.normal(size=(3, 3))
        C2 = G @ G.T + 0.3 * np.eye(3)
        c2 = [C2[0, 0], C2[0, 1], C2[0, 2], C2[1, 1], C2[1, 2], C2[2, 2]]
        sv = list(rng.normal(size=25) * 0.5)
        for idx in (10, 13, 15, 20, 24):  # S400 S220 S202 S040 S022 S004 offsets (kept positive)
            sv[idx] = abs(sv[idx]) + 1.0
        S4C2.append(c2)
        S4in.append(sv)
        S4out.append(np.asarray(s4c(*c2, *sv)).reshape(-1, order='F'))
    out['m4c_in'] = np.array(Min)
    out['m4c_out'] = np.array(Cout)
    out['c5m_in'] = np.array(C5in)
    out['c5m_out'] = np.array(M5out)
    out['c4m_in'] = np.array(C4in)
    out['c4m_out'] = np.array(C4out)
    out['s4c_C2'] = np.array(S4C2)
    out['s4c_S'] = np.array(S4in)
    out['s4c_out'] = np.array(S4out)
    return out


def matlab_fixtures():
    base = os.path.join(REF, 'legacy', '3D_MATLAB', 'tests', 'goldenfiles')
    out = {}

    def walk(prefix, v):
        if isinstance(v, np.ndarray) and v.dtype.names:
            for nm in v.dtype.names:
                walk(prefix + '.' + nm, v[nm][0, 0])
        elif isinstance(v, np.ndarray) and v.dtype.kind in 'fiub':
            out[prefix] = np.asarray(v, dtype=float)

    for f in sorted(os.listdir(base)):
        if not f.endswith('.mat'):
            continue
        d = sio.loadmat(os.path.join(base, f))
        walk(f[:-4], d['golden_data']['tests'][0, 0])
    return out


def mpi_bin(name):
    path = os.path.join(REF, 'test', 'goldenfiles', f'mpi_1rank_{name}.bin')
    raw = open(path, 'rb').read()
    nranks, Np = np.frombuffer(raw[:16], dtype='<i8')
    tmax, tfinal = np.frombuffer(raw[16:32], dtype='<f8')
    steps = int(np.frombuffer(raw[32:40], dtype='<i8')[0])
    M = np.frombuffer(raw[40:], dtype='<f8').reshape((35, int(Np), int(Np))).transpose(2, 1, 0)  # (Np, Np, 35) column-major
    return dict(nranks=int(nranks), Np=int(Np), tmax=float(tmax), tfinal=float(tfinal), steps=steps, M=np.ascontiguousarray(M))


def main():
    rng = np.random.default_rng(20240611)
    np.savez_compressed(os.path.join(HERE, 'autogen.npz'), **autogen_fixtures(rng))
    np.savez_compressed(os.path.join(HERE, 'matlab_unit.npz'), **matlab_fixtures())
    for nm in ('small', 'medium'):
        np.savez_compressed(os.path.join(HERE, f'mpi_1rank_{nm}.npz'), **mpi_bin(nm))
    print('wrote fixtures to', HERE)


if __name__ == '__main__':
    main()
