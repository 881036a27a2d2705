"""Host-side parameters, grid and initial conditions.

Mirrors, for one rank:
  * ``run_simulation``'s parameter set (src/simulation_runner.jl:816-883);
  * the grid (src/simulation_runner.jl:133-158, 718-729) including Julia's
    exact ``range`` element values (rational ``floatrange`` when start and
    step are short decimals, else exact-sum rounding);
  * the hard-coded crossing-jets IC (src/simulation_runner.jl:200-271) and the
    custom ``CubicRegion`` IC (src/initial_conditions.jl:152-302) with the
    named jet configurations of examples/run_3d_custom_jets.jl:64-272;
  * ``InitializeM4_35`` Gaussian moments (src/moments/InitializeM4_35.jl:204).

The IC is built once on the host, as in the reference; everything per step
runs on the GPU.
"""
from dataclasses import dataclass
from fractions import Fraction
import math

import numpy as np

# 35-moment order of the reference (src/utils/moment_idx.jl:73-76)
E35 = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (3, 0, 0), (4, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0), (3, 1, 0), (0, 2, 0),
       (1, 2, 0), (2, 2, 0), (0, 3, 0), (1, 3, 0), (0, 4, 0), (0, 0, 1), (1, 0, 1), (2, 0, 1), (3, 0, 1), (0, 0, 2),
       (1, 0, 2), (2, 0, 2), (0, 0, 3), (1, 0, 3), (0, 0, 4), (0, 1, 1), (1, 1, 1), (2, 1, 1), (0, 2, 1), (1, 2, 1),
       (0, 3, 1), (0, 1, 2), (1, 1, 2), (0, 1, 3), (0, 2, 2)]
MOMENT_NAMES = ["M%d%d%d" % e for e in E35]


@dataclass
class CubicRegion:
    """A box of constant Gaussian state (src/initial_conditions.jl:34-55)."""
    center: tuple
    width: tuple
    density: float
    velocity: tuple
    temperature: float = 1.0


# ----------------------------------------------------------------- params
def run_simulation_params(Nx=20, Ny=20, Nz=1, tmax=0.1, Kn=1.0, Ma=0.0, flag2D=0, CFL=0.5, **extra):
    """The NamedTuple ``run_simulation`` builds (src/simulation_runner.jl:841-883)."""
    dx, dy, dz = 1.0 / Nx, 1.0 / Ny, 1.0 / Nz
    dtmax = CFL * min(dx, dy, dz)
    nnmax = math.ceil(tmax / dtmax) + 100000
    p = dict(Nx=Nx, Ny=Ny, Nz=Nz, tmax=tmax, Kn=Kn, Ma=Ma, flag2D=flag2D, CFL=CFL, Nmom=35, nnmax=nnmax, dtmax=dtmax,
             rhol=1.0, rhor=0.01, T=1.0, r110=0.0, r101=0.0, r011=0.0, symmetry_check_interval=10,
             homogeneous_z=True, enable_memory_tracking=False, debug_output=False)
    p.update(extra)
    return p


def default_params(**kw):
    """Defaults of examples/parse_params.jl:32-85 (dtmax 1e-2, CFL 0.7 ...)."""
    p = dict(Nx=20, Ny=20, Nz=20, tmax=0.1, Kn=1.0, Ma=0.0, flag2D=0, CFL=0.7, Nmom=35, nnmax=20000000, dtmax=1e-2,
             rhol=1.0, rhor=0.01, T=1.0, r110=0.0, r101=0.0, r011=0.0, symmetry_check_interval=100,
             homogeneous_z=False, enable_memory_tracking=False, debug_output=False,
             xmin=-0.5, xmax=0.5, ymin=-0.5, ymax=0.5, zmin=-0.5, zmax=0.5)
    p.update(kw)
    return p


def extents(p):
    return (p.get("xmin", -0.5), p.get("xmax", 0.5), p.get("ymin", -0.5), p.get("ymax", 0.5),
            p.get("zmin", -0.5), p.get("zmax", 0.5))


def grid_spacing(p):
    """dx, dy, dz from the extents (params.dx is ignored, src/simulation_runner.jl:131-139)."""
    xmin, xmax, ymin, ymax, zmin, zmax = extents(p)
    return dict(dx=(xmax - xmin) / p["Nx"], dy=(ymax - ymin) / p["Ny"], dz=(zmax - zmin) / p["Nz"])


# ------------------------------------------------------ Julia float ranges
def _rat(x):
    """Julia Base.rat for Float64 (continued fraction, |.| <= maxintfloat(Float32))."""
    y = x
    a, b, c, d = 1, 0, 0, 1
    m = 16777216
    while abs(y) <= m:
        f = int(y)  # trunc
        y -= f
        a, c = f * a + c, a
        b, d = f * b + d, b
        if max(abs(a), abs(b)) > m:
            return c, d
        if b != 0 and float(a) / float(b) == x:
            break
        if y == 0:
            break
        y = 1.0 / y
    return a, b


def julia_range(start, step, n):
    """Element values of Julia ``range(start, step=step, length=n)``."""
    sn, sd = _rat(start)
    tn, td = _rat(step)
    if sd != 0 and td != 0 and sn / sd == start and tn / td == step:
        den = sd * td // math.gcd(sd, td)
        m = 2.0 ** 53
        if abs(den * start) <= m and abs(den * step) <= m and den % sd == 0 and den % td == 0:
            s0, st = round(den * start), round(den * step)
            return np.array([float(Fraction(s0 + i * st, den)) for i in range(n)])
    fs, ft = Fraction(start), Fraction(step)
    return np.array([float(fs + i * ft) for i in range(n)])


def julia_linrange(a, b, n):
    """Element values of Julia ``range(a, b, length=n)``."""
    if n == 1:
        return np.array([a])
    return julia_range(a, (b - a) / (n - 1), n) if False else np.array(
        [float(Fraction(a) * Fraction(n - 1 - i, n - 1) + Fraction(b) * Fraction(i, n - 1)) for i in range(n)])


def grid(p):
    """The ``grid`` NamedTuple returned on rank 0 (src/simulation_runner.jl:718-729)."""
    xmin, xmax, ymin, ymax, zmin, zmax = extents(p)
    g = grid_spacing(p)
    return dict(x=julia_linrange(xmin, xmax, p["Nx"] + 1), y=julia_linrange(ymin, ymax, p["Ny"] + 1),
                z=julia_linrange(zmin, zmax, p["Nz"] + 1), dx=g["dx"], dy=g["dy"], dz=g["dz"],
                xm=julia_range(xmin + g["dx"] / 2, g["dx"], p["Nx"]),
                ym=julia_range(ymin + g["dy"] / 2, g["dy"], p["Ny"]),
                zm=julia_range(zmin + g["dz"] / 2, g["dz"], p["Nz"]))


# -------------------------------------------------------- Gaussian moments
def _binom(n, k):
    return math.comb(n, k)


def gaussian_moments(rho, u, v, w, C200, C110, C101, C020, C011, C002):
    """InitializeM4_35: raw moments (order <= 4) of a Gaussian, 35-vector.

    The central moments are those of X = A Z, A = sqrt(C2) (symmetric root),
    Z standard normal; for a diagonal covariance A = diag(sqrt(Cii)) and the
    fourth-order central moment is S400 * (A11^2)^2 as in the reference's
    S4toC4_3D_r expansion.
    """
    Z = {}  # standardized moments of the standard normal up to order 4
    for (i, j, k) in E35:
        def m1(n):
            return {0: 1.0, 1: 0.0, 2: 1.0, 3: 0.0, 4: 3.0}[n]
        Z[(i, j, k)] = m1(i) * m1(j) * m1(k)
    C = {}
    if C110 == 0 and C101 == 0 and C011 == 0:
        a = [math.sqrt(C200), math.sqrt(C020), math.sqrt(C002)]
        pw = [[1.0, x, x * x, x * x * x, (x * x) * (x * x)] for x in a]
        for (i, j, k) in E35:
            C[(i, j, k)] = Z[(i, j, k)] * pw[0][i] * pw[1][j] * pw[2][k]
    else:
        C2 = np.array([[C200, C110, C101], [C110, C020, C011], [C101, C011, C002]])
        lam, V = np.linalg.eigh(C2)
        A = (V * np.sqrt(np.maximum(lam, 0.0))) @ V.T
        Zf = lambda c: Z.get(tuple(c), 0.0) if sum(c) <= 4 else 0.0  # noqa: E731
        for e in E35:
            rows = [r for r in range(3) for _ in range(e[r])]
            s = 0.0
            for code in range(3 ** len(rows)):
                cnt, coef, cc = [0, 0, 0], 1.0, code
                for r in rows:
                    col = cc % 3
                    cc //= 3
                    cnt[col] += 1
                    coef *= A[r, col]
                s += coef * Zf(cnt)
            C[e] = s
    C[(0, 0, 0)] = 1.0
    C[(1, 0, 0)] = C[(0, 1, 0)] = C[(0, 0, 1)] = 0.0
    M = np.zeros(35)
    pu = [u ** n for n in range(5)]
    pv = [v ** n for n in range(5)]
    pw_ = [w ** n for n in range(5)]
    for n, (i, j, k) in enumerate(E35):
        s = 0.0
        for a_ in range(i + 1):
            for b in range(j + 1):
                for c in range(k + 1):
                    if a_ + b + c == 1:
                        continue
                    s += _binom(i, a_) * _binom(j, b) * _binom(k, c) * C[(a_, b, c)] * (pu[i - a_] * pv[j - b] * pw_[k - c])
        M[n] = rho * s
    return M


def region_to_moments(region, r110=0.0, r101=0.0, r011=0.0):
    """src/initial_conditions.jl:224-238."""
    T = region.temperature
    C200 = C020 = C002 = T
    return gaussian_moments(region.density, region.velocity[0], region.velocity[1], region.velocity[2], C200,
                            r110 * math.sqrt(C200 * C020), r101 * math.sqrt(C200 * C002), C020,
                            r011 * math.sqrt(C020 * C002), C002)


def cell_overlaps_cube(cc, cs, cube):
    """src/initial_conditions.jl:281-302 (strict inequalities)."""
    if any(math.isinf(wv) for wv in cube.width):
        return True
    for q in range(3):
        x, dxq, cq, wq = cc[q], cs[q], cube.center[q], cube.width[q]
        if not (max(x - dxq / 2, cq - wq / 2) < min(x + dxq / 2, cq + wq / 2)):
            return False
    return True


# ------------------------------------------------------ jet configurations
def jet_configuration(name, p):
    """get_jet_configuration (examples/run_3d_custom_jets.jl:64-272)."""
    xmin, xmax, ymin, ymax, zmin, zmax = extents(p)
    xc, yc, zc = (xmin + xmax) / 2, (ymin + ymax) / 2, (zmin + zmax) / 2
    Lx = xmax - xmin
    Ma, rhol, rhor, T = p["Ma"], p["rhol"], p["rhor"], p["T"]
    jet_width = p.get("jet_size", 0.1) * Lx
    off_mult = p.get("offset_mult", 0.6)
    inf = float("inf")
    bg = CubicRegion((xc, yc, zc), (inf, inf, inf), rhor, (0.0, 0.0, 0.0), T)
    W = (jet_width, jet_width, jet_width)
    if name == "crossing":
        Uc = Ma / math.sqrt(3.0)
        o = jet_width * off_mult
        jets = [CubicRegion((xc - o, yc - o, zc + o), W, rhol, (Uc, Uc, -Uc), T),
                CubicRegion((xc + o, yc + o, zc - o), W, rhol, (-Uc, -Uc, Uc), T)]
    elif name == "crossing2D":
        Uc = Ma / math.sqrt(2.0)
        o = jet_width * off_mult
        jets = [CubicRegion((xc - o, yc - o, zc), W, rhol, (Uc, Uc, 0.0), T),
                CubicRegion((xc + o, yc + o, zc), W, rhol, (-Uc, -Uc, 0.0), T)]
    elif name == "triple-jet":
        Uc = Ma
        o = jet_width * 1.2
        jets = [CubicRegion((xc, yc, zc), W, rhol, (Uc, 0.0, 0.0), T),
                CubicRegion((xc - o, yc, zc), W, rhol, (0.0, Uc, 0.0), T),
                CubicRegion((xc + o, yc, zc), W, rhol, (0.0, -Uc, 0.0), T)]
    else:
        raise ValueError("unknown jet configuration: %s" % name)
    return bg, jets


# ------------------------------------------------------------- IC builders
def hardcoded_ic(p):
    """The runner's built-in crossing cubes (src/simulation_runner.jl:200-271)."""
    Nx, Ny, Nz = p["Nx"], p["Ny"], p["Nz"]
    T = p["T"]
    r110, r101, r011 = p.get("r110", 0.0), p.get("r101", 0.0), p.get("r011", 0.0)
    C2 = (T, r110 * math.sqrt(T * T), r101 * math.sqrt(T * T), T, r011 * math.sqrt(T * T), T)
    bg = gaussian_moments(p["rhor"], 0.0, 0.0, 0.0, *C2)
    Uc = p["Ma"] / math.sqrt(2.0)
    Mt = gaussian_moments(p["rhol"], -Uc, -Uc, 0.0, *C2)
    Mb = gaussian_moments(p["rhol"], Uc, Uc, 0.0, *C2)
    Cx, Cy = int(math.floor(0.1 * Nx)), int(math.floor(0.1 * Ny))
    Mint_x, Maxt_x, Minb_x, Maxb_x = Nx // 2 + 1, Nx // 2 + 1 + Cx, Nx // 2 - Cx, Nx // 2
    Mint_y, Maxt_y, Minb_y, Maxb_y = Ny // 2 + 1, Ny // 2 + 1 + Cy, Ny // 2 - Cy, Ny // 2
    Cz = min(Cx, Cy)
    Mint_z, Maxt_z = Nz // 2 + 1 - Cz // 2, Nz // 2 + 1 + Cz // 2
    gi = np.arange(1, Nx + 1)[:, None, None]
    gj = np.arange(1, Ny + 1)[None, :, None]
    gk = np.arange(1, Nz + 1)[None, None, :]
    inz = (gk >= Mint_z) & (gk <= Maxt_z)
    bot = (gi >= Minb_x) & (gi <= Maxb_x) & (gj >= Minb_y) & (gj <= Maxb_y) & inz
    top = (gi >= Mint_x) & (gi <= Maxt_x) & (gj >= Mint_y) & (gj <= Maxt_y) & inz
    M = np.empty((Nx, Ny, Nz, 35), order="F")
    M[...] = bg
    M[bot] = Mb
    M[top] = Mt
    return M


def custom_ic(p, background, jets):
    """initialize_moment_field_mpi for one rank (src/initial_conditions.jl:152-217)."""
    Nx, Ny, Nz = p["Nx"], p["Ny"], p["Nz"]
    g = grid(p)
    xm, ym, zm = g["xm"], g["ym"], g["zm"]
    r = (p.get("r110", 0.0), p.get("r101", 0.0), p.get("r011", 0.0))
    dx = abs(xm[1] - xm[0]) if Nx > 1 else 0.0
    dy = abs(ym[1] - ym[0]) if Ny > 1 else 0.0
    dz = abs(zm[1] - zm[0]) if Nz > 1 else 0.0
    bgM = region_to_moments(background, *r)
    jetM = [region_to_moments(j, *r) for j in jets]

    def mask1(coords, d, q, jet):
        c, wq = jet.center[q], jet.width[q]
        return np.array([max(x - d / 2, c - wq / 2) < min(x + d / 2, c + wq / 2) for x in coords])

    M = np.empty((Nx, Ny, Nz, 35), order="F")
    M[...] = bgM
    for jet, Mj in zip(jets, jetM):
        if any(math.isinf(wv) for wv in jet.width):
            M[...] = Mj
            continue
        mx, my, mz = mask1(xm, dx, 0, jet), mask1(ym, dy, 1, jet), mask1(zm, dz, 2, jet)
        sel = mx[:, None, None] & my[None, :, None] & mz[None, None, :]
        M[sel] = Mj
    return M


def initial_state(p):
    """The IC ``simulation_runner`` builds (custom regions when use_custom_ic)."""
    if p.get("use_custom_ic", False):
        return custom_ic(p, p["ic_background"], list(p["ic_jets"]))
    return hardcoded_ic(p)


def with_jets(p, config="crossing"):
    """params merged with a named jet configuration, as the example scripts do."""
    bg, jets = jet_configuration(config, p)
    q = dict(p)
    q.update(ic_background=bg, ic_jets=jets, use_custom_ic=True, config=config)
    return q


def ic_tables(p):
    """The tables of the device IC fill (hyq_set_state_ic) that reproduce
    initial_state(p): (xm, ym, zm, dx, dy, dz, bg[35], regions, moments[35 x R]);
    a region is (kind, everywhere, lo[3], hi[3], (i0, i1, j0, j1, k0, k1))."""
    Nx, Ny, Nz = p["Nx"], p["Ny"], p["Nz"]
    g = grid(p)
    xm, ym, zm = g["xm"], g["ym"], g["zm"]
    if p.get("use_custom_ic", False):
        background, jets = p["ic_background"], list(p["ic_jets"])
        r = (p.get("r110", 0.0), p.get("r101", 0.0), p.get("r011", 0.0))
        dx = abs(xm[1] - xm[0]) if Nx > 1 else 0.0
        dy = abs(ym[1] - ym[0]) if Ny > 1 else 0.0
        dz = abs(zm[1] - zm[0]) if Nz > 1 else 0.0
        bg = region_to_moments(background, *r)
        regions, moments = [], []
        for jet in jets:
            every = any(math.isinf(wv) for wv in jet.width)
            lo = [0.0, 0.0, 0.0] if every else [jet.center[q] - jet.width[q] / 2 for q in range(3)]
            hi = [0.0, 0.0, 0.0] if every else [jet.center[q] + jet.width[q] / 2 for q in range(3)]
            regions.append((0, int(every), lo, hi, (0, -1, 0, -1, 0, -1)))
            moments.append(region_to_moments(jet, *r))
        return xm, ym, zm, dx, dy, dz, bg, regions, moments
    T = p["T"]
    r110, r101, r011 = p.get("r110", 0.0), p.get("r101", 0.0), p.get("r011", 0.0)
    C2 = (T, r110 * math.sqrt(T * T), r101 * math.sqrt(T * T), T, r011 * math.sqrt(T * T), T)
    bg = gaussian_moments(p["rhor"], 0.0, 0.0, 0.0, *C2)
    Uc = p["Ma"] / math.sqrt(2.0)
    Mt = gaussian_moments(p["rhol"], -Uc, -Uc, 0.0, *C2)
    Mb = gaussian_moments(p["rhol"], Uc, Uc, 0.0, *C2)
    Cx, Cy = int(math.floor(0.1 * Nx)), int(math.floor(0.1 * Ny))
    Mint_x, Maxt_x, Minb_x, Maxb_x = Nx // 2 + 1, Nx // 2 + 1 + Cx, Nx // 2 - Cx, Nx // 2
    Mint_y, Maxt_y, Minb_y, Maxb_y = Ny // 2 + 1, Ny // 2 + 1 + Cy, Ny // 2 - Cy, Ny // 2
    Cz = min(Cx, Cy)
    Mint_z, Maxt_z = Nz // 2 + 1 - Cz // 2, Nz // 2 + 1 + Cz // 2
    zero3 = [0.0, 0.0, 0.0]
    regions = [(1, 0, zero3, zero3, (Minb_x - 1, Maxb_x - 1, Minb_y - 1, Maxb_y - 1, Mint_z - 1, Maxt_z - 1)),
               (1, 0, zero3, zero3, (Mint_x - 1, Maxt_x - 1, Mint_y - 1, Maxt_y - 1, Mint_z - 1, Maxt_z - 1))]
    return xm, ym, zm, 0.0, 0.0, 0.0, bg, regions, [Mb, Mt]
