"""Seeded synthetic workloads of the WENOFV hot path (the shapes of BASELINE's configs).

Initial cell averages use the 4x4 Gauss-Legendre rule of CWENOFV::initializeAve
(src/WENOFV.cpp:232-279).  Everything is drawn from numpy's PCG64 with the seeds given; the
arrays are SoA ``U[v, j, i]``.
"""
from __future__ import annotations

import math

import numpy as np

# 4-point Gauss-Legendre rule (third_party/scTools/GaussQuadratureInRef.hpp:64-75)
GLEG_X = np.array([-0.861136311594052575223946488893, -0.339981043584856264802665759103,
                   0.339981043584856264802665759103, 0.861136311594052575223946488893])
GLEG_W = np.array([0.347854845137453857373063949222, 0.652145154862546142626936050778,
                   0.652145154862546142626936050778, 0.347854845137453857373063949222])


def cell_average(f, nx, ny, xl=0.0, xr=1.0, yl=0.0, yr=1.0):
    """average of f(x, y) -> (nv, ...) over every cell with the 4x4 Gauss-Legendre rule"""
    dx, dy = (xr - xl) / nx, (yr - yl) / ny
    xc = xl + (np.arange(nx) + 0.5) * dx
    yc = yl + (np.arange(ny) + 0.5) * dy
    acc = None
    for a in range(4):
        for b in range(4):
            X = xc[None, :] + 0.5 * dx * GLEG_X[a]
            Y = yc[:, None] + 0.5 * dy * GLEG_X[b]
            X, Y = np.broadcast_arrays(X, Y)
            v = np.asarray(f(X, Y)) * (0.25 * GLEG_W[a] * GLEG_W[b])
            acc = v if acc is None else acc + v
    return np.ascontiguousarray(acc, dtype=np.float64)


# ---- config 1: scalar linear advection u_t + u_x + u_y = 0 --------------------------------
def advection_sine(nx, ny):
    return cell_average(lambda x, y: np.sin(2 * np.pi * (x + y))[None], nx, ny)


# ---- config 2: Euler four-quadrant Riemann problem ----------------------------------------
def euler_quadrants(nx, ny, seed=2, gamma=1.4):
    rng = np.random.default_rng(seed)
    q = []
    for _ in range(4):
        rho = rng.uniform(0.1, 1.5)
        p = rng.uniform(0.03, 1.5)
        u, v = rng.uniform(-1.2, 1.2, size=2)
        q.append((rho, u, v, p))

    def f(x, y):
        k = (x >= 0.5).astype(int) + 2 * (y >= 0.5).astype(int)
        out = np.zeros((4,) + x.shape)
        for m, (rho, u, v, p) in enumerate(q):
            sel = k == m
            out[0][sel] = rho
            out[1][sel] = rho * u
            out[2][sel] = rho * v
            out[3][sel] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
        return out

    return cell_average(f, nx, ny), q


# ---- config 3: two-phase liquid column ------------------------------------------------------
def column_params(ratio=1000.0, g1=4.4, pinf1=6e3, g2=1.4, pinf2=0.0, p0=1.0, rho2=1.0):
    """linear-EOS parameters of the reference's TwoPhaseEquation from the stiffened-gas data,
    linearised at pressure p0: c_k^2 = gamma_k (p0 + pinf_k) / rho_k0"""
    rho1 = ratio * rho2
    return dict(rho10=rho1, rho20=rho2, sound1=math.sqrt(g1 * (p0 + pinf1) / rho1),
                sound2=math.sqrt(g2 * (p0 + pinf2) / rho2))


def periodic_field(rng, nk=3):
    """a smooth periodic Gaussian random field on [0,1]^2 with unit RMS"""
    ks = [(a, b) for a in range(-nk, nk + 1) for b in range(-nk, nk + 1) if (a, b) != (0, 0)]
    amp = rng.standard_normal((len(ks), 2)) / math.sqrt(len(ks))

    C = np.zeros((2 * nk + 1, 2 * nk + 1))
    D = np.zeros_like(C)
    for (a, b), (c, d) in zip(ks, amp):
        C[b + nk, a + nk], D[b + nk, a + nk] = c, d
    waves = np.arange(-nk, nk + 1)

    def f(x, y):
        x, y = np.asarray(x, dtype=np.float64), np.asarray(y, dtype=np.float64)
        if x.ndim == 2 and x.shape == y.shape and np.all(x == x[:1, :]) and np.all(y == y[:, :1]):
            # tensor-product points: cos/sin(2 pi (a x + b y)) by the angle-sum identities,
            # summed over the modes as small matrix products
            px, py = 2 * np.pi * waves[:, None] * x[0][None, :], 2 * np.pi * waves[:, None] * y[:, 0][None, :]
            cx, sx, cy, sy = np.cos(px), np.sin(px), np.cos(py), np.sin(py)
            s = cy.T @ C @ cx - sy.T @ C @ sx + sy.T @ D @ cx + cy.T @ D @ sx
            return s * math.sqrt(2.0)
        s = np.zeros_like(x)
        for (a, b), (c, d) in zip(ks, amp):
            ph = 2 * np.pi * (a * x + b * y)
            s = s + c * np.cos(ph) + d * np.sin(ph)
        return s * math.sqrt(2.0)

    return f


def liquid_column(nx, ny, seed=3, ratio=1000.0, radius=0.2, eps=1e-6, amp=1e-2, p0=1.0, params=None):
    """disk of phase 1 at (0.5, 0.5) in phase 2, tanh-smoothed over 2 cells, pressure p0,
    velocity = amp x seeded periodic Gaussian fields; the smoothing width is 2 cells of the
    coarser direction (a thinner front on a stretched grid is a discontinuity that the
    reference's scheme does not survive: it then blows up within ~50 steps)"""
    prm = params or column_params(ratio=ratio, p0=p0)
    rng = np.random.default_rng(seed)
    fu, fv = periodic_field(rng), periodic_field(rng)
    h = max(1.0 / nx, 1.0 / ny)
    rho1 = p0 / prm["sound1"] ** 2 + prm["rho10"]  # getU0, include/Equations.hpp:987-988 (g_preb = 0)
    rho2 = p0 / prm["sound2"] ** 2 + prm["rho20"]

    def f(x, y):
        r = np.hypot(x - 0.5, y - 0.5)
        z1 = eps + (1 - 2 * eps) * 0.5 * (1 - np.tanh((r - radius) / (2 * h)))
        a1, a2 = z1 * rho1, (1 - z1) * rho2
        rho = a1 + a2
        return np.stack([a1, a2, rho * amp * fu(x, y), rho * amp * fv(x, y)])

    return cell_average(f, nx, ny), prm


def sg_params(ratio=1000.0, g1=4.4, pinf1=6e3, g2=1.4, pinf2=0.0, p0=1.0, rho2=1.0):
    """stiffened-gas parameters (eq kind 3): phase k on its isentrope through (p0, rho_k0)"""
    return dict(rho10=ratio * rho2, rho20=rho2, preb=p0, gamma1=g1, pinf1=pinf1, gamma2=g2, pinf2=pinf2)


def sg_column(nx, ny, seed=3, ratio=1000.0, radius=0.2, eps=1e-6, amp=1e-2, p0=1.0):
    """the liquid column of liquid_column with stiffened-gas phases at the uniform pressure
    p0, where the phase densities are rho10 and rho20 themselves"""
    prm = sg_params(ratio=ratio, p0=p0)
    rng = np.random.default_rng(seed)
    fu, fv = periodic_field(rng), periodic_field(rng)
    h = max(1.0 / nx, 1.0 / ny)

    def f(x, y):
        r = np.hypot(x - 0.5, y - 0.5)
        z1 = eps + (1 - 2 * eps) * 0.5 * (1 - np.tanh((r - radius) / (2 * h)))
        a1, a2 = z1 * prm["rho10"], (1 - z1) * prm["rho20"]
        rho = a1 + a2
        return np.stack([a1, a2, rho * amp * fu(x, y), rho * amp * fv(x, y)])

    return cell_average(f, nx, ny), prm


def point_column(nx, ny, seed=3, ratio=1000.0, radius=0.2, eps=1e-6, amp=1e-2, p0=1.0):
    """the liquid column sampled at cell centres with a one-mode-ring velocity field: the
    same physics as liquid_column, cheap enough to build thousands of grids for serving"""
    prm = column_params(ratio=ratio, p0=p0)
    rng = np.random.default_rng(seed)
    fu, fv = periodic_field(rng, nk=1), periodic_field(rng, nk=1)
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    rho1 = p0 / prm["sound1"] ** 2 + prm["rho10"]
    rho2 = p0 / prm["sound2"] ** 2 + prm["rho20"]
    r = np.hypot(X - 0.5, Y - 0.5)
    z1 = eps + (1 - 2 * eps) * 0.5 * (1 - np.tanh((r - radius) / (2.0 * max(1.0 / nx, 1.0 / ny))))
    a1, a2 = z1 * rho1, (1 - z1) * rho2
    rho = a1 + a2
    return np.ascontiguousarray(np.stack([a1, a2, rho * amp * fu(X, Y), rho * amp * fv(X, Y)])), prm


# ---- batched ensemble (config 4) ------------------------------------------------------------
BATCH_GRIDS = [(64, 64), (96, 96), (128, 128), (192, 192), (256, 256), (256, 64), (512, 128)]


def ensemble(n, seed=4, grids=None):
    """n two-phase columns with seeded grid, radius in [0.1,0.3], density ratio in [10,1000],
    eps in {1e-8, 1e-6} and WENO-JS/WENO-Z mixed; returns a list of (U0, params dict)"""
    rng = np.random.default_rng(seed)
    grids = grids or BATCH_GRIDS
    out = []
    for k in range(n):
        nx, ny = grids[rng.integers(len(grids))]
        r = rng.uniform(0.1, 0.3)
        ratio = rng.uniform(10, 1000)
        eps = [1e-8, 1e-6][rng.integers(2)]
        scheme = int(rng.integers(2))
        U0, prm = liquid_column(nx, ny, seed=1000 + k, ratio=ratio, radius=r, eps=eps)
        out.append((U0, dict(prm, nx=nx, ny=ny, scheme=scheme, radius=r, ratio=ratio, eps=eps)))
    return out


def periodic_frame(U):
    """NEUMANN2 ghost frame [nv][ny+8][nx+8] holding the periodic wrap of U, cell (i, j) at
    [v][j+4][i+4] (the interior entries are U itself; the solvers do not read them)."""
    nv, ny, nx = U.shape
    jj = np.arange(-4, ny + 4) % ny
    ii = np.arange(-4, nx + 4) % nx
    return np.ascontiguousarray(U[:, jj][:, :, ii])
