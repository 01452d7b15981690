"""The stiffened-gas two-phase model (WENOFV_EQ_TWO_PHASE_SG) on the GPU against the oracle.

The model is an extension (the reference has the linear EOS only), so the oracle's
restatement is the only reference.  Its pressure equilibrium calls pow, whose CUDA and C
library results differ by a few ulp, and the Newton iteration may stop one step apart, so
the tolerances are stated instead of bit equality:

* pointwise fluxes and eigenvectors: FP64_STRICT within 1e-12 of the state's scale, FP64
  within 1e-11;
* a few RK steps of a 64x48 column: FP64_STRICT within 1e-12 of max |U|, FP64 within 1e-10,
  the CFL time step within 100 times those (the equilibrium pressure carries the liquid's
  density rounding times rho_1 c_1^2, which the gas of a mixed cell feels relative to p ~ 1);
* conservation to roundoff and positive partial densities on a 256^2 column.
"""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle import EQ_TWO_PHASE_SG, Problem
from test_oracle import sg_states

pytestmark = pytest.mark.gpu


def sg_eq(wb):
    prm = cases.sg_params()
    return wb.make_eq(kind=wb.EQ_TWO_PHASE_SG, rho10=prm["rho10"], rho20=prm["rho20"], preb=prm["preb"],
                      gamma1=prm["gamma1"], pinf1=prm["pinf1"], gamma2=prm["gamma2"], pinf2=prm["pinf2"]), prm


@pytest.mark.parametrize("flux", [0, 1])
@pytest.mark.parametrize("normal", [(1.0, 0.0), (0.0, 1.0)])
def test_sg_riemann_probe(wb, oracle_lib, flux, normal):
    rng = np.random.default_rng(11)
    UL, _, _ = sg_states(rng, 600)
    UR, _, _ = sg_states(rng, 600)
    eq, prm = sg_eq(wb)
    p = Problem(nx=8, ny=8, eq_kind=EQ_TWO_PHASE_SG, **prm)
    ref = np.array([oracle_lib.riemann(p, flux, a, b, *normal) for a, b in zip(UL, UR)])
    scale = np.abs(ref).max(axis=1, keepdims=True) + np.abs(UL).max(axis=1, keepdims=True)
    strict = wb.probe_riemann(eq, flux, UL, UR, *normal, precision=wb.FP64_STRICT)
    assert np.all(np.abs(strict - ref) <= 1e-12 * scale)
    fast = wb.probe_riemann(eq, flux, UL, UR, *normal, precision=wb.FP64)
    assert np.all(np.abs(fast - ref) <= 1e-11 * scale)


@pytest.mark.parametrize("normal", [(1.0, 0.0), (0.0, 1.0)])
def test_sg_eigen_probe(wb, oracle_lib, normal):
    U, _, _ = sg_states(np.random.default_rng(12), 300)
    eq, prm = sg_eq(wb)
    p = Problem(nx=8, ny=8, eq_kind=EQ_TWO_PHASE_SG, **prm)
    L, R = wb.probe_eigen(eq, U, *normal, precision=wb.FP64_STRICT)
    for k in range(len(U)):
        Lr, Rr = oracle_lib.eigen(p, U[k], *normal)
        assert np.abs(L[k] - Lr).max() <= 1e-10 * (np.abs(Lr).max() + 1.0)
        assert np.abs(R[k] - Rr).max() <= 1e-10 * (np.abs(Rr).max() + 1.0)


@pytest.mark.parametrize("recon,flux", [(1, 1), (0, 1), (1, 0), (0, 0)])
def test_sg_column_against_oracle(wb, oracle_lib, recon, flux):
    nx, ny = 64, 48
    U0, prm = cases.sg_column(nx, ny, seed=8)
    p = Problem(nx=nx, ny=ny, eq_kind=EQ_TWO_PHASE_SG, scheme=1, flux=flux, recon=recon, limiter=1, **prm)
    V, n, t, dts = oracle_lib.advance(p, U0, t_end=1e9, max_steps=5)
    eq, _ = sg_eq(wb)
    for prec, tol in ((wb.FP64_STRICT, 1e-12), (wb.FP64, 1e-10)):
        cfg = wb.make_config(nx, ny, scheme=1, flux=flux, recon=recon, limiter=1, precision=prec)
        with wb.Solver(cfg, eq) as s:
            s.upload(U0)
            # a relative 1e-16 in the liquid's density is 1e-16 rho_1 c_1^2 ~ 3e-12 in the pressure,
            # which the gas of a mixed cell feels relative to p ~ 1
            assert abs(s.compute_dt() - dts[0]) <= 100 * tol * dts[0]
            t2, n2 = s.advance(1e9, max_steps=5)
            assert n2 == n and abs(t2 - t) <= 1e-12 * t
            U = s.download()
            assert s.status()[0] == 0
        assert np.abs(U - V).max() <= tol * np.abs(V).max(), (prec, np.abs(U - V).max() / np.abs(V).max())


def test_sg_column_256_conservation_and_bounds(wb):
    U0, prm = cases.sg_column(256, 256, seed=3)
    eq, _ = sg_eq(wb)
    cfg = wb.make_config(256, 256, scheme=1, flux=1, recon=1, limiter=1, precision=wb.FP64)
    with wb.Solver(cfg, eq) as s:
        s.upload(U0)
        s.advance(1e9, max_steps=50)
        U = s.download()
        assert s.status()[0] == 0
    m0, m1 = U0.sum(axis=(1, 2)), U.sum(axis=(1, 2))
    assert np.all(np.abs(m1 - m0) <= 1e-12 * np.abs(U0).sum(axis=(1, 2)))
    assert (U[0] > 0).all() and (U[1] > 0).all()
