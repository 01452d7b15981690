"""Parity at the full sizes of the benchmark workloads, on step prefixes.

* The 1024 x 1024 liquid column (the bench workload: two-phase, linear EOS linearised from
  the stiffened-gas data at density ratio 1000, WENO-Z, HLLC, limiter, characteristic,
  SSP-RK3, CFL 0.5): FP64_STRICT equals the oracle bit for bit after 3 steps, and the
  unmodified compiled reference (4 slab ranks, its own grid rounding) after 2 steps; FP64
  agrees with the oracle to FAST_RTOL of max |U|.
* The 512 x 512 Euler four-quadrant problem with outflow boundaries (WENO-Z, HLLC,
  conservative, CFL 0.4): FP64_STRICT equals the oracle bit for bit after 10 steps, FP64
  within FAST_RTOL.  The reference has no Euler system; the oracle is the restatement.
* FP32-bulk on the same prefixes: pooled relative L1 against the oracle below FP32_RTOL_L1.

The oracle runs on all host threads (the column's 3 steps take a few seconds).
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import BC_OUTFLOW, EQ_EULER, Problem, reference_available, run_reference
import cases

pytestmark = pytest.mark.gpu
FAST_RTOL = 3e-11    # max |FP64 - oracle| / max |U| (as the small-grid parity tests)
FP32_RTOL_L1 = 1e-6  # pooled relative L1 of FP32-bulk against the oracle on these prefixes
THREADS = os.cpu_count() or 1


def rel_max(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def run_gpu(wb, p: Problem, U0, precision, steps):
    cfg = wb.make_config(p.nx, p.ny, bc=p.bc, rk=p.rk, cfl=p.cfl, scheme=p.scheme, limiter=p.limiter, flux=p.flux,
                         recon=p.recon, ref_slabs=p.ref_slabs, precision=precision)
    eq = wb.make_eq(kind=p.eq_kind, rho10=p.rho10, rho20=p.rho20, sound1=p.sound1, sound2=p.sound2, gamma=p.gamma)
    with wb.Solver(cfg, eq) as s:
        s.upload(U0)
        t, n = s.advance(1e9, max_steps=steps)
        assert n == steps
        return s.download(), t


@pytest.fixture(scope="module")
def column1024():
    U0, prm = cases.liquid_column(1024, 1024, seed=3)
    return U0, prm


def test_column_1024_equals_oracle(wb, oracle_lib, column1024):
    U0, prm = column1024
    p = Problem(nx=1024, ny=1024, rk=2, cfl=0.5, scheme=1, flux=1, recon=1, limiter=1, threads=THREADS, **prm)
    V, n, t, _ = oracle_lib.advance(p, U0, t_end=1e9, max_steps=3)
    assert n == 3
    U, tg = run_gpu(wb, p, U0, wb.FP64_STRICT, 3)
    assert tg == t and np.array_equal(U, V)
    U, _ = run_gpu(wb, p, U0, wb.FP64, 3)
    assert rel_max(U, V) <= FAST_RTOL
    U, _ = run_gpu(wb, p, U0, wb.FP32_BULK, 3)
    assert rel_l1(U, V) <= FP32_RTOL_L1
    assert (U[0] > 0).all() and (U[1] > 0).all()


@pytest.mark.skipif(not reference_available(), reason="the compiled reference is not built here")
def test_column_1024_equals_compiled_reference(wb, column1024):
    U0, prm = column1024
    p = Problem(nx=1024, ny=1024, rk=2, cfl=0.5, scheme=1, flux=1, recon=1, limiter=1, ref_slabs=4, **prm)
    r = run_reference(p, testcase=2, U0=U0, steps=2, timeout=1200)
    U, _ = run_gpu(wb, p, U0, wb.FP64_STRICT, 2)
    assert np.array_equal(U, r.U)


def test_euler_512_equals_oracle(wb, oracle_lib):
    U0, _ = cases.euler_quadrants(512, 512, seed=2)
    p = Problem(nx=512, ny=512, bc=BC_OUTFLOW, eq_kind=EQ_EULER, rk=2, cfl=0.4, scheme=1, flux=1, recon=0,
                threads=THREADS)
    V, n, t, _ = oracle_lib.advance(p, U0, t_end=1e9, max_steps=10)
    assert n == 10
    U, tg = run_gpu(wb, p, U0, wb.FP64_STRICT, 10)
    assert tg == t and np.array_equal(U, V)
    U, _ = run_gpu(wb, p, U0, wb.FP64, 10)
    assert rel_max(U, V) <= FAST_RTOL
    U, _ = run_gpu(wb, p, U0, wb.FP32_BULK, 10)
    assert rel_l1(U, V) <= FP32_RTOL_L1
