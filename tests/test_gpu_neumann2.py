"""NEUMANN2 (BOUNDARYTYPE 3, "boundary from the initial data", include/Equations.hpp:30): the
ghost cells come from a fixed frame of averages that the caller sets once.  The reference
declares the kind (ZALESAK selects it, include/Equations.hpp:696) but setBoundaryAverages2
(src/WENOFV.cpp:2249-2295) has no branch for it, so parity is held to the oracle's restatement
of the rule: FP64_STRICT bit for bit, through the C ABI, on grids from narrower than the halo
up to ragged sizes, in a context and in a batch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import BC_NEUMANN2, BC_PERIOD, EQ_EULER, EQ_LINEAR_ADV, Problem
import cases

pytestmark = pytest.mark.gpu


def _solver(wb, p: Problem, precision):
    cfg = wb.make_config(p.nx, p.ny, bc=p.bc, rk=p.rk, cfl=p.cfl, scheme=p.scheme, limiter=p.limiter, flux=p.flux,
                         recon=p.recon, precision=precision)
    eq = wb.make_eq(kind=p.eq_kind, rho10=p.rho10, rho20=p.rho20, sound1=p.sound1, sound2=p.sound2,
                    gamma=p.gamma, adv_u=p.adv_u, adv_v=p.adv_v, gravity=p.gravity)
    return wb.Solver(cfg, eq)


def _runs(nx, ny):
    # the frame is the periodic wrap of a second, differently seeded state: ghost values that
    # no interior rule reproduces
    mild = dict(ratio=2.0, eps=0.05) if min(nx, ny) < 8 else {}
    U0, prm = cases.liquid_column(nx, ny, seed=nx * 10 + ny, **mild)
    F0, _ = cases.liquid_column(nx, ny, seed=nx * 10 + ny + 1, **mild)
    E0, _ = cases.euler_quadrants(nx, ny, seed=4)
    EF, _ = cases.euler_quadrants(nx, ny, seed=5)
    A0 = cases.advection_sine(nx, ny)
    fr = cases.periodic_frame
    return [(Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(F0), scheme=1, flux=1, recon=1, limiter=1, gravity=9.81, **prm), U0),
            (Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(F0), scheme=2, flux=0, recon=0, limiter=1, **prm), U0),
            (Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(F0), scheme=1, flux=1, recon=3, limiter=1, **prm), U0),
            (Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(F0), scheme=2, flux=1, recon=2, limiter=1, **prm), U0),
            (Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(EF), eq_kind=EQ_EULER, scheme=1, flux=1, recon=1, cfl=0.4), E0),
            (Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=fr(A0[:, ::-1].copy()), eq_kind=EQ_LINEAR_ADV, scheme=0, flux=0,
                     recon=0), A0)]


@pytest.mark.parametrize("nx,ny", [(3, 2), (8, 8), (27, 5), (53, 70)])
def test_neumann2_strict(wb, oracle_lib, nx, ny):
    for p, X0 in _runs(nx, ny):
        with oracle_lib.cube_rounded():
            V, *_ = oracle_lib.advance(p, X0, t_end=1e9, max_steps=3)
            R = oracle_lib.rhs(p, X0)
        with _solver(wb, p, wb.FP64_STRICT) as s:
            s.set_frame(p.frame)
            s.upload(X0)
            if p.nx * p.ny > 100:
                assert np.array_equal(s.rhs(), R), (p.eq_kind, p.scheme, p.recon)
            s.upload(X0)
            s.advance(1e9, max_steps=3)
            assert s.status()[0] == 0
            assert np.array_equal(s.download(), V), (p.eq_kind, p.scheme, p.recon)


def test_neumann2_fast_forms(wb, oracle_lib):
    nx, ny = 53, 70
    p, U0 = _runs(nx, ny)[0]
    V, *_ = oracle_lib.advance(p, U0, t_end=1e9, max_steps=5)
    # stated bounds: FP64 contracted, max norm 1e-10 of max |V|; FP32-bulk, pooled relative
    # L1 1e-6 (the bar of the periodic FP32-bulk tests)
    with _solver(wb, p, wb.FP64) as s:
        s.set_frame(p.frame)
        s.upload(U0)
        s.advance(1e9, max_steps=5)
        assert np.abs(s.download() - V).max() <= 1e-10 * np.abs(V).max()
    with _solver(wb, p, wb.FP32_BULK) as s:
        s.set_frame(p.frame)
        s.upload(U0)
        s.advance(1e9, max_steps=5)
        assert np.abs(s.download() - V).sum() <= 1e-6 * np.abs(V).sum()


def test_neumann2_batch_with_other_kinds(wb, oracle_lib):
    # a NEUMANN2 instance next to a periodic one in one persistent launch
    (p1, U1), (p2, U2) = _runs(27, 5)[0], _runs(40, 33)[1]
    p3 = Problem(**{**p2.__dict__, "bc": BC_PERIOD, "frame": None})
    probs = [(p1, U1), (p2, U2), (p3, U2)]
    cfgs = [wb.make_config(p.nx, p.ny, bc=p.bc, scheme=p.scheme, flux=p.flux, recon=p.recon, limiter=p.limiter,
                           precision=wb.FP64_STRICT) for p, _ in probs]
    eqs = [wb.make_eq(rho10=p.rho10, rho20=p.rho20, sound1=p.sound1, sound2=p.sound2, gravity=p.gravity) for p, _ in probs]
    b = wb.Batch(cfgs, eqs)
    try:
        with pytest.raises(wb.WenofvError):  # no frame yet
            b.advance(1e9, max_steps=2)
        for k, (p, U) in enumerate(probs):
            if p.bc == BC_NEUMANN2:
                b.set_frame(k, p.frame)
            b.upload(k, U)
        b.advance(1e9, max_steps=2)
        with oracle_lib.cube_rounded():
            for k, (p, U) in enumerate(probs):
                V, *_ = oracle_lib.advance(p, U, t_end=1e9, max_steps=2)
                assert np.array_equal(b.download(k), V), k
    finally:
        b.close()


def test_neumann2_errors(wb):
    cfg = wb.make_config(16, 16, bc=wb.BC_NEUMANN2)
    with wb.Solver(cfg, wb.make_eq()) as s:
        U0, _ = cases.liquid_column(16, 16, seed=2)
        s.upload(U0)
        with pytest.raises(wb.WenofvError) as e:  # stepping before the frame is set
            s.advance(1e9, max_steps=1)
        assert e.value.code == wb.EINVAL
        with pytest.raises(ValueError):
            s.set_frame(np.zeros((4, 16, 16)))
    with wb.Solver(wb.make_config(16, 16), wb.make_eq()) as s:  # a frame on a periodic grid
        with pytest.raises(wb.WenofvError) as e:
            s.set_frame(np.ones((4, 24, 24)))
        assert e.value.code == wb.EINVAL
    # the serving API and the allocation-free step take no NEUMANN2 grid (they have no frame)
    eq = wb.make_eq()
    rc = wb.load().wenofv_step_noalloc(C.byref(cfg), C.byref(eq), None, None, 16, 0.0, None, None)
    assert rc == wb.ENOTSUP
