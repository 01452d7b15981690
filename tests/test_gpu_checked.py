"""The self-checking build (lib/libwenofv_b200_checked.so) on small and ragged grids.

compute-sanitizer is not available, so the library is also built with every global index of
the stage kernel checked against its buffer before the access: a violation sets
WENOFV_FLAG_BOUNDS (and the call returns WENOFV_ENUMERIC) instead of touching the memory.
A child process loads that build and runs tiny and ragged grids through every
reconstruction, the boundary kinds (NEUMANN2's frame included), the three arithmetic forms and a batch. No flag may be
raised, and FP64_STRICT must still equal the oracle bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CHECKED = os.path.join(ROOT, "two-phase-3equation-2d-pal-column_b200", "lib", "libwenofv_b200_checked.so")


def child():
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from conftest import import_package
    from oracle import BC_NEUMANN2, BC_OUTFLOW, EQ_EULER, Oracle, Problem
    import cases

    wb = import_package()
    assert wb.LIB_PATH == CHECKED
    o = Oracle()
    n_cases = 0
    o.L.ofv_set_cube_rounded(1)  # WENOEXP's l^3 as the device kernels form it
    for nx, ny, scheme in [(1, 1, 1), (3, 2, 1), (8, 8, 1), (12, 8, 1), (27, 5, 1), (26, 33, 1), (130, 9, 1),
                           (1, 1, 2), (3, 2, 2), (24, 8, 2), (25, 7, 2), (50, 33, 2)]:
        for recon in (0, 1, 2, 3, 4):
            mild = dict(ratio=2.0, eps=0.05)
            U0, prm = cases.liquid_column(nx, ny, seed=nx + 7 * ny, **mild)
            p = Problem(nx=nx, ny=ny, scheme=scheme, flux=1, recon=recon, limiter=1, **prm)
            V, *_ = o.advance(p, U0, t_end=1e9, max_steps=2)
            for prec in (wb.FP64_STRICT, wb.FP64, wb.FP32_BULK):
                if (scheme == 2 or recon == 4) and prec == wb.FP32_BULK:
                    continue
                cfg = wb.make_config(nx, ny, scheme=scheme, flux=1, recon=recon, limiter=1, precision=prec)
                eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
                with wb.Solver(cfg, eq) as s:
                    s.upload(U0)
                    s.advance(1e9, max_steps=2)
                    flags, cell = s.status()
                    assert flags == 0, (nx, ny, scheme, recon, prec, flags, cell)
                    U = s.download()
                if prec == wb.FP64_STRICT and recon == 4:  # THINC: CUDA's exp/log/tanh
                    o.L.ofv_set_thinc_ulp(1)
                    W, *_ = o.advance(p, U0, t_end=1e9, max_steps=2)
                    o.L.ofv_set_thinc_ulp(0)
                    tol = 16 * np.abs(W - V).max() + 1e-14 * np.abs(V).max()
                    assert np.abs(U - V).max() <= tol, (nx, ny, scheme, recon)
                elif prec == wb.FP64_STRICT:
                    assert np.array_equal(U, V), (nx, ny, scheme, recon)
                n_cases += 1
    for nx, ny, bc in [(1, 1, 1), (3, 2, 2), (26, 9, 4), (25, 33, 1)]:  # walls, two-phase with gravity
        U0, prm = cases.liquid_column(nx, ny, seed=nx + ny, ratio=2.0, eps=0.05)
        for scheme in (1, 2):
            p = Problem(nx=nx, ny=ny, bc=bc, scheme=scheme, flux=1, recon=1, limiter=1, gravity=9.81, **prm)
            V, *_ = o.advance(p, U0, t_end=1e9, max_steps=2)
            cfg = wb.make_config(nx, ny, bc=bc, scheme=scheme, flux=1, recon=1, limiter=1, precision=wb.FP64_STRICT)
            eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"], gravity=9.81)
            with wb.Solver(cfg, eq) as s:
                s.upload(U0)
                s.advance(1e9, max_steps=2)
                assert s.status()[0] == 0, (nx, ny, bc, scheme)
                assert np.array_equal(s.download(), V), (nx, ny, bc, scheme)
            n_cases += 1
    for nx, ny, scheme in [(1, 1, 1), (3, 2, 2), (26, 9, 1), (25, 33, 2)]:  # NEUMANN2 ghost frame
        U0, prm = cases.liquid_column(nx, ny, seed=nx + ny, ratio=2.0, eps=0.05)
        F0, _ = cases.liquid_column(nx, ny, seed=nx + ny + 1, ratio=2.0, eps=0.05)
        p = Problem(nx=nx, ny=ny, bc=BC_NEUMANN2, frame=cases.periodic_frame(F0), scheme=scheme, flux=1, recon=1,
                    limiter=1, **prm)
        V, *_ = o.advance(p, U0, t_end=1e9, max_steps=2)
        cfg = wb.make_config(nx, ny, bc=BC_NEUMANN2, scheme=scheme, flux=1, recon=1, limiter=1, precision=wb.FP64_STRICT)
        eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
        with wb.Solver(cfg, eq) as s:
            s.set_frame(p.frame)
            s.upload(U0)
            s.advance(1e9, max_steps=2)
            assert s.status()[0] == 0, (nx, ny, scheme)
            assert np.array_equal(s.download(), V), (nx, ny, scheme)
        n_cases += 1
    for nx, ny, scheme in [(5, 3, 1), (40, 9, 1), (5, 3, 2), (40, 9, 2)]:  # Euler, outflow
        U0, _ = cases.euler_quadrants(nx, ny, seed=3)
        cfg = wb.make_config(nx, ny, bc=wb.BC_OUTFLOW, cfl=0.4, scheme=scheme, flux=1, recon=1, precision=wb.FP64_STRICT)
        with wb.Solver(cfg, wb.make_eq(kind=wb.EQ_EULER)) as s:
            s.upload(U0)
            s.advance(1e9, max_steps=2)
            assert s.status()[0] == 0
            p = Problem(nx=nx, ny=ny, bc=BC_OUTFLOW, eq_kind=EQ_EULER, scheme=scheme, flux=1, recon=1, cfl=0.4)
            assert np.array_equal(s.download(), o.advance(p, U0, t_end=1e9, max_steps=2)[0])
        n_cases += 1
    ens = cases.ensemble(5, seed=9, grids=[(1, 1), (26, 26), (27, 5), (64, 40)])
    cfgs = [wb.make_config(q["nx"], q["ny"], scheme=q["scheme"], flux=1, recon=1, limiter=1, precision=wb.FP64)
            for _, q in ens]
    eqs = [wb.make_eq(rho10=q["rho10"], rho20=q["rho20"], sound1=q["sound1"], sound2=q["sound2"]) for _, q in ens]
    b = wb.Batch(cfgs, eqs)
    for k, (U0, _) in enumerate(ens):
        b.upload(k, U0)
    for rows in (8, 64):
        b.set_tiling(rows)
        b.advance(1e9, max_steps=2)
    b.close()
    print("checked cases:", n_cases + 1)


@pytest.mark.gpu
def test_checked_build_raises_no_bounds_flag():
    if not os.path.exists(CHECKED):
        pytest.skip("the self-checking build is missing (make -C two-phase-3equation-2d-pal-column_b200)")
    env = dict(os.environ, WENOFV_LIB=CHECKED)
    cp = subprocess.run([sys.executable, os.path.abspath(__file__), "--child"], capture_output=True, text=True,
                        env=env, timeout=900)
    assert cp.returncode == 0, cp.stdout[-2000:] + cp.stderr[-4000:]
    assert "checked cases:" in cp.stdout


if __name__ == "__main__" and "--child" in sys.argv:
    child()
