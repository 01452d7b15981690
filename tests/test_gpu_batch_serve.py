"""Batched ensembles and the serving loop (no counterpart in the reference).

* Every instance of a batch equals the same instance solved alone (bit for bit in
  FP64_STRICT, where neighbouring instances cannot change an instance's arithmetic).
* Every served request equals the same solve run alone through the single-grid API, however
  it was mixed with other requests (bit for bit in FP64_STRICT).
"""
from __future__ import annotations

import time

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def column_cfg(wb, nx, ny, prm, precision, scheme=1, limiter=1):
    cfg = wb.make_config(nx, ny, scheme=scheme, flux=1, recon=1, limiter=limiter, precision=precision)
    eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
    return cfg, eq


def alone(wb, cfg, eq, U0, t_end=1e9, max_steps=0):
    with wb.Solver(cfg, eq) as s:
        s.upload(U0)
        t, n = s.advance(t_end, max_steps=max_steps)
        return s.download(), n


@pytest.mark.parametrize("precision", ["FP64_STRICT", "FP64"])
def test_batch_equals_alone(wb, precision):
    prec = getattr(wb, precision)
    ens = cases.ensemble(6, seed=5, grids=[(64, 64), (96, 40), (130, 33), (52, 70)])
    cfgs, eqs = [], []
    for U0, prm in ens:
        c, e = column_cfg(wb, prm["nx"], prm["ny"], prm, prec, scheme=prm["scheme"])
        cfgs.append(c)
        eqs.append(e)
    b = wb.Batch(cfgs, eqs)
    for k, (U0, _) in enumerate(ens):
        b.upload(k, U0)
    t_end = [0.002 * (k + 1) for k in range(len(ens))]  # uneven end times
    ns = b.advance(t_end)
    for k, (U0, _) in enumerate(ens):
        ref, n = alone(wb, cfgs[k], eqs[k], U0, t_end=t_end[k])
        assert ns[k] == n
        got = b.download(k)
        if prec == wb.FP64_STRICT:
            assert np.array_equal(got, ref)
        else:
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    b.close()


def test_batch_mixed_equations_and_tiling(wb):
    # a two-phase instance, an Euler instance (outflow) and an advection instance in one batch
    U1, prm = cases.liquid_column(64, 48, seed=7)
    c1, e1 = column_cfg(wb, 64, 48, prm, wb.FP64_STRICT)
    U2, _ = cases.euler_quadrants(40, 40)
    c2 = wb.make_config(40, 40, bc=wb.BC_OUTFLOW, cfl=0.4, scheme=1, flux=1, recon=0, precision=wb.FP64_STRICT)
    e2 = wb.make_eq(kind=wb.EQ_EULER)
    U3 = cases.advection_sine(150, 20)
    c3 = wb.make_config(150, 20, scheme=0, flux=0, recon=0, precision=wb.FP64_STRICT)
    e3 = wb.make_eq(kind=wb.EQ_LINEAR_ADV)
    # and a WENOEXP column (7-point stencils: its own strip width and launch group)
    c4, e4 = column_cfg(wb, 64, 48, prm, wb.FP64_STRICT, scheme=2)
    refs = [alone(wb, c, e, U, max_steps=5)[0] for c, e, U in ((c1, e1, U1), (c2, e2, U2), (c3, e3, U3), (c4, e4, U1))]
    for rows, ctas in ((8, 1), (16, 0), (64, 2)):
        b = wb.Batch([c1, c2, c3, c4], [e1, e2, e3, e4])
        for k, U in enumerate((U1, U2, U3, U1)):
            b.upload(k, U)
        b.set_tiling(rows, ctas)
        ns = b.advance([1e9] * 4, max_steps=5)
        assert list(ns) == [5, 5, 5, 5]
        for k in range(4):
            assert np.array_equal(b.download(k), refs[k])
        b.close()


def test_batch_autotune_keeps_state(wb):
    ens = cases.ensemble(4, seed=9, grids=[(64, 64), (96, 48)])
    cfgs, eqs = [], []
    for U0, prm in ens:
        c, e = column_cfg(wb, prm["nx"], prm["ny"], prm, wb.FP64_STRICT, scheme=prm["scheme"])
        cfgs.append(c)
        eqs.append(e)
    b = wb.Batch(cfgs, eqs)
    for k, (U0, _) in enumerate(ens):
        b.upload(k, U0)
    rows, ctas, ms = b.autotune()
    assert rows in (0, 16, 32, 64) and ms > 0  # 0: the automatic rows per item
    for k, (U0, _) in enumerate(ens):
        assert np.array_equal(b.download(k), U0)  # the autotuner restores the state
    b.advance([1e9] * len(ens), max_steps=3)
    for k, (U0, _) in enumerate(ens):
        ref, _ = alone(wb, cfgs[k], eqs[k], U0, max_steps=3)
        assert np.array_equal(b.download(k), ref)
    b.close()


def test_batch_cta_width_keeps_results(wb):
    # the same instances with the stage kernels of 128 and of 256 threads (strips of 26 and 58
    # columns), and with the per-instance choice: FP64_STRICT results equal the instances
    # solved alone bit for bit, whatever the width and the tiling
    ens = cases.ensemble(4, seed=9, grids=[(64, 64), (256, 64), (96, 96), (200, 40)])
    cfgs, eqs = [], []
    for U0, prm in ens:
        c, e = column_cfg(wb, prm["nx"], prm["ny"], prm, wb.FP64_STRICT, scheme=prm["scheme"])
        cfgs.append(c)
        eqs.append(e)
    refs = [alone(wb, c, e, U0, max_steps=4)[0] for c, e, (U0, _) in zip(cfgs, eqs, ens)]
    b = wb.Batch(cfgs, eqs)
    for nt, rows in ((128, 16), (256, 64), (0, 0), (256, 8)):
        b.set_threads(nt)
        b.set_tiling(rows, 0)
        assert b.tiling() == (rows, 0, nt)
        for k, (U0, _) in enumerate(ens):
            b.upload(k, U0)
        b.advance(1e9, max_steps=4)
        for k in range(len(ens)):
            assert np.array_equal(b.download(k), refs[k]), (nt, rows, k)
    with pytest.raises(wb.WenofvError) as e:
        b.set_threads(192)
    assert e.value.code == wb.EINVAL
    b.close()


def _drain(srv, ids, timeout=300.0):
    out = {}
    t0 = time.time()
    while len(out) < len(ids):
        for rid in ids:
            if rid in out:
                continue
            got = srv.poll(rid)
            if got is not None:
                out[rid] = got
        if time.time() - t0 > timeout:
            raise TimeoutError("server did not finish")
        time.sleep(0.002)
    return out


def test_server_alone_equals_mixed(wb):
    rng = np.random.default_rng(11)
    reqs = []
    for k in range(10):
        nx, ny = [(64, 64), (96, 48), (128, 64), (40, 40)][k % 4]
        if k % 3 == 2:
            U0, _ = cases.euler_quadrants(nx, ny, seed=k)
            cfg = wb.make_config(nx, ny, bc=wb.BC_OUTFLOW, cfl=0.4, scheme=1, flux=1, recon=0, precision=wb.FP64_STRICT)
            eq = wb.make_eq(kind=wb.EQ_EULER)
        else:
            U0, prm = cases.liquid_column(nx, ny, seed=k)
            cfg, eq = column_cfg(wb, nx, ny, prm, wb.FP64_STRICT)
        reqs.append((cfg, eq, U0, int(rng.integers(6, 30))))
    srv = wb.Server(0, hbm_budget_bytes=3 << 20, max_slots=4)  # small budget: requests queue
    ids = []
    for cfg, eq, U0, ns in reqs:
        ids.append(srv.submit(cfg, eq, U0, 1e9, max_steps=ns))
        time.sleep(0.001 * rng.integers(0, 3))  # arrivals while others run
    res = _drain(srv, ids)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["active"] == 0 and st["resident_bytes"] == 0
    for rid, (cfg, eq, U0, ns) in zip(ids, reqs):
        U, info = res[rid]
        assert info.status == 0 and info.steps == ns
        assert info.t_submit <= info.t_admit <= info.t_done
        ref, n = alone(wb, cfg, eq, U0, max_steps=ns)
        assert np.array_equal(U, ref)
    srv.close()


# FP32-bulk requests served beside FP64 ones (four launch groups, each its own branch of the
# captured graph): each served result equals the same solve alone through the single-grid API
# to SERVE_FP32_RTOL of max |U| (the per-instance arithmetic does not depend on the mix, so in
# practice the results are the same bits)
SERVE_FP32_RTOL = 1e-12


def test_server_alone_equals_mixed_fp32(wb):
    rng = np.random.default_rng(12)
    reqs = []
    for k in range(12):
        nx, ny = [(64, 64), (96, 48), (128, 64), (40, 40)][k % 4]
        prec = wb.FP64 if k % 4 == 3 else wb.FP32_BULK
        if k % 3 == 2:
            U0, _ = cases.euler_quadrants(nx, ny, seed=k)
            cfg = wb.make_config(nx, ny, bc=wb.BC_OUTFLOW, cfl=0.4, scheme=1, flux=1, recon=0, precision=prec)
            eq = wb.make_eq(kind=wb.EQ_EULER)
        else:
            U0, prm = cases.liquid_column(nx, ny, seed=k)
            cfg, eq = column_cfg(wb, nx, ny, prm, prec)
        reqs.append((cfg, eq, U0, int(rng.integers(6, 40))))
    srv = wb.Server(0, hbm_budget_bytes=4 << 20, max_slots=5)
    ids = []
    for cfg, eq, U0, ns in reqs:
        ids.append(srv.submit(cfg, eq, U0, 1e9, max_steps=ns))
        time.sleep(0.001 * rng.integers(0, 3))
    res = _drain(srv, ids)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["active"] == 0 and st["resident_bytes"] == 0
    for rid, (cfg, eq, U0, ns) in zip(ids, reqs):
        U, info = res[rid]
        assert info.status == 0 and info.steps == ns
        ref, n = alone(wb, cfg, eq, U0, max_steps=ns)
        assert np.abs(U - ref).max() <= SERVE_FP32_RTOL * np.abs(ref).max()
    srv.close()


def test_server_admits_after_retirement_without_regrowth(wb):
    # a stream of requests larger in total than the arena: slots and arena blocks are reused
    U0, prm = cases.liquid_column(64, 64, seed=4)
    cfg, eq = column_cfg(wb, 64, 64, prm, wb.FP64)
    per = 3 * 4 * 64 * 64 * 8 + (2 * 64 + 64) * 8
    srv = wb.Server(0, hbm_budget_bytes=3 * per + 4096, max_slots=8)
    ids = [srv.submit(cfg, eq, U0, 1e9, max_steps=4 + (k % 3)) for k in range(9)]
    res = _drain(srv, ids)
    ref = {n: alone(wb, cfg, eq, U0, max_steps=n)[0] for n in (4, 5, 6)}
    for k, rid in enumerate(ids):
        U, info = res[rid]
        assert info.status == 0 and info.steps == 4 + (k % 3)
        assert np.array_equal(U, ref[4 + (k % 3)])
    assert srv.stats()["resident_bytes"] == 0
    srv.close()


def test_server_rejects_and_isolates_failures(wb):
    srv = wb.Server(0, hbm_budget_bytes=1 << 20, max_slots=2)
    U0, prm = cases.liquid_column(256, 256, seed=1)
    cfg, eq = column_cfg(wb, 256, 256, prm, wb.FP64)
    with pytest.raises(wb.WenofvError) as e:
        srv.submit(cfg, eq, U0, 0.01)  # over the budget
    assert e.value.code == wb.ENOMEM
    U1, prm = cases.liquid_column(16, 16, seed=2)
    c0, e0 = column_cfg(wb, 16, 16, prm, wb.FP64)
    c0.bc = wb.BC_NEUMANN2
    with pytest.raises(wb.WenofvError) as e:
        srv.submit(c0, e0, U1, 0.01)  # a request carries no ghost frame
    assert e.value.code == wb.ENOTSUP
    c1, e1 = column_cfg(wb, 16, 16, prm, wb.FP64)
    U1[1, 3, 3] = np.nan  # a failing request does not disturb the others
    bad = srv.submit(c1, e1, U1, 1e9, max_steps=3)
    U2, prm2 = cases.liquid_column(16, 16, seed=3)
    c2, e2 = column_cfg(wb, 16, 16, prm2, wb.FP64)
    good = srv.submit(c2, e2, U2, 1e9, max_steps=3)
    t0 = time.time()
    failed = False
    while time.time() - t0 < 60:
        try:
            if srv.poll(bad) is not None:
                break
        except wb.WenofvError as err:
            assert err.code == wb.ENUMERIC
            failed = True
            break
        time.sleep(0.002)
    assert failed
    res = _drain(srv, [good])
    U, info = res[good]
    ref, _ = alone(wb, c2, e2, U2, max_steps=3)
    assert np.abs(U - ref).max() <= 1e-12 * np.abs(ref).max()
    srv.close()


def test_batch_member_with_nan_is_isolated(wb):
    # a corrupted instance stops with a NaN flag; the others finish as if alone
    ens = cases.ensemble(3, seed=8, grids=[(64, 64), (48, 40)])
    cfgs, eqs = [], []
    for U0, prm in ens:
        c, e = column_cfg(wb, prm["nx"], prm["ny"], prm, wb.FP64_STRICT, scheme=prm["scheme"])
        cfgs.append(c)
        eqs.append(e)
    b = wb.Batch(cfgs, eqs)
    bad = ens[1][0].copy()
    bad[2, 5, 7] = np.nan
    for k, (U0, _) in enumerate(ens):
        b.upload(k, bad if k == 1 else U0)
    with pytest.raises(wb.WenofvError) as e:
        b.advance(1e9, max_steps=5)
    assert e.value.code == wb.ENUMERIC
    for k in (0, 2):
        ref, n = alone(wb, cfgs[k], eqs[k], ens[k][0], max_steps=5)
        assert np.array_equal(b.download(k), ref)
    b.close()


def test_device_allocation_failure_is_reported(wb):
    # 46000^2 cells x 4 variables x 3 buffers x 8 B = 203 GB: more than the GPU holds
    cfg = wb.make_config(46000, 46000, precision=wb.FP64)
    eq = wb.make_eq()
    with pytest.raises(wb.WenofvError) as e:
        wb.Solver(cfg, eq)
    assert e.value.code == wb.ENOMEM
    # the device stays usable afterwards
    U0, prm = cases.liquid_column(32, 32, seed=1)
    c, q = column_cfg(wb, 32, 32, prm, wb.FP64_STRICT)
    ref, n = alone(wb, c, q, U0, max_steps=2)
    assert n == 2 and np.isfinite(ref).all()
