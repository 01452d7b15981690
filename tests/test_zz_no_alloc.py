"""The no-allocation RK step (wenofv_step_noalloc) against the regular one (wenofv_step).

Some callers cannot call cudaMalloc: they manage device memory through their own pool or a
framework allocator, reserve all free memory at start-up, or cannot afford the device
synchronisation that cudaMalloc/cudaFree imply inside a latency-bound loop.  For them the
library offers one RK step that works on the caller's own device input and output arrays
and keeps its scratch in a fixed device array inside the library.  This test (run last, in
a file of its own) feeds both entry points the same states through the C ABI, twice in a
row, and requires the same results: bit for bit in FP64_STRICT, and to the FP64 tolerance
of the other parity tests (1e-11 of max |U|) in FP64 and FP32-bulk, for every RK method.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import cases

pytestmark = pytest.mark.gpu


def _noalloc_step(wb, cfg, eq, d_in, d_out, pitch, dt, stream=None):
    import torch

    flags = C.c_uint32(0)
    rc = wb.load().wenofv_step_noalloc(C.byref(cfg), C.byref(eq), C.c_void_p(d_in.data_ptr()),
                                       C.c_void_p(d_out.data_ptr()), pitch, dt,
                                       C.c_void_p(stream if stream else 0), C.byref(flags))
    if rc != wb.OK:
        raise wb.WenofvError(rc, "wenofv_step_noalloc")
    torch.cuda.synchronize()
    return flags.value


# every RK method (their buffer roles differ: RK1 writes the output directly, RK2 and RK3 go
# through the scratch state), each form, and a call on a side stream
@pytest.mark.parametrize("precision,recon,lim,rk,side", [
    ("FP64_STRICT", 1, 1, 2, False), ("FP64_STRICT", 0, 0, 2, False), ("FP64", 1, 1, 2, False),
    ("FP64_STRICT", 1, 1, 0, False), ("FP64_STRICT", 1, 1, 1, False), ("FP64", 0, 1, 1, True),
    ("FP32_BULK", 1, 1, 2, False), ("FP32_BULK", 0, 1, 0, True)])
def test_noalloc_step_matches_step(wb, precision, recon, lim, rk, side):
    import torch

    prec = getattr(wb, precision)
    nx, ny, pitch = 83, 61, 90  # ragged strips, pitch wider than the row
    U0, prm = cases.liquid_column(nx, ny, seed=17)
    cfg = wb.make_config(nx, ny, rk=rk, scheme=1, flux=1, recon=recon, limiter=lim, ref_slabs=0, precision=prec)
    eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])

    # the existing entry point: two steps with the CFL step of the initial state
    with wb.Solver(cfg, eq) as s:
        s.upload(U0)
        dt = s.compute_dt()
        s.step(dt)
        ref1 = s.download()
        s.step(dt)
        ref2 = s.download()

    dev = torch.device("cuda:0")
    a = torch.zeros((4, ny, pitch), dtype=torch.float64, device=dev)
    b = torch.zeros_like(a)
    a[:, :, :nx] = torch.from_numpy(U0).to(dev)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(device=dev) if side else None
    sp = stream.cuda_stream if side else None
    assert _noalloc_step(wb, cfg, eq, a, b, pitch, dt, sp) == 0
    got1 = b[:, :, :nx].cpu().numpy()
    assert _noalloc_step(wb, cfg, eq, b, a, pitch, dt, sp) == 0  # second call in a row, buffers swapped
    got2 = a[:, :, :nx].cpu().numpy()
    if prec == wb.FP64_STRICT:
        assert np.array_equal(got1, ref1) and np.array_equal(got2, ref2)
    else:
        # the same kernels run in both entry points: FP64 and FP32-bulk agree to the FP64
        # parity tolerance of the other tests (1e-11 of max |U|)
        scale = np.abs(ref2).max()
        assert np.abs(got1 - ref1).max() <= 1e-11 * scale and np.abs(got2 - ref2).max() <= 1e-11 * scale


def test_noalloc_step_reports_nan_state_and_keeps_device(wb):
    """a NaN cell raises the NaN-state bit in *flags; the next clean call starts from a clear
    status word (the shared array keeps the last call's contents, so the call resets it)"""
    import torch

    nx, ny = 40, 32
    U0, prm = cases.liquid_column(nx, ny, seed=5)
    cfg = wb.make_config(nx, ny, scheme=1, flux=1, recon=1, limiter=0, precision=wb.FP64)
    eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
    dev = torch.device("cuda:0")
    bad = U0.copy()
    bad[2, 10, 7] = np.nan
    a = torch.from_numpy(bad).to(dev).contiguous()
    b = torch.zeros_like(a)
    torch.cuda.synchronize()
    before = torch.cuda.current_device()
    f = _noalloc_step(wb, cfg, eq, a, b, nx, 1e-4)
    assert f & wb.FLAG_NAN_STATE
    assert torch.cuda.current_device() == before
    a = torch.from_numpy(U0).to(dev).contiguous()
    torch.cuda.synchronize()
    assert _noalloc_step(wb, cfg, eq, a, b, nx, 1e-4) == 0


def test_noalloc_step_rejects_oversized_grids(wb):
    import torch

    cfg = wb.make_config(1024, 1024, precision=wb.FP64)
    eq = wb.make_eq()
    x = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    y = torch.zeros(8, dtype=torch.float64, device="cuda:0")
    flags = C.c_uint32(0)
    L = wb.load()
    rc = L.wenofv_step_noalloc(C.byref(cfg), C.byref(eq), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                               1024, 1e-4, None, C.byref(flags))
    assert rc == wb.EINVAL
    assert b"at most" in L.wenofv_last_error()
    # aliasing input and output is rejected too
    cfg2 = wb.make_config(16, 16)
    rc = L.wenofv_step_noalloc(C.byref(cfg2), C.byref(eq), C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()),
                               16, 1e-4, None, None)
    assert rc == wb.EINVAL
    # an infinite or NaN dt is rejected before any GPU work
    for bad_dt in (float("inf"), float("nan"), -1e-4):
        rc = L.wenofv_step_noalloc(C.byref(cfg2), C.byref(eq), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                   16, bad_dt, None, None)
        assert rc == wb.EINVAL
