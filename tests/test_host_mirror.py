"""The C++ host mirror of the reference's driver (CConfig / TwoPhaseEquation / CWENOFV on
the CUDA backend, two-phase-3equation-2d-pal-column_b200/host).

CPU: it builds, reads settings.cfg with the reference's key = value rules, rejects the
cases the CUDA backend does not run, and its initial cell averages (initializeAve on the
reference's slab grid) equal the reference's own bit for bit.
GPU: `run()` of the mirror with PRECISION = FP64_STRICT reproduces the reference's final
state of SMOOTH and SHARP bit for bit.
"""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR
from oracle import Problem, reference_available, run_reference

HOST = os.path.join(PKG_DIR, "host")
BIN = os.path.join(HOST, "_build", "wenofv_host")
CFG = os.path.join(HOST, "config", "settings.cfg")
# TwoPhaseEquation parameters of the periodic test cases (rho10, rho20, sound1, sound2)
CASE_PARAMS = {0: (1.2, 1.0, 1.0, 1.0), 1: (1000.0, 1.0, 30.0, 30.0), 2: (1000.0, 1.0, 70.0, 70.0)}


@pytest.fixture(scope="module")
def host_bin():
    if not os.path.exists(os.path.join(PKG_DIR, "lib", "libwenofv_b200.so")):
        pytest.skip("libwenofv_b200.so not built")
    subprocess.run(["make", "-C", HOST], check=True, capture_output=True)
    return BIN


def run_host(host_bin, *kv, dump_ic=None, cwd=None, timeout=600):
    args = [host_bin, CFG] + list(kv)
    if dump_ic:
        args += ["--dump-ic", dump_ic]
    return subprocess.run(args, capture_output=True, text=True, timeout=timeout, cwd=cwd)


def to_soa(raw, nx, ny):
    return np.ascontiguousarray(raw.reshape(nx, ny, 4).transpose(2, 1, 0))


def test_host_builds_and_rejects_unsupported(host_bin, tmp_path):
    cp = run_host(host_bin, "TESTCASE=9", dump_ic=str(tmp_path / "x.bin"))
    assert cp.returncode == 1
    cp = run_host(host_bin, "BACKEND=CPU", dump_ic=str(tmp_path / "x.bin"))
    assert cp.returncode == 1 and "CUDA backend only" in cp.stderr
    cp = run_host(host_bin, "ELEMNUMX=30", dump_ic=str(tmp_path / "x.bin"))
    assert cp.returncode == 1 and "REFSLABS" in cp.stderr
    cp = subprocess.run([host_bin, str(tmp_path / "missing.cfg")], capture_output=True, text=True)
    assert cp.returncode == 1 and "Failed to open" in cp.stderr


def test_settings_reader_rules(host_bin, tmp_path):
    # comments, blank lines, CR line ends and blanks around '=' as the reference accepts them
    cfg = tmp_path / "s.cfg"
    cfg.write_bytes(b"# c\n\nTESTCASE =  2 \r\nELEMNUMX=16\nELEMNUMY = 8\r\n\rjunk\nnot a key\n")
    cp = subprocess.run([host_bin, str(cfg), "--dump-ic", str(tmp_path / "ic.bin")], capture_output=True, text=True)
    assert cp.returncode == 0, cp.stderr
    assert "Invalid line: not a key" in cp.stderr
    U = to_soa(np.fromfile(tmp_path / "ic.bin"), 16, 8)
    assert U[0].max() > 500 and np.isclose(U[0].min(), 1000 * 1e-8)  # SHARP: the square of phase 1 in phase 2


@pytest.mark.skipif(not reference_available(), reason="the compiled reference is not built here")
@pytest.mark.parametrize("testcase", [0, 1, 2])
def test_initial_averages_equal_reference(host_bin, tmp_path, testcase):
    nx, ny = 32, 24
    path = str(tmp_path / "ic.bin")
    cp = run_host(host_bin, f"TESTCASE={testcase}", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", dump_ic=path)
    assert cp.returncode == 0, cp.stderr
    mine = to_soa(np.fromfile(path), nx, ny)
    r10, r20, c1, c2 = CASE_PARAMS[testcase]
    p = Problem(nx=nx, ny=ny, rho10=r10, rho20=r20, sound1=c1, sound2=c2)
    ref = run_reference(p, testcase=testcase, steps=1)
    assert np.array_equal(mine, ref.U0)


@pytest.mark.gpu
@pytest.mark.skipif(not reference_available(), reason="the compiled reference binary is not present")
@pytest.mark.parametrize("testcase,kv", [(0, ("RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=0", "PPlimiter=0")),
                                         (2, ("RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")),
                                         (2, ("RECONSTRUCTIONTYPE=0", "RIEMANNFLUX=1", "PPlimiter=1", "STEPMODE=1")),
                                         (2, ("RECONSTRUCTIONTYPE=2", "RIEMANNFLUX=1", "PPlimiter=1")),
                                         (0, ("RECONSTRUCTIONTYPE=3", "RIEMANNFLUX=0", "PPlimiter=0")),
                                         (2, ("SCHEME=2", "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1"))])
def test_host_run_equals_reference(host_bin, tmp_path, testcase, kv):
    nx, ny, tend = 32, 32, 0.01
    out = str(tmp_path / "u.bin")
    cp = run_host(host_bin, f"TESTCASE={testcase}", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", "PRECISION=FP64_STRICT",
                  "REFSLABS=4", f"ENDTIME={tend}", f"OUTPUT={out}", *kv)
    assert cp.returncode == 0, cp.stderr
    mine = to_soa(np.fromfile(out), nx, ny)
    opts = dict(x.split("=") for x in kv if not x.startswith("STEPMODE"))
    r10, r20, c1, c2 = CASE_PARAMS[testcase]
    p = Problem(nx=nx, ny=ny, rho10=r10, rho20=r20, sound1=c1, sound2=c2, recon=int(opts["RECONSTRUCTIONTYPE"]),
                flux=int(opts["RIEMANNFLUX"]), limiter=int(opts["PPlimiter"]), scheme=int(opts.get("SCHEME", 1)),
                rk=2, cfl=0.5)
    ref = run_reference(p, testcase=testcase, t_end=tend)
    assert np.array_equal(mine, ref.U)


# Accuracy of z1 against the exact solution on SMOOTH at t = 0.05, as the reference's
# outputAccuracy computes it (src/WENOFV.cpp:3152-3251), for runs of the reference made with
# a one-rank build (so REFSLABS = 1): (L_inf, L1, L2) to 15 digits.
SMOOTH_KNOWN = [
    ((100, "SCHEME=1", "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=0"),
     (3.841719623982887e-07, 2.400853109961034e-07, 2.689826478231563e-07)),
    ((128, "SCHEME=0", "RECONSTRUCTIONTYPE=0", "RIEMANNFLUX=0"),
     (9.072026528854360e-07, 4.452180407799647e-07, 5.149646872224241e-07)),
    ((128, "SCHEME=1", "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1"),
     (7.220356113869786e-08, 4.566660819012802e-08, 5.089875840234343e-08)),
]


def smooth_accuracy(U, n, t):
    """(L_inf, L1, L2) of z1 = getVolumeFrac(U) against the 4x4 Gauss-Legendre average of the
    translated initial volume fraction (rho10 = 1.2, rho20 = 1, c1 = c2 = 1, eps = 1e-8)"""
    from cases import GLEG_W, GLEG_X

    eps, c1, c2, r10, r20 = 1e-8, 1.0, 1.0, 1.2, 1.0
    d = 1.0 / n
    xl = 0.0 - 3 * d + (np.arange(n) + 3) * d
    xr = 0.0 - 3 * d + (np.arange(n) + 4) * d
    xc = (xl + xr) / 2
    ex = np.zeros((n, n))  # [j][i]
    for a in range(4):
        for b in range(4):
            X = xc[None, :] + 0.5 * d * GLEG_X[a]
            Y = xc[:, None] + 0.5 * d * GLEG_X[b]
            z = eps + (1 - 2 * eps) * np.sin(2.0 * np.pi * (X - t)) ** 2 + 0 * Y
            ex += z * (0.5 * d * GLEG_W[a]) * (0.5 * d * GLEG_W[b]) / d / d
    a1, a2 = U[0], U[1]
    q = r20 * c2 * c2 - r10 * c1 * c1
    qs = a2 * c2 * c2 - a1 * c1 * c1
    r = ((q - qs) + np.sqrt((q - qs) ** 2 + 4.0 * a1 * c1 * c1 * a2 * c2 * c2)) / (2.0 * a2 * c2 * c2)
    err = np.abs(ex - r / (1 + r))
    return err.max(), err.mean(), np.sqrt((err ** 2).mean())


@pytest.mark.gpu
@pytest.mark.parametrize("case,known", SMOOTH_KNOWN)
def test_smooth_accuracy_known_answers(host_bin, tmp_path, case, known):
    n, *kv = case
    out = str(tmp_path / "u.bin")
    cp = run_host(host_bin, "TESTCASE=0", f"ELEMNUMX={n}", f"ELEMNUMY={n}", "RKMETH=2", "CFL=0.5", "PPlimiter=0",
                  "PRECISION=FP64_STRICT", "REFSLABS=1", f"OUTPUT={out}", *kv)
    assert cp.returncode == 0, cp.stderr
    U = to_soa(np.fromfile(out), n, n)
    got = smooth_accuracy(U, n, 0.05)
    assert np.allclose(got, known, rtol=1e-6, atol=0), (got, known)


@pytest.mark.gpu
def test_host_writes_the_reference_output_files(host_bin, tmp_path):
    # the shipped settings (SMOOTH 100^2, WENO-Z, characteristic, LLF) with the output of
    # outputResults: average_*.plt and accuracy_*.csv, as the reference writes them
    out = tmp_path / "out"
    cp = run_host(host_bin, "PRECISION=FP64_STRICT", "REFSLABS=1", f"OUTPUTDIR={out}")
    assert cp.returncode == 0, cp.stderr
    names = sorted(os.listdir(out))
    assert "average_initial.plt" in names and "average_final.plt" in names and "average_0.05_intermediate.plt" in names
    lines = (out / "average_final.plt").read_text().splitlines()
    assert lines[0] == "TITLE=FvSolution" and lines[1].split()[:4] == ["VARIABLES=X", "Y", "RHO1Z1", "RHO2Z2"]
    assert lines[2].startswith("ZONE T=TA, I=100, J=100")
    rows = [list(map(float, ln.split())) for ln in lines[3:]]
    assert len(rows) == 100 * 100 and all(len(r) == 13 for r in rows)  # ... PRE theta Pr
    acc = (out / "accuracy_final.csv").read_text().splitlines()
    assert acc[0] == "Cell Number, Linf-norm, L1-norm, L2-norm"
    vals = [float(x) for x in acc[1].split(",")]
    assert vals[0] == 100 and np.allclose(vals[1:], SMOOTH_KNOWN[0][1], rtol=1e-6, atol=0)


@pytest.mark.gpu
@pytest.mark.skipif(not reference_available(), reason="the compiled reference binary is not present")
@pytest.mark.parametrize("recon", [1, 0])
def test_host_output_files_equal_reference(host_bin, tmp_path, recon):
    """average_final.plt and slice_final.plt of the mirror against the files the compiled
    reference's own outputAve / outputSliceAve write on the same run (SHARP 32^2 to t = 0.01 with
    the limiter, which limits some cells there, so the theta column is exercised)"""
    nx, tend = 32, 0.01
    out = tmp_path / "mine"
    cp = run_host(host_bin, "TESTCASE=2", f"ELEMNUMX={nx}", f"ELEMNUMY={nx}", "PRECISION=FP64_STRICT", "REFSLABS=4",
                  f"ENDTIME={tend}", f"RECONSTRUCTIONTYPE={recon}", "RIEMANNFLUX=1", "PPlimiter=1", "SCHEME=1",
                  f"OUTPUTDIR={out}", "SLICEOUTPUT=1")
    assert cp.returncode == 0, cp.stderr
    ref = tmp_path / "ref"
    ref.mkdir()
    from oracle import REF_BIN
    rp = subprocess.run([REF_BIN, "--testcase", "2", "--nx", str(nx), "--ny", str(nx), "--rk", "2", "--cfl", "0.5",
                         "--scheme", "1", "--limiter", "1", "--flux", "1", "--recon", str(recon), "--tend", repr(tend),
                         "--output-ave", str(ref)], capture_output=True, text=True, timeout=600)
    assert rp.returncode == 0, rp.stderr[-2000:]
    for name in ("average_final.plt", "slice_final.plt"):
        a = (out / name).read_text().splitlines()
        b = (ref / name).read_text().splitlines()
        assert [x.rstrip() for x in a] == [x.rstrip() for x in b], name
    theta = [int(float(ln.split()[11])) for ln in (ref / "average_final.plt").read_text().splitlines()[3:]]
    assert 0 < sum(theta) < nx * nx  # some cells limited, not all


# the periodic cases' (u0, v0, epsa): include/Equations.hpp:490-689
CASE_FLOW = {0: (1.0, 1.0, 1e-8), 1: (2.0, 2.0, 1e-4), 2: (1.0, 1.0, 1e-8)}
CASE_BOX = {0: (0.0, 1.0, 0.0, 1.0), 1: (-1.0, 1.0, -1.0, 1.0), 2: (0.0, 1.0, 0.0, 1.0)}


@pytest.mark.gpu
@pytest.mark.parametrize("testcase", [0, 1, 2])
def test_device_initial_averages(wb, host_bin, tmp_path, testcase):
    # wenofv_init_testcase against the host mirror's averages (which equal the reference's)
    nx, ny = 32, 24
    path = str(tmp_path / "ic.bin")
    assert run_host(host_bin, f"TESTCASE={testcase}", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", dump_ic=path).returncode == 0
    host = to_soa(np.fromfile(path), nx, ny)
    r10, r20, c1, c2 = CASE_PARAMS[testcase]
    xl, xr, yl, yr = CASE_BOX[testcase]
    cfg = wb.make_config(nx, ny, xl=xl, xr=xr, yl=yl, yr=yr, ref_slabs=4)
    with wb.Solver(cfg, wb.make_eq(rho10=r10, rho20=r20, sound1=c1, sound2=c2)) as s:
        s.init_testcase(testcase, *CASE_FLOW[testcase])
        dev = s.download()
    assert np.abs(dev - host).max() <= 1e-14 * np.abs(host).max()


@pytest.mark.gpu
def test_device_accuracy_known_answer(wb):
    # SMOOTH 128^2, WENO-JS, conservative, LLF, RK3 to t = 0.05, initialised and measured on
    # the GPU: the reference's own accuracy report (one-rank run)
    n = 128
    cfg = wb.make_config(n, n, rk=2, cfl=0.5, scheme=0, flux=0, recon=0, limiter=0, ref_slabs=1,
                         precision=wb.FP64_STRICT)
    with wb.Solver(cfg, wb.make_eq(rho10=1.2, rho20=1.0, sound1=1.0, sound2=1.0)) as s:
        s.init_testcase(0, *CASE_FLOW[0])
        t, k = s.advance(0.05)
        norms = s.accuracy(0, *CASE_FLOW[0], t)
        U = s.download()
    assert k == 52
    assert np.allclose(norms, SMOOTH_KNOWN[1][1], rtol=1e-6, atol=0)
    # the errors are ~1e-7 differences of O(1) averages, so a 1-ulp change of the exact
    # solution's sin (device against numpy) moves them by ~1e-9 relative
    assert np.allclose(norms, smooth_accuracy(U, n, t), rtol=1e-8, atol=0)


# the wall cases: domain, (rho10, rho20, sound1, sound2) and gravity of setEquationParameters
WALL_CASES = {3: ((0.0, 1.61, 0.0, 0.805), (1000.0, 1.0, 100.0, 100.0), 9.81),
              6: ((0.0, 1.0, 0.0, 4.0), (1.225, 0.1694, 100.0, 100.0), 9.81),
              7: ((0.0, 0.5, 0.0, 0.5), (1000.0, 1.0, 100.0, 100.0), 2 * np.pi)}


@pytest.mark.gpu
@pytest.mark.parametrize("testcase", sorted(WALL_CASES))
def test_host_wall_cases_equal_oracle(host_bin, oracle_lib, tmp_path, testcase):
    # DAMBREAK, RTI and STANDING_WAVE, which the reference declares but cannot run: the host
    # mirror's initial data, NEUMANN walls and gravity through the library, against the
    # oracle advanced from the same initial averages
    nx, ny, tend = 32, 16, 2e-4
    ic, out = str(tmp_path / "ic.bin"), str(tmp_path / "u.bin")
    kv = (f"TESTCASE={testcase}", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", "PRECISION=FP64_STRICT", "REFSLABS=4",
          "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")
    assert run_host(host_bin, *kv, dump_ic=ic).returncode == 0
    cp = run_host(host_bin, *kv, f"ENDTIME={tend}", f"OUTPUT={out}")
    assert cp.returncode == 0, cp.stderr
    U0, mine = to_soa(np.fromfile(ic), nx, ny), to_soa(np.fromfile(out), nx, ny)
    (xl, xr, yl, yr), (r10, r20, c1, c2), g = WALL_CASES[testcase]
    p = Problem(nx=nx, ny=ny, xl=xl, xr=xr, yl=yl, yr=yr, bc=1, rho10=r10, rho20=r20, sound1=c1, sound2=c2,
                gravity=g, scheme=1, recon=1, flux=1, limiter=1, ref_slabs=4, rk=2, cfl=0.5)
    V, n, t, _ = oracle_lib.advance(p, U0, t_end=tend)
    assert n > 0 and abs(t - tend) <= 1e-10
    assert np.array_equal(mine, V)


def test_host_zalesak_frame(host_bin, tmp_path):
    # ZALESAK selects NEUMANN2: the host mirror writes the ghost frame of its initial data
    # (the disc far from the edges, solid-body rotation u = pi (0.5 - y), v = pi (x - 0.5))
    nx, ny = 16, 12
    ic = str(tmp_path / "ic.bin")
    assert run_host(host_bin, "TESTCASE=8", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", "REFSLABS=4", dump_ic=ic).returncode == 0
    F = np.fromfile(ic + ".frame").reshape(4, ny + 8, nx + 8)
    assert np.all(F[:, 4:-4, 4:-4] == 0.0)  # the interior is not part of the frame
    ghost = np.ones((ny + 8, nx + 8), bool)
    ghost[4:-4, 4:-4] = False
    rho = F[0] + F[1]
    assert np.allclose(F[0][ghost], 1000.0 * 1e-8) and np.allclose(F[1][ghost], 1.0 - 1e-8)
    yc = (np.arange(-4, ny + 4) + 0.5) / ny
    xc = (np.arange(-4, nx + 4) + 0.5) / nx
    assert np.allclose(F[2][ghost], (rho * np.pi * (0.5 - yc)[:, None])[ghost], rtol=1e-12, atol=1e-12)
    assert np.allclose(F[3][ghost], (rho * np.pi * (xc - 0.5)[None, :])[ghost], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_host_zalesak_equals_oracle(host_bin, oracle_lib, tmp_path):
    # the rotating disc through the library with its NEUMANN2 frame, against the oracle
    # advanced from the same initial averages and frame
    nx, ny, tend = 32, 32, 2e-3
    ic, out = str(tmp_path / "ic.bin"), str(tmp_path / "u.bin")
    kv = ("TESTCASE=8", f"ELEMNUMX={nx}", f"ELEMNUMY={ny}", "PRECISION=FP64_STRICT", "REFSLABS=4",
          "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")
    assert run_host(host_bin, *kv, dump_ic=ic).returncode == 0
    cp = run_host(host_bin, *kv, f"ENDTIME={tend}", f"OUTPUT={out}")
    assert cp.returncode == 0, cp.stderr
    U0, mine = to_soa(np.fromfile(ic), nx, ny), to_soa(np.fromfile(out), nx, ny)
    F = np.fromfile(ic + ".frame").reshape(4, ny + 8, nx + 8)
    p = Problem(nx=nx, ny=ny, bc=3, frame=F, rho10=1000.0, rho20=1.0, sound1=70.0, sound2=70.0, scheme=1, recon=1,
                flux=1, limiter=1, ref_slabs=4, rk=2, cfl=0.5)
    V, n, t, _ = oracle_lib.advance(p, U0, t_end=tend)
    assert n > 0 and abs(t - tend) <= 1e-10
    assert np.array_equal(mine, V)


@pytest.mark.gpu
def test_host_sharp_oscillation_output(host_bin, tmp_path):
    # SHARP writes outputUPoscillation's file at the initial and final moments: the velocity
    # and pressure deviations from the uniform flow (1, 1), consistent with average_*.plt
    out = tmp_path / "out"
    kv = ("TESTCASE=2", "ELEMNUMX=32", "ELEMNUMY=32", "REFSLABS=4", "ENDTIME=0.05", "PRECISION=FP64_STRICT",
          "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")
    cp = run_host(host_bin, *kv, f"OUTPUTDIR={out}")
    assert cp.returncode == 0, cp.stderr
    # the time series of outputUPoscillationByTime at step 1 and every 200th step, the same
    # from the device loop (run in pieces) and from the host loop
    steps = json.loads(cp.stdout.strip().splitlines()[-1])["steps"]
    assert steps >= 200
    out_h = tmp_path / "out_host"
    cp = run_host(host_bin, *kv, "STEPMODE=1", f"OUTPUTDIR={out_h}")
    assert cp.returncode == 0, cp.stderr
    ts = (out / "oscillationByTime_32.plt").read_text()
    assert ts == (out_h / "oscillationByTime_32.plt").read_text()
    ts = ts.splitlines()
    assert ts[0] == "TITLE=FvSolution" and ts[2] == "ZONE T=TA"
    assert ts[1].split() == ["VARIABLES=Time", "Speed_oscillation", "P_oscillation", "U_oscillation", "V_oscillation"]
    series = np.array([list(map(float, ln.split())) for ln in ts[3:]])
    assert series.shape == (1 + steps // 200, 5) and np.all(np.diff(series[:, 0]) > 0) and np.all(series[:, 1:3] >= 0)
    # outputThincknessByTime at the same steps: 1 / the largest z1 jump, about 1 cell for the
    # sharp square after one step, growing as the scheme smears it
    th = (out / "thincknessByTime.plt").read_text()
    assert th == (out_h / "thincknessByTime.plt").read_text()
    th = th.splitlines()
    assert th[:4] == ["TITLE=FvSolution", "VARIABLES=time thinckness", "", "ZONE T=TA"]
    thick = np.array([list(map(float, ln.split())) for ln in th[4:]])
    assert np.array_equal(thick[:, 0], series[:, 0]) and 1.0 <= thick[0, 1] < 2.0 and thick[-1, 1] >= thick[0, 1]
    for moment in ("initial", "final"):
        lines = (out / f"UPoscillation_{moment}.plt").read_text().splitlines()
        assert lines[0] == "TITLE=FvSolution"
        assert lines[1].split() == ["VARIABLES=X", "Y", "Speed_oscillation", "P_oscillation", "U_oscillation", "V_oscillation"]
        assert lines[2].startswith("ZONE T=TA, I=32, J=32")
        osc = np.array([list(map(float, ln.split())) for ln in lines[3:]])
        ave = np.array([list(map(float, ln.split())) for ln in (out / f"average_{moment}.plt").read_text().splitlines()[3:]])
        assert osc.shape == (32 * 32, 6)
        assert np.array_equal(osc[:, :2], ave[:, :2])
        u, v, p = ave[:, 8], ave[:, 9], ave[:, 10]
        # the printed columns carry 6 significant digits
        assert np.allclose(osc[:, 4], np.abs(u - 1) / 70.0, rtol=1e-4, atol=1e-9)
        assert np.allclose(osc[:, 5], np.abs(v - 1) / 70.0, rtol=1e-4, atol=1e-9)
        assert np.allclose(osc[:, 3], np.abs(p) / 1000.0 / 70.0 ** 2, rtol=1e-4, atol=1e-12)
        assert np.allclose(osc[:, 2], np.hypot(osc[:, 4], osc[:, 5]), rtol=1e-4, atol=1e-9)


@pytest.mark.gpu
def test_host_dambreak_pressure_probes(host_bin, tmp_path):
    # DAMBREAK's outputPressureByTime: wall pressures at 3, 15, 30 and 80 mm over rho10 g H0,
    # at step 1 and every 200th step; the same from the device loop and the host loop
    kv = ("TESTCASE=3", "ELEMNUMX=32", "ELEMNUMY=16", "REFSLABS=4", "ENDTIME=0.06", "PRECISION=FP64_STRICT",
          "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")
    out, out_h = tmp_path / "out", tmp_path / "out_host"
    cp = run_host(host_bin, *kv, f"OUTPUTDIR={out}")
    assert cp.returncode == 0, cp.stderr
    steps = json.loads(cp.stdout.strip().splitlines()[-1])["steps"]
    assert steps >= 200
    cp = run_host(host_bin, *kv, "STEPMODE=1", f"OUTPUTDIR={out_h}")
    assert cp.returncode == 0, cp.stderr
    text = (out / "pressureByTime.plt").read_text()
    assert text == (out_h / "pressureByTime.plt").read_text()
    lines = text.splitlines()
    assert lines[:4] == ["TITLE=FvSolution", "VARIABLES=Time P_y3mm P_y15mm P_y30mm P_y80mm", "", "ZONE T=TA"]
    series = np.array([list(map(float, ln.split())) for ln in lines[4:]])
    assert series.shape == (1 + steps // 200, 5) and np.all(np.diff(series[:, 0]) > 0)
    # getPressure of the linearised model is the deviation from g_preb, which starts at 0:
    # after one step it is still far below the hydrostatic scale (1 on this axis)
    assert np.all(np.abs(series[0, 1:]) < 1e-3)


@pytest.mark.gpu
def test_host_rti_symmetry_error(host_bin, tmp_path):
    # RTI's outputSymmetryErr: z1 of the left half against its mirror image, at step 1 and
    # every 200th step.  The initial interface is mirror-symmetric; the 4-slab grid metric is
    # not to the last bit, and the Rayleigh-Taylor instability amplifies that rounding-level
    # asymmetry (about 1e-12 after one step, 2e-8 after 200 on this grid)
    kv = ("TESTCASE=6", "ELEMNUMX=16", "ELEMNUMY=32", "REFSLABS=4", "ENDTIME=0.07", "PRECISION=FP64_STRICT",
          "RECONSTRUCTIONTYPE=1", "RIEMANNFLUX=1", "PPlimiter=1")
    out = tmp_path / "out"
    cp = run_host(host_bin, *kv, f"OUTPUTDIR={out}")
    assert cp.returncode == 0, cp.stderr
    steps = json.loads(cp.stdout.strip().splitlines()[-1])["steps"]
    assert steps >= 200
    err = np.array([list(map(float, ln.split())) for ln in (out / "symmetry_err.plt").read_text().splitlines()])
    assert err.shape == (1 + steps // 200, 2) and np.all(np.diff(err[:, 0]) > 0)
    assert np.all(err[:, 1] >= 0) and err[0, 1] < 1e-10 and np.all(err[:, 1] < 1e-6)
