"""ctypes binding of the CPU oracle and a runner for the compiled reference.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py, and only as the checker.  The product library never loads it.

* ``Problem`` / ``Oracle`` wrap ``_build/liboracle.so`` (the C restatement,
  wenofv_oracle.c) with numpy arrays in SoA layout ``U[v, j, i]``.
* ``run_reference`` runs ``_ref/wenofv_ref``, the unmodified reference solver built by
  the Makefile in this directory (4 ranks as threads over an in-process MPI shim).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import json
import os
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "wenofv_ref")

EQ_TWO_PHASE, EQ_LINEAR_ADV, EQ_EULER, EQ_TWO_PHASE_SG = 0, 1, 2, 3
BC_PERIOD, BC_NEUMANN, BC_NOSLIP, BC_NEUMANN2, BC_FREESLIP, BC_OUTFLOW = 0, 1, 2, 3, 4, 5


class _Eq(C.Structure):
    _fields_ = [("kind", C.c_int), ("rho10", C.c_double), ("rho20", C.c_double),
                ("sound1", C.c_double), ("sound2", C.c_double), ("preb", C.c_double),
                ("gamma", C.c_double), ("adv_u", C.c_double), ("adv_v", C.c_double),
                ("gamma1", C.c_double), ("pinf1", C.c_double), ("gamma2", C.c_double), ("pinf2", C.c_double),
                ("gravity", C.c_double)]


class _Problem(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("xl", C.c_double), ("xr", C.c_double),
                ("yl", C.c_double), ("yr", C.c_double), ("bc", C.c_int), ("rk", C.c_int),
                ("cfl", C.c_double), ("scheme", C.c_int), ("limiter", C.c_int), ("flux", C.c_int),
                ("recon", C.c_int), ("ref_slabs", C.c_int), ("threads", C.c_int), ("eq", _Eq),
                ("frame", C.c_void_p)]


@dataclass
class Problem:
    """One solve's options, named like the reference's settings.cfg keys where they exist."""
    nx: int
    ny: int
    xl: float = 0.0
    xr: float = 1.0
    yl: float = 0.0
    yr: float = 1.0
    bc: int = BC_PERIOD
    rk: int = 2              # RKMETH
    cfl: float = 0.5         # CFL
    scheme: int = 1          # SCHEME (0 WENO-JS, 1 WENO-Z, 2 WENOEXP)
    limiter: int = 0         # PPlimiter
    flux: int = 0            # RIEMANNFLUX (0 LLF, 1 HLLC)
    recon: int = 1           # RECONSTRUCTIONTYPE (0 conservative, 1 characteristic, 2-4 primitive)
    ref_slabs: int = 0       # 4 = the reference's 4-slab grid metric
    threads: int = 0
    eq_kind: int = EQ_TWO_PHASE
    rho10: float = 1.2
    rho20: float = 1.0
    sound1: float = 1.0
    sound2: float = 1.0
    preb: float = 0.0
    gamma: float = 1.4
    adv_u: float = 1.0
    adv_v: float = 1.0
    # stiffened-gas phases (EQ_TWO_PHASE_SG): isentropes through (preb, rho10) and (preb, rho20)
    gamma1: float = 4.4
    pinf1: float = 6.0e3
    gamma2: float = 1.4
    pinf2: float = 0.0
    gravity: float = 0.0     # assembleSourceTerm's g_g0 (two-phase kinds)
    # NEUMANN2: fixed ghost averages [nvar][ny+8][nx+8], interior at offset (4, 4)
    frame: np.ndarray | None = None

    @property
    def nvar(self) -> int:
        return 1 if self.eq_kind == EQ_LINEAR_ADV else 4

    def to_c(self) -> _Problem:
        e = _Eq(self.eq_kind, self.rho10, self.rho20, self.sound1, self.sound2, self.preb,
                self.gamma, self.adv_u, self.adv_v, self.gamma1, self.pinf1, self.gamma2, self.pinf2, self.gravity)
        fp = None
        if self.bc == BC_NEUMANN2:
            if self.frame is None:
                raise ValueError("NEUMANN2 needs a frame of ghost averages")
            fr = np.ascontiguousarray(self.frame, dtype=np.float64)
            if fr.shape != (self.nvar, self.ny + 8, self.nx + 8):
                raise ValueError(f"frame shape {fr.shape} != {(self.nvar, self.ny + 8, self.nx + 8)}")
            self._frame_keep = fr  # the C struct holds a raw pointer into it
            fp = fr.ctypes.data
        return _Problem(self.nx, self.ny, self.xl, self.xr, self.yl, self.yr, self.bc, self.rk,
                        self.cfl, self.scheme, self.limiter, self.flux, self.recon, self.ref_slabs,
                        self.threads, e, fp)


_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class Oracle:
    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        L = C.CDLL(path)
        PP = C.POINTER(_Problem)
        EP = C.POINTER(_Eq)
        L.ofv_weno_js.restype = C.c_double
        L.ofv_weno_js.argtypes = [_DP, C.c_int]
        L.ofv_weno_z.restype = C.c_double
        L.ofv_weno_z.argtypes = [_DP, C.c_int]
        L.ofv_weno_exp.restype = C.c_double
        L.ofv_weno_exp.argtypes = [_DP, C.c_int, C.c_double]
        L.ofv_weno_exp_thinc.restype = C.c_double
        L.ofv_weno_exp_thinc.argtypes = [_DP, C.c_int, C.c_double]
        L.ofv_set_cube_rounded.argtypes = [C.c_int]
        L.ofv_set_thinc_ulp.argtypes = [C.c_int]
        for n in ("ofv_volume_frac", "ofv_pressure", "ofv_sound_speed"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [EP, _DP]
        L.ofv_max_eig.restype = C.c_double
        L.ofv_max_eig.argtypes = [EP, _DP, C.c_double, C.c_double]
        L.ofv_riemann.argtypes = [EP, C.c_int, _DP, _DP, C.c_double, C.c_double, _DP]
        L.ofv_eigen_L.argtypes = [EP, _DP, C.c_double, C.c_double, _DP]
        L.ofv_eigen_R.argtypes = [EP, _DP, C.c_double, C.c_double, _DP]
        L.ofv_metric.argtypes = [PP, _DP, _DP, _DP]
        L.ofv_compute_dt.restype = C.c_double
        L.ofv_compute_dt.argtypes = [PP, _DP, C.POINTER(C.c_int)]
        L.ofv_rhs.argtypes = [PP, _DP, _DP, C.c_void_p]
        L.ofv_face_states.argtypes = [PP, _DP, _DP]
        L.ofv_step.argtypes = [PP, _DP, C.c_double]
        L.ofv_advance.restype = C.c_int
        L.ofv_advance.argtypes = [PP, _DP, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_int,
                                  C.c_void_p]
        self.L = L

    @contextlib.contextmanager
    def cube_rounded(self):
        """WENOEXP's l^3 rounded once (the device kernels' form) instead of the C library's
        pow(l, 3) (the reference's) inside the block.  The switch is process-wide."""
        self.L.ofv_set_cube_rounded(1)
        try:
            yield self
        finally:
            self.L.ofv_set_cube_rounded(0)

    @contextlib.contextmanager
    def thinc_ulp(self):
        """PRIMITIVE3's THINC exp/log/tanh each moved one ulp up inside the block: the
        difference to the default run measures how far the reference's own result moves
        with the last bit of its math library.  The switch is process-wide."""
        self.L.ofv_set_thinc_ulp(1)
        try:
            yield self
        finally:
            self.L.ofv_set_thinc_ulp(0)

    # pointwise -----------------------------------------------------------------
    def weno(self, scheme: int, v, gp: int, dx: float = 0.0) -> float:
        """One Gauss-point value: WENO-JS/Z on 5 values, WENOEXP (scheme 2) on 7 and dx, and
        PRIMITIVE3's WENOEXP/THINC z1 kernel (scheme "thinc") on 7 and dx."""
        a = np.ascontiguousarray(v, dtype=np.float64)
        if scheme == "thinc":
            assert a.size == 7
            return self.L.ofv_weno_exp_thinc(a, gp, dx)
        if scheme == 2:
            assert a.size == 7
            return self.L.ofv_weno_exp(a, gp, dx)
        return (self.L.ofv_weno_z if scheme == 1 else self.L.ofv_weno_js)(a, gp)

    def riemann(self, p: Problem, flux: int, UL, UR, nx: float, ny: float) -> np.ndarray:
        out = np.zeros(4)
        e = p.to_c().eq
        self.L.ofv_riemann(C.byref(e), flux, np.ascontiguousarray(UL, dtype=np.float64),
                           np.ascontiguousarray(UR, dtype=np.float64), nx, ny, out)
        return out[: p.nvar]

    def eigen(self, p: Problem, U, nx: float, ny: float):
        L = np.zeros(16)
        R = np.zeros(16)
        e = p.to_c().eq
        u = np.ascontiguousarray(U, dtype=np.float64)
        self.L.ofv_eigen_L(C.byref(e), u, nx, ny, L)
        self.L.ofv_eigen_R(C.byref(e), u, nx, ny, R)
        n = p.nvar
        return L[: n * n].reshape(n, n), R[: n * n].reshape(n, n)

    def thermo(self, p: Problem, U):
        """(volume fraction, pressure less preb, sound speed) of one state"""
        e = p.to_c().eq
        u = np.ascontiguousarray(U, dtype=np.float64)
        return (self.L.ofv_volume_frac(C.byref(e), u), self.L.ofv_pressure(C.byref(e), u),
                self.L.ofv_sound_speed(C.byref(e), u))

    def max_eig(self, p: Problem, U, nx: float, ny: float) -> float:
        e = p.to_c().eq
        return self.L.ofv_max_eig(C.byref(e), np.ascontiguousarray(U, dtype=np.float64), nx, ny)

    # grid operators ------------------------------------------------------------
    def metric(self, p: Problem):
        dxc, dxl, dy = np.zeros(p.nx), np.zeros(p.nx), np.zeros(p.ny)
        self.L.ofv_metric(C.byref(p.to_c()), dxc, dxl, dy)
        return dxc, dxl, dy

    def compute_dt(self, p: Problem, U: np.ndarray) -> float:
        flag = C.c_int(0)
        return self.L.ofv_compute_dt(C.byref(p.to_c()), np.ascontiguousarray(U), C.byref(flag))

    def rhs(self, p: Problem, U: np.ndarray) -> np.ndarray:
        out = np.zeros_like(U)
        self.L.ofv_rhs(C.byref(p.to_c()), np.ascontiguousarray(U), out, None)
        return out

    def face_states(self, p: Problem, U: np.ndarray) -> np.ndarray:
        out = np.zeros(p.nx * p.ny * 16 * p.nvar)
        self.L.ofv_face_states(C.byref(p.to_c()), np.ascontiguousarray(U), out)
        return out.reshape(p.ny, p.nx, 4, p.nvar, 4)

    def step(self, p: Problem, U: np.ndarray, dt: float) -> np.ndarray:
        V = np.array(U, dtype=np.float64, copy=True)
        self.L.ofv_step(C.byref(p.to_c()), V, dt)
        return V

    def advance(self, p: Problem, U: np.ndarray, t_end: float, t0: float = 0.0, max_steps: int = 0):
        V = np.array(U, dtype=np.float64, copy=True)
        cap = max_steps if max_steps > 0 else 1_000_000
        dts = np.zeros(cap)
        tout = C.c_double(0.0)
        n = self.L.ofv_advance(C.byref(p.to_c()), V, t0, t_end, C.byref(tout), max_steps,
                               dts.ctypes.data_as(C.c_void_p))
        return V, n, tout.value, dts[:n]


# ---------------------------------------------------------------------------------
# the compiled reference
# ---------------------------------------------------------------------------------

@dataclass
class RefResult:
    U: np.ndarray | None = None
    U0: np.ndarray | None = None
    rhs: np.ndarray | None = None
    faces: np.ndarray | None = None
    dts: np.ndarray | None = None
    timing: dict = field(default_factory=dict)


def _f(x) -> str:
    """shortest round-trip decimal of a float (numpy scalars included)"""
    return repr(float(x))


def reference_available() -> bool:
    return os.path.exists(REF_BIN)


def run_reference(p: Problem, testcase: int = 0, U0: np.ndarray | None = None, steps: int = 0,
                  t_end: float = 0.0, want_rhs: bool = False, time: bool = False,
                  timeout: float = 600.0, warmup: int = 0, source_case: int = -1) -> RefResult:
    """Run the unmodified reference (4 slab ranks) on the two-phase system.

    ``testcase`` selects the reference's own test case (its domain, boundary and, when
    ``U0`` is None, its initial averages).  Equation parameters of ``p`` override the
    test case's (the harness writes them into TwoPhaseEquation after initializeSolver).
    """
    if not reference_available():
        raise FileNotFoundError(f"{REF_BIN} missing: run `make -C oracle ref`")
    n = 4 * p.nx * p.ny
    with tempfile.TemporaryDirectory() as d:
        args = [REF_BIN, "--testcase", str(testcase), "--nx", str(p.nx), "--ny", str(p.ny),
                "--rk", str(p.rk), "--cfl", _f(p.cfl), "--scheme", str(p.scheme),
                "--limiter", str(p.limiter), "--flux", str(p.flux), "--recon", str(p.recon),
                "--rho10", _f(p.rho10), "--rho20", _f(p.rho20), "--sound1", _f(p.sound1),
                "--sound2", _f(p.sound2),
                "--dump-u0", os.path.join(d, "u0.bin"), "--out", os.path.join(d, "u.bin"),
                "--dts", os.path.join(d, "dts.bin")]
        if U0 is not None:
            np.ascontiguousarray(U0, dtype=np.float64).tofile(os.path.join(d, "in.bin"))
            args += ["--u0", os.path.join(d, "in.bin")]
        if t_end > 0:
            args += ["--tend", _f(t_end)]
        else:
            args += ["--steps", str(steps)]
        if want_rhs:
            args += ["--rhs", os.path.join(d, "rhs.bin"), "--faces", os.path.join(d, "faces.bin")]
        if time:
            args += ["--time"]
        if warmup:
            args += ["--warmup", str(warmup)]
        if source_case >= 0:  # the test case of assembleSourceTerm (its gravity)
            args += ["--source-case", str(source_case)]
        cp = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
        if cp.returncode != 0:
            raise RuntimeError(f"reference failed ({cp.returncode}): {cp.stderr[-2000:]}")
        shape = (4, p.ny, p.nx)
        r = RefResult()
        r.U = np.fromfile(os.path.join(d, "u.bin")).reshape(shape)
        r.U0 = np.fromfile(os.path.join(d, "u0.bin")).reshape(shape)
        r.dts = np.fromfile(os.path.join(d, "dts.bin"))
        if want_rhs:
            r.rhs = np.fromfile(os.path.join(d, "rhs.bin")).reshape(shape)
            r.faces = np.fromfile(os.path.join(d, "faces.bin")).reshape(p.ny, p.nx, 4, 4, 4)
        if time:
            r.timing = json.loads(cp.stdout.strip().splitlines()[-1])
        assert r.U.size == n
        return r
