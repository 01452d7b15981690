"""ctypes binding of libwenofv_b200.so (the C ABI in include/wenofv.h).

This is plumbing for the tests and bench.py: the host API that mirrors the reference's
CWENOFV / TwoPhaseEquation / CConfig is the C++ code under host/.  Every call goes to the
sm_100a kernels; there is no CPU path.  Loading fails loudly when the library is missing.

Arrays cross the boundary as float64 numpy arrays in SoA layout ``U[v, j, i]`` unless a
layout constant says otherwise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# WENOFV_LIB selects another build of the library, e.g. lib/libwenofv_b200_checked.so
LIB_PATH = os.environ.get("WENOFV_LIB") or os.path.join(HERE, "lib", "libwenofv_b200.so")

OK, EINVAL, ENOMEM, ENUMERIC, ETIMEDOUT, ECUDA, ENOTSUP, EBUSY, ENOTFOUND = range(9)
EQ_TWO_PHASE, EQ_LINEAR_ADV, EQ_EULER, EQ_TWO_PHASE_SG = 0, 1, 2, 3
BC_PERIOD, BC_NEUMANN, BC_NOSLIP, BC_NEUMANN2, BC_FREESLIP, BC_OUTFLOW = 0, 1, 2, 3, 4, 5
FP64, FP64_STRICT, FP32_BULK = 0, 1, 2
LAYOUT_SOA, LAYOUT_REF_AOS = 0, 1
FLAG_NAN_DT, FLAG_BAD_THETA, FLAG_NAN_FLUX, FLAG_NAN_STATE, FLAG_BOUNDS = 1, 2, 4, 8, 16

# every entry point declared in include/wenofv.h
EXPORTS = (
    "wenofv_abi_version", "wenofv_strerror", "wenofv_last_error", "wenofv_default_config",
    "wenofv_create", "wenofv_destroy", "wenofv_upload", "wenofv_set_frame", "wenofv_download", "wenofv_compute_dt",
    "wenofv_step", "wenofv_rhs", "wenofv_advance", "wenofv_status", "wenofv_synchronize",
    "wenofv_stream", "wenofv_device_state", "wenofv_theta_flags", "wenofv_snapshot_begin", "wenofv_snapshot_wait",
    "wenofv_step_noalloc", "wenofv_init_testcase", "wenofv_accuracy",
    "wenofv_batch_create", "wenofv_batch_destroy", "wenofv_batch_upload", "wenofv_batch_set_frame", "wenofv_batch_download",
    "wenofv_batch_advance", "wenofv_batch_set_tiling", "wenofv_batch_stream", "wenofv_batch_autotune",
    "wenofv_batch_set_threads", "wenofv_batch_tiling",
    "wenofv_server_create", "wenofv_server_destroy", "wenofv_server_submit", "wenofv_server_poll",
    "wenofv_server_clock", "wenofv_server_stats",
    "wenofv_probe_weno", "wenofv_probe_weno_exp", "wenofv_probe_riemann", "wenofv_probe_eigen", "wenofv_probe_fma_peak",
)


class EqParams(C.Structure):
    """wenofv_eq_params: TwoPhaseEquation's g_rho10, g_rho20, g_sound1, g_sound2, g_preb + extensions"""
    _fields_ = [("eq_kind", C.c_int), ("rho10", C.c_double), ("rho20", C.c_double),
                ("sound1", C.c_double), ("sound2", C.c_double), ("preb", C.c_double),
                ("gamma", C.c_double), ("adv_u", C.c_double), ("adv_v", C.c_double),
                ("gamma1", C.c_double), ("pinf1", C.c_double), ("gamma2", C.c_double), ("pinf2", C.c_double),
                ("gravity", C.c_double)]


class Config(C.Structure):
    """wenofv_config: the settings.cfg keys plus domain, boundary, metric, form and device"""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("xl", C.c_double), ("xr", C.c_double),
                ("yl", C.c_double), ("yr", C.c_double), ("bc", C.c_int), ("rk_method", C.c_int),
                ("cfl", C.c_double), ("scheme", C.c_int), ("pp_limiter", C.c_int),
                ("riemann_flux", C.c_int), ("reconstruction", C.c_int), ("ref_slabs", C.c_int),
                ("precision", C.c_int), ("device", C.c_int)]


class TestCase(C.Structure):
    _fields_ = [("testcase", C.c_int), ("u0", C.c_double), ("v0", C.c_double), ("epsa", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("steps", C.c_int64), ("flags", C.c_uint32), ("status", C.c_int)]


class WenofvError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {what_code(code)} ({code})")


_lib = None


def what_code(code: int) -> str:
    L = load()
    return L.wenofv_strerror(code).decode() + " -- " + L.wenofv_last_error().decode()


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the library once; raises when it is absent (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with __graft_entry__.build() or make -C {HERE}")
    L = C.CDLL(path)
    P, D, I, I64 = C.c_void_p, C.c_double, C.c_int, C.c_int64
    DP = C.POINTER(C.c_double)
    L.wenofv_abi_version.restype = I
    L.wenofv_strerror.restype = C.c_char_p
    L.wenofv_strerror.argtypes = [I]
    L.wenofv_last_error.restype = C.c_char_p
    L.wenofv_default_config.argtypes = [C.POINTER(Config)]
    L.wenofv_create.argtypes = [C.POINTER(Config), C.POINTER(EqParams), C.POINTER(P)]
    L.wenofv_destroy.argtypes = [P]
    L.wenofv_upload.argtypes = [P, DP, I]
    L.wenofv_download.argtypes = [P, DP, I]
    L.wenofv_set_frame.argtypes = [P, DP]
    L.wenofv_batch_set_frame.argtypes = [P, I, DP]
    L.wenofv_compute_dt.argtypes = [P, DP]
    L.wenofv_step.argtypes = [P, D]
    L.wenofv_rhs.argtypes = [P, DP, I]
    L.wenofv_advance.argtypes = [P, D, D, I64, DP, C.POINTER(I64)]
    L.wenofv_status.argtypes = [P, C.POINTER(C.c_uint32), C.POINTER(I64)]
    L.wenofv_synchronize.argtypes = [P]
    L.wenofv_stream.restype = P
    L.wenofv_stream.argtypes = [P]
    L.wenofv_device_state.argtypes = [P, C.POINTER(P), C.POINTER(I)]
    L.wenofv_theta_flags.argtypes = [P, C.POINTER(C.c_uint8), I]
    L.wenofv_snapshot_begin.argtypes = [P, DP, I]
    L.wenofv_snapshot_wait.argtypes = [P]
    L.wenofv_batch_create.argtypes = [I, C.POINTER(Config), C.POINTER(EqParams), C.POINTER(P)]
    L.wenofv_batch_destroy.argtypes = [P]
    L.wenofv_batch_upload.argtypes = [P, I, DP, I]
    L.wenofv_batch_download.argtypes = [P, I, DP, I]
    L.wenofv_batch_advance.argtypes = [P, DP, I64, C.POINTER(I64)]
    L.wenofv_batch_set_tiling.argtypes = [P, I, I]
    L.wenofv_batch_stream.argtypes = [P, C.POINTER(P)]
    L.wenofv_batch_autotune.argtypes = [P, C.POINTER(I), C.POINTER(I), DP]
    L.wenofv_batch_set_threads.argtypes = [P, I]
    L.wenofv_batch_tiling.argtypes = [P, C.POINTER(I), C.POINTER(I), C.POINTER(I)]
    L.wenofv_server_create.argtypes = [I, C.c_size_t, I, C.POINTER(P)]
    L.wenofv_server_destroy.argtypes = [P]
    L.wenofv_server_submit.argtypes = [P, C.POINTER(Config), C.POINTER(EqParams), DP, D, I64, C.POINTER(I64)]
    L.wenofv_server_poll.argtypes = [P, I64, DP, C.POINTER(RequestInfo)]
    L.wenofv_server_clock.restype = D
    L.wenofv_server_clock.argtypes = [P]
    L.wenofv_server_stats.argtypes = [P] + [C.POINTER(I64)] * 5
    L.wenofv_probe_weno.argtypes = [I, I, DP, I, DP, I]
    L.wenofv_probe_weno_exp.argtypes = [I, DP, I, D, DP, I]
    L.wenofv_probe_riemann.argtypes = [C.POINTER(EqParams), I, I, DP, DP, I, D, D, DP, I]
    L.wenofv_probe_eigen.argtypes = [C.POINTER(EqParams), I, DP, I, D, D, DP, DP, I]
    L.wenofv_probe_fma_peak.argtypes = [I, I, DP]
    L.wenofv_init_testcase.argtypes = [P, C.POINTER(TestCase)]
    L.wenofv_accuracy.argtypes = [P, C.POINTER(TestCase), D, DP]
    L.wenofv_step_noalloc.argtypes = [C.POINTER(Config), C.POINTER(EqParams), P, P, I, D, P, C.POINTER(C.c_uint32)]
    _lib = L
    return L


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(rc: int, what: str):
    if rc != OK:
        raise WenofvError(rc, what)


def make_config(nx: int, ny: int, *, xl=0.0, xr=1.0, yl=0.0, yr=1.0, bc=BC_PERIOD, rk=2, cfl=0.5,
                scheme=1, limiter=0, flux=0, recon=1, ref_slabs=0, precision=FP64, device=0) -> Config:
    return Config(nx, ny, xl, xr, yl, yr, bc, rk, cfl, scheme, limiter, flux, recon, ref_slabs,
                  precision, device)


def make_eq(kind=EQ_TWO_PHASE, rho10=1.2, rho20=1.0, sound1=1.0, sound2=1.0, preb=0.0, gamma=1.4,
            adv_u=1.0, adv_v=1.0, gamma1=4.4, pinf1=6.0e3, gamma2=1.4, pinf2=0.0, gravity=0.0) -> EqParams:
    """kind EQ_TWO_PHASE_SG: stiffened-gas phases (gamma_k, pinf_k) on their isentropes through
    (preb, rho10) and (preb, rho20); sound1/sound2 are ignored"""
    return EqParams(kind, rho10, rho20, sound1, sound2, preb, gamma, adv_u, adv_v, gamma1, pinf1, gamma2, pinf2, gravity)


def nvar(eq: EqParams) -> int:
    return 1 if eq.eq_kind == EQ_LINEAR_ADV else 4


class Solver:
    """One grid on one GPU (wenofv_ctx)."""

    def __init__(self, cfg: Config, eq: EqParams):
        self.L = load()
        self.cfg, self.eq = cfg, eq
        self.nv = nvar(eq)
        h = C.c_void_p()
        _check(self.L.wenofv_create(C.byref(cfg), C.byref(eq), C.byref(h)), "wenofv_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.wenofv_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.nv, self.cfg.ny, self.cfg.nx)

    def upload(self, U: np.ndarray, layout=LAYOUT_SOA):
        a = np.ascontiguousarray(U, dtype=np.float64)
        _check(self.L.wenofv_upload(self.h, _dp(a), layout), "wenofv_upload")

    def set_frame(self, frame: np.ndarray):
        """NEUMANN2 ghost averages, [nv][ny+8][nx+8] with cell (i, j) at [v][j+4][i+4]."""
        a = np.ascontiguousarray(frame, dtype=np.float64)
        if a.shape != (self.nv, self.cfg.ny + 8, self.cfg.nx + 8):
            raise ValueError(f"frame shape {a.shape} != {(self.nv, self.cfg.ny + 8, self.cfg.nx + 8)}")
        _check(self.L.wenofv_set_frame(self.h, _dp(a)), "wenofv_set_frame")

    def download(self, layout=LAYOUT_SOA) -> np.ndarray:
        out = np.empty(self.shape if layout == LAYOUT_SOA else (self.cfg.nx, self.cfg.ny, self.nv))
        _check(self.L.wenofv_download(self.h, _dp(out), layout), "wenofv_download")
        return out

    def download_into(self, out: np.ndarray, layout=LAYOUT_SOA) -> np.ndarray:
        """download into a caller's C-contiguous float64 array (e.g. pinned host memory)"""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != int(np.prod(self.shape)):
            raise ValueError("need a C-contiguous float64 array of the state's size")
        _check(self.L.wenofv_download(self.h, _dp(out), layout), "wenofv_download")
        return out

    def init_testcase(self, testcase: int, u0: float, v0: float, epsa: float):
        """the reference's initial averages of a periodic test case, computed on the GPU"""
        tc = TestCase(testcase, u0, v0, epsa)
        _check(self.L.wenofv_init_testcase(self.h, C.byref(tc)), "wenofv_init_testcase")

    def accuracy(self, testcase: int, u0: float, v0: float, epsa: float, t: float):
        """(L_inf, L1, L2) of z1 against the translated initial data, computed on the GPU"""
        tc = TestCase(testcase, u0, v0, epsa)
        out = np.zeros(3)
        _check(self.L.wenofv_accuracy(self.h, C.byref(tc), t, _dp(out)), "wenofv_accuracy")
        return tuple(out)

    def compute_dt(self) -> float:
        d = C.c_double()
        _check(self.L.wenofv_compute_dt(self.h, C.byref(d)), "wenofv_compute_dt")
        return d.value

    def step(self, dt: float):
        _check(self.L.wenofv_step(self.h, dt), "wenofv_step")

    def rhs(self) -> np.ndarray:
        out = np.empty(self.shape)
        _check(self.L.wenofv_rhs(self.h, _dp(out), LAYOUT_SOA), "wenofv_rhs")
        return out

    def advance(self, t_end: float, t_now: float = 0.0, max_steps: int = 0):
        t = C.c_double()
        n = C.c_int64()
        _check(self.L.wenofv_advance(self.h, t_now, t_end, max_steps, C.byref(t), C.byref(n)), "wenofv_advance")
        return t.value, n.value

    def status(self):
        f = C.c_uint32()
        c = C.c_int64()
        _check(self.L.wenofv_status(self.h, C.byref(f), C.byref(c)), "wenofv_status")
        return f.value, c.value

    def synchronize(self):
        _check(self.L.wenofv_synchronize(self.h), "wenofv_synchronize")

    def stream(self) -> int:
        return self.L.wenofv_stream(self.h) or 0

    def theta_flags(self, layout=LAYOUT_SOA) -> np.ndarray:
        """the final stage's per-cell limiter record (1 where theta < 1 - 1e-8)"""
        out = np.zeros((self.cfg.ny, self.cfg.nx) if layout == LAYOUT_SOA else (self.cfg.nx, self.cfg.ny), np.uint8)
        _check(self.L.wenofv_theta_flags(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8)), layout), "wenofv_theta_flags")
        return out

    def snapshot_begin(self, out: np.ndarray, layout=LAYOUT_SOA):
        """asynchronous copy of the current state into out (kept alive until snapshot_wait)"""
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.size != int(np.prod(self.shape)):
            raise ValueError("need a C-contiguous float64 array of the state's size")
        self._snap = out
        _check(self.L.wenofv_snapshot_begin(self.h, _dp(out), layout), "wenofv_snapshot_begin")

    def snapshot_wait(self) -> np.ndarray:
        _check(self.L.wenofv_snapshot_wait(self.h), "wenofv_snapshot_wait")
        out, self._snap = getattr(self, "_snap", None), None
        return out

    def device_state(self):
        p = C.c_void_p()
        pitch = C.c_int()
        _check(self.L.wenofv_device_state(self.h, C.byref(p), C.byref(pitch)), "wenofv_device_state")
        return p.value, pitch.value


class Batch:
    """Many uneven instances advanced together (wenofv_batch)."""

    def __init__(self, cfgs, eqs):
        self.L = load()
        n = len(cfgs)
        self.cfgs = (Config * n)(*cfgs)
        self.eqs = (EqParams * n)(*eqs)
        self.n = n
        h = C.c_void_p()
        _check(self.L.wenofv_batch_create(n, self.cfgs, self.eqs, C.byref(h)), "wenofv_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.wenofv_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def shape(self, i):
        return (nvar(self.eqs[i]), self.cfgs[i].ny, self.cfgs[i].nx)

    def upload(self, i, U):
        a = np.ascontiguousarray(U, dtype=np.float64)
        _check(self.L.wenofv_batch_upload(self.h, i, _dp(a), LAYOUT_SOA), "wenofv_batch_upload")

    def set_frame(self, i, frame: np.ndarray):
        nv, ny, nx = self.shape(i)
        a = np.ascontiguousarray(frame, dtype=np.float64)
        if a.shape != (nv, ny + 8, nx + 8):
            raise ValueError(f"frame shape {a.shape} != {(nv, ny + 8, nx + 8)}")
        _check(self.L.wenofv_batch_set_frame(self.h, i, _dp(a)), "wenofv_batch_set_frame")

    def download(self, i) -> np.ndarray:
        out = np.empty(self.shape(i))
        _check(self.L.wenofv_batch_download(self.h, i, _dp(out), LAYOUT_SOA), "wenofv_batch_download")
        return out

    def advance(self, t_end, max_steps: int = 0):
        te = np.ascontiguousarray(np.broadcast_to(np.asarray(t_end, dtype=np.float64), (self.n,)))
        ns = (C.c_int64 * self.n)()
        _check(self.L.wenofv_batch_advance(self.h, _dp(te), max_steps, ns), "wenofv_batch_advance")
        return np.array(ns[:], dtype=np.int64)

    def set_tiling(self, rows: int, ctas_per_sm: int = 0):
        _check(self.L.wenofv_batch_set_tiling(self.h, rows, ctas_per_sm), "wenofv_batch_set_tiling")

    def set_threads(self, threads_per_cta: int):
        """0: per instance (the default); 128 or 256: that CTA width wherever it exists"""
        _check(self.L.wenofv_batch_set_threads(self.h, threads_per_cta), "wenofv_batch_set_threads")

    def tiling(self):
        """(rows per item, CTAs per SM, threads per CTA); 0 = automatic"""
        r, c, t = C.c_int(), C.c_int(), C.c_int()
        _check(self.L.wenofv_batch_tiling(self.h, C.byref(r), C.byref(c), C.byref(t)), "wenofv_batch_tiling")
        return r.value, c.value, t.value

    def autotune(self):
        r, c, ms = C.c_int(), C.c_int(), C.c_double()
        _check(self.L.wenofv_batch_autotune(self.h, C.byref(r), C.byref(c), C.byref(ms)), "wenofv_batch_autotune")
        return r.value, c.value, ms.value

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self.L.wenofv_batch_stream(self.h, C.byref(s)), "wenofv_batch_stream")
        return s.value or 0


class Server:
    """Continuous-batching solve server (wenofv_server)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 << 30, max_slots: int = 256):
        self.L = load()
        h = C.c_void_p()
        _check(self.L.wenofv_server_create(device, hbm_budget_bytes, max_slots, C.byref(h)), "wenofv_server_create")
        self.h = h
        self.shapes = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.wenofv_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def submit(self, cfg: Config, eq: EqParams, U0: np.ndarray, t_end: float, max_steps: int = 0) -> int:
        a = np.ascontiguousarray(U0, dtype=np.float64)
        rid = C.c_int64()
        _check(self.L.wenofv_server_submit(self.h, C.byref(cfg), C.byref(eq), _dp(a), t_end, max_steps, C.byref(rid)),
               "wenofv_server_submit")
        self.shapes[rid.value] = (nvar(eq), cfg.ny, cfg.nx)
        return rid.value

    def poll(self, rid: int):
        """(U, info) when done, None while running; raises WenofvError for a failed request"""
        out = np.empty(self.shapes[rid])
        info = RequestInfo()
        rc = self.L.wenofv_server_poll(self.h, rid, _dp(out), C.byref(info))
        if rc == EBUSY:
            return None
        del self.shapes[rid]
        _check(rc, "wenofv_server_poll")
        return out, info

    def clock(self) -> float:
        return self.L.wenofv_server_clock(self.h)

    def stats(self):
        v = [C.c_int64() for _ in range(5)]
        _check(self.L.wenofv_server_stats(self.h, *[C.byref(x) for x in v]), "wenofv_server_stats")
        return dict(zip(("admitted", "completed", "queued", "active", "resident_bytes"), [x.value for x in v]))


# ---- device probes of the pointwise kernels ---------------------------------------------------
def probe_weno(scheme: int, stencils: np.ndarray, precision=FP64, device=0) -> np.ndarray:
    L = load()
    s = np.ascontiguousarray(stencils, dtype=np.float64).reshape(-1, 5)
    out = np.empty((s.shape[0], 4))
    _check(L.wenofv_probe_weno(scheme, precision, _dp(s), s.shape[0], _dp(out), device), "wenofv_probe_weno")
    return out


def probe_weno_exp(stencils: np.ndarray, dx: float, precision=FP64, device=0) -> np.ndarray:
    L = load()
    s = np.ascontiguousarray(stencils, dtype=np.float64).reshape(-1, 7)
    out = np.empty((s.shape[0], 4))
    _check(L.wenofv_probe_weno_exp(precision, _dp(s), s.shape[0], dx, _dp(out), device), "wenofv_probe_weno_exp")
    return out


def probe_riemann(eq: EqParams, flux: int, UL, UR, nx: float, ny: float, precision=FP64, device=0) -> np.ndarray:
    L = load()
    nv = nvar(eq)
    l = np.ascontiguousarray(UL, dtype=np.float64).reshape(-1, nv)
    r = np.ascontiguousarray(UR, dtype=np.float64).reshape(-1, nv)
    out = np.empty_like(l)
    _check(L.wenofv_probe_riemann(C.byref(eq), flux, precision, _dp(l), _dp(r), l.shape[0], nx, ny, _dp(out), device),
           "wenofv_probe_riemann")
    return out


def probe_eigen(eq: EqParams, U, nx: float, ny: float, precision=FP64, device=0):
    L = load()
    nv = nvar(eq)
    u = np.ascontiguousarray(U, dtype=np.float64).reshape(-1, nv)
    Lm = np.zeros((u.shape[0], 16))
    Rm = np.zeros((u.shape[0], 16))
    _check(L.wenofv_probe_eigen(C.byref(eq), precision, _dp(u), u.shape[0], nx, ny, _dp(Lm), _dp(Rm), device),
           "wenofv_probe_eigen")
    return Lm[:, : nv * nv].reshape(-1, nv, nv), Rm[:, : nv * nv].reshape(-1, nv, nv)


def fma_peak_tflops(precision=FP64, device=0) -> float:
    """measured FMA throughput of the FP64 (or FP32) CUDA-core pipe, TFLOP/s"""
    L = load()
    t = C.c_double()
    _check(L.wenofv_probe_fma_peak(precision, device, C.byref(t)), "wenofv_probe_fma_peak")
    return t.value
