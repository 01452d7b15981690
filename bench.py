"""Benchmark of the WENOFV time-advance hot path on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload column1024|column1024_exp|euler512|advection128] [--form fp64|fp64_strict|fp32_bulk]

A step is one SSP-RK3 time step (3 fused stage launches, the last with the CFL
reduction) over the whole grid of the workload.  The metric is cell-stage updates per
second: interior cells x RK stages x steps / time.

* value: K steps on the device-resident state, each timed with CUDA events on the solver's
  stream; L2 (126 MB) is flushed by a 256 MiB write between steps, outside the timed events.
* e2e: the same K steps through the public C-ABI calls with host arrays: upload of the
  step's input state, the step, download of its result.
* roofline: the stage kernel is bound by the FP64 CUDA-core pipe (the path is a stencil,
  not a contraction); achieved = counted algorithmic flops per launch (profiles/flop_table.txt)
  / average launch time; peak = FMA throughput measured in this run by the library's probe.
* cpu_baseline: the unmodified reference (oracle/_ref, 4 slab ranks per process, as many
  processes as the host has groups of 4 cores) on a bounded sample of the same workload.
* --impl reference: that reference arm alone, on rank 0 (other ranks exit 0).

Multi-GPU (torchrun): replicas only -- each rank advances its own copy of the workload on
its own GPU with no collective on the data path; the barrier and the max over ranks of the
timed duration use torch.distributed.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import cases  # noqa: E402

# option sets of the workloads, for the flop table lookup
FLOP_KEYS = {
    "column1024": ("two_phase", 1, 1, 1, 1),    # characteristic, WENO-Z, HLLC, limiter
    "column1024_exp": ("two_phase", 1, 2, 1, 1),  # the same with WENOEXP (7-point stencils)
    "column1024_prim3": ("two_phase", 4, 1, 1, 1),  # PRIMITIVE3: z1 by WENOEXP/THINC, p, u, v by WENO-Z
    "column1024_sg": ("two_phase_sg", 1, 1, 1, 1),  # the column with stiffened-gas phases
    "euler512": ("euler", 0, 1, 1, 0),          # conservative, WENO-Z, HLLC
    "advection128": ("linear_advection", 0, 0, 0, 0),
}
BYTES_PER_CELL_STAGE = {"column1024": 96.0, "column1024_exp": 96.0, "column1024_prim3": 96.0, "column1024_sg": 96.0,
                        "euler512": 96.0, "advection128": 24.0}


def flops_per_cell_stage(name: str) -> float:
    eq, recon, scheme, flux, lim = FLOP_KEYS[name]
    for line in open(os.path.join(ROOT, "profiles", "flop_table.txt")):
        if not line.startswith("{"):
            continue
        d = json.loads(line)
        if (d["eq"], d["recon"], d["scheme"], d["flux"], d["limiter"]) == (eq, recon, scheme, flux, lim):
            return float(d["flops_per_cell_stage"])
    raise KeyError(name)


def workload_desc(name: str) -> dict:
    """the description of a named workload (its `config` in the JSON line, both arms)"""
    if name in ("column1024", "column1024_exp", "column1024_prim3"):
        sch = 2 if name == "column1024_exp" else 1
        rec = 4 if name == "column1024_prim3" else 1
        return dict(workload="liquid_column_1024_ref_eos" + {"column1024": "", "column1024_exp": "_wenoexp",
                                                             "column1024_prim3": "_primitive3"}[name], grid="1024x1024",
                    equation="two-phase 3-equation, linear EOS "
                    "linearised from stiffened gas (g1=4.4, pinf1=6e3, g2=1.4, pinf2=0) at p=1, density ratio 1000",
                    bc="periodic", scheme="WENOEXP" if sch == 2 else ("WENOEXP/THINC (z1), WENO-Z" if rec == 4 else "WENO-Z"),
                    flux="HLLC", reconstruction="primitive3 (z1, p, u, v)" if rec == 4 else "characteristic", limiter=True,
                    rk="SSP-RK3", cfl=0.5, ic="disk r=0.2 tanh-smoothed over 2 cells, eps=1e-6, seeded periodic "
                    "Gaussian velocity field amplitude 1e-2 (seed 3)")
    if name == "column1024_sg":
        return dict(workload="liquid_column_1024_stiffened_gas", grid="1024x1024",
                    equation="two-phase 3-equation, stiffened-gas phases on their isentropes (g1=4.4, pinf1=6e3; "
                    "g2=1.4, pinf2=0) through p=1, density ratio 1000, Newton pressure equilibrium",
                    bc="periodic", scheme="WENO-Z", flux="HLLC", reconstruction="characteristic", limiter=True,
                    rk="SSP-RK3", cfl=0.5, ic="disk r=0.2 tanh-smoothed over 2 cells, eps=1e-6, p=1, seeded periodic "
                    "Gaussian velocity field amplitude 1e-2 (seed 3)")
    if name == "euler512":
        return dict(workload="euler_quadrants_512", grid="512x512", equation="Euler gamma=1.4", bc="outflow",
                    scheme="WENO-Z", flux="HLLC", reconstruction="conservative", limiter=False, rk="SSP-RK3", cfl=0.4,
                    ic="four quadrants, (rho,u,v,p) from seed 2")
    if name == "advection128":
        return dict(workload="linear_advection_128", grid="128x128", equation="u_t+u_x+u_y=0", bc="periodic",
                    scheme="WENO-JS", flux="LLF", reconstruction="conservative", limiter=False, rk="SSP-RK3", cfl=0.5,
                    ic="sin(2 pi (x+y))")
    raise SystemExit(f"unknown workload {name}")


def workload_config(name: str, form: str, world: int) -> dict:
    """the `config` object of the JSON line: identical in the GPU arm and the reference arm"""
    return dict(workload_desc(name), form=form, l2="flushed between steps by a 256 MiB write outside the timed events",
                parallelism=f"replicas x{world}")


def workload(name: str, wb, form: int):
    """(U0, config, eq, description dict) of a named workload"""
    desc = workload_desc(name)
    if name in ("column1024", "column1024_exp", "column1024_prim3"):
        sch = 2 if name == "column1024_exp" else 1
        rec = 4 if name == "column1024_prim3" else 1
        U0, prm = cases.liquid_column(1024, 1024, seed=3)
        cfg = wb.make_config(1024, 1024, rk=2, cfl=0.5, scheme=sch, limiter=1, flux=1, recon=rec, precision=form)
        eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
    elif name == "column1024_sg":
        U0, prm = cases.sg_column(1024, 1024, seed=3)
        cfg = wb.make_config(1024, 1024, rk=2, cfl=0.5, scheme=1, limiter=1, flux=1, recon=1, precision=form)
        eq = wb.make_eq(kind=wb.EQ_TWO_PHASE_SG, rho10=prm["rho10"], rho20=prm["rho20"], preb=prm["preb"],
                        gamma1=prm["gamma1"], pinf1=prm["pinf1"], gamma2=prm["gamma2"], pinf2=prm["pinf2"])
    elif name == "euler512":
        U0, _ = cases.euler_quadrants(512, 512, seed=2)
        cfg = wb.make_config(512, 512, bc=wb.BC_OUTFLOW, rk=2, cfl=0.4, scheme=1, flux=1, recon=0, precision=form)
        eq = wb.make_eq(kind=wb.EQ_EULER, gamma=1.4)
    else:  # advection128
        U0 = cases.advection_sine(128, 128)
        cfg = wb.make_config(128, 128, rk=2, cfl=0.5, scheme=0, flux=0, recon=0, precision=form)
        eq = wb.make_eq(kind=wb.EQ_LINEAR_ADV)
    return U0, cfg, eq, desc


# ---- host CPU baseline ------------------------------------------------------------------------
def cpu_baseline(name: str, steps: int, warmup: int, sample_n: int = 1024, single_core: bool = False):
    """The reference (or, where it cannot run the workload, the oracle port) on the host cores.

    The reference runs the workload at its full size (sample_n = 1024 for the columns): as
    many concurrent processes as the host has groups of 4 cores, each the unmodified solver
    with its 4 slab ranks on 4 threads, each timing `steps` SSP-RK3 steps after `warmup`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    ncores = os.cpu_count() or 1
    sch = "2" if name == "column1024_exp" else "1"
    rec = "4" if name == "column1024_prim3" else "1"
    if name in ("column1024", "column1024_exp", "column1024_prim3") and O.reference_available():
        def ref_args(n, d, U, nsteps, nwarm):
            U.tofile(os.path.join(d, "u0.bin"))
            prm = cases.column_params()
            return [O.REF_BIN, "--testcase", "2", "--nx", str(n), "--ny", str(n), "--rk", "2",
                    "--cfl", "0.5", "--scheme", sch, "--limiter", "1", "--flux", "1", "--recon", rec,
                    "--rho10", O._f(prm["rho10"]), "--rho20", O._f(prm["rho20"]), "--sound1", O._f(prm["sound1"]),
                    "--sound2", O._f(prm["sound2"]), "--u0", os.path.join(d, "u0.bin"), "--steps", str(nsteps),
                    "--warmup", str(nwarm), "--time"]

        U0, _ = cases.liquid_column(sample_n, sample_n, seed=3)
        nproc = max(1, ncores // 4)
        with tempfile.TemporaryDirectory() as d:
            args = ref_args(sample_n, d, U0, steps, warmup)
            t0 = time.perf_counter()
            procs = [subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
                     for _ in range(nproc)]
            outs = [pr.communicate(timeout=3600) for pr in procs]
            wall = time.perf_counter() - t0
            secs = []
            for (o, e), pr in zip(outs, procs):
                if pr.returncode != 0:
                    raise RuntimeError(e[-500:])
                secs.append(json.loads(o.strip().splitlines()[-1])["seconds"])
        units = nproc * sample_n * sample_n * 3 * steps
        single = None
        if single_core and shutil.which("taskset"):
            # one reference process pinned to one core (its 4 slab ranks share it), 256^2
            with tempfile.TemporaryDirectory() as d1:
                U1, _ = cases.liquid_column(256, 256, seed=3)
                cp = subprocess.run(["taskset", "-c", "0"] + ref_args(256, d1, U1, 1, 0), capture_output=True,
                                    text=True, timeout=1800)
                if cp.returncode == 0:
                    s1 = json.loads(cp.stdout.strip().splitlines()[-1])["seconds"]
                    single = dict(value=256 * 256 * 3 / s1, cores=1, steps=1, grid="256x256")
        return dict(value=units / max(secs), unit="cell-stage updates/s", cores=4 * nproc, kind="reference",
                    single_core=single, steps=steps, warmup=warmup,
                    sample=f"{nproc} concurrent processes of the unmodified reference (4 slab ranks each, "
                           f"threads over an in-process MPI shim) on the same workload at its full size "
                           f"{sample_n}x{sample_n} (same equation, options and initial data), {steps} timed "
                           f"SSP-RK3 step(s) after {warmup} warm-up step(s) each; {ncores} host cores; "
                           f"wall {wall:.1f} s",
                    seconds=max(secs))
    # the oracle port on all host threads (the reference has no Euler or scalar advection)
    sample_n = min(sample_n, 256)
    if name == "euler512":
        U0, _ = cases.euler_quadrants(sample_n, sample_n, seed=2)
        p = O.Problem(nx=sample_n, ny=sample_n, bc=O.BC_OUTFLOW, eq_kind=O.EQ_EULER, rk=2, cfl=0.4, scheme=1,
                      flux=1, recon=0, threads=ncores)
    elif name == "column1024_sg":
        U0, prm = cases.sg_column(sample_n, sample_n, seed=3)
        p = O.Problem(nx=sample_n, ny=sample_n, eq_kind=O.EQ_TWO_PHASE_SG, rk=2, cfl=0.5, scheme=1, flux=1, recon=1,
                      limiter=1, threads=ncores, **prm)
    elif name == "advection128":
        sample_n = 128
        U0 = cases.advection_sine(128, 128)
        p = O.Problem(nx=128, ny=128, eq_kind=O.EQ_LINEAR_ADV, rk=2, cfl=0.5, scheme=0, flux=0, recon=0,
                      threads=ncores)
    else:
        U0, prm = cases.liquid_column(sample_n, sample_n, seed=3)
        p = O.Problem(nx=sample_n, ny=sample_n, rk=2, cfl=0.5, scheme=int(sch), flux=1, recon=int(rec), limiter=1,
                      threads=ncores, **prm)
    orc = O.Oracle()
    dt = orc.compute_dt(p, U0)
    V = U0
    for _ in range(warmup):
        V = orc.step(p, V, dt)
    t0 = time.perf_counter()
    for _ in range(steps):
        V = orc.step(p, V, dt)
    secs = time.perf_counter() - t0
    return dict(value=sample_n * sample_n * 3 * steps / secs, unit="cell-stage updates/s", cores=ncores, kind="port",
                sample=f"the C restatement (oracle/wenofv_oracle.c, OpenMP over {ncores} threads), {steps} SSP-RK3 "
                       f"steps at {sample_n}x{sample_n} of the same workload",
                seconds=secs)


# ---- ranks ------------------------------------------------------------------------------------------
def max_over_ranks(x: float, dist, local: int = 0) -> float:
    """the largest value over all ranks (times are taken on each rank's own device, and the
    job's duration is the slowest rank's); the reduction runs on the rank's GPU under NCCL
    and on the CPU under gloo"""
    if dist is None:
        return float(x)
    import torch

    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, units_per_rank: float, seconds: float) -> float:
    """whole-job throughput of independent replicas: all ranks' units over the slowest time"""
    return world * units_per_rank / seconds


# ---- clocks ------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path:
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in rows if num(r[3]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return dict(sm_mhz=float(np.median(sm)) if sm else None, sm_max_mhz=max(mx) if mx else None,
                    reasons=reasons, samples=len(rows), power_w_max=max(pw) if pw else None)


def read_traffic(workload_name: str):
    """DRAM bytes per stage-kernel launch from the committed ncu summary, when there is one"""
    path = os.path.join(ROOT, "profiles", f"stage_kernel_{workload_name}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---- our arm --------------------------------------------------------------------------------------
def run_ours(args, rank, world, dist):
    import importlib.util

    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    spec = importlib.util.spec_from_file_location("wenofv_b200", os.path.join(ROOT, "two-phase-3equation-2d-pal-column_b200", "__init__.py"))
    wb = importlib.util.module_from_spec(spec)
    sys.modules["wenofv_b200"] = wb
    spec.loader.exec_module(wb)

    form = {"fp64": wb.FP64, "fp64_strict": wb.FP64_STRICT, "fp32_bulk": wb.FP32_BULK}[args.form]
    U0, cfg, eq, desc = workload(args.workload, wb, form)
    cfg.device = local
    s = wb.Solver(cfg, eq)
    s.upload(U0)
    ncells = cfg.nx * cfg.ny
    nstages = 3
    peak = wb.fma_peak_tflops(wb.FP32_BULK if form == wb.FP32_BULK else wb.FP64, local)
    dt = s.compute_dt()

    stream = torch.cuda.ExternalStream(s.stream())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        s.step(dt)
    s.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    # device-resident timing
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()  # L2 flush, outside the timed events
                evs[k][0].record(stream)
                s.step(dt)
                evs[k][1].record(stream)
        s.synchronize()
        torch.cuda.synchronize()
    barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = float(np.sum(step_ms))
    total_ms = max_over_ranks(total_ms, dist, local)
    value = world * ncells * nstages * args.steps / (total_ms * 1e-3)
    flags, _ = s.status()

    U_dev_end = s.download()
    # FP32-bulk beside FP64: the same steps from the same state, device-timed the same way,
    # and the error of its result against the FP64 one
    fp32 = None
    if form == wb.FP64 and args.workload not in ("advection128", "column1024_exp", "column1024_prim3", "column1024_sg") \
            and not args.no_fp32:
        fp32 = compare_fp32(args, wb, cfg, eq, U0, dt, U_dev_end, ncells, nstages, flush, barrier, dist, world, local)

    # end to end through the public API with host arrays (pinned host memory)
    U_host = torch.empty(U_dev_end.shape, dtype=torch.float64, pin_memory=True).numpy()
    U_host[...] = U_dev_end
    nbytes = U_host.nbytes
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        s.upload(U_host)
        s.step(dt)
        s.download_into(U_host)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, local)
    e2e = dict(value=world * ncells * nstages * args.steps / e2e_s, unit="cell-stage updates/s",
               h2d_bytes_per_step=nbytes, d2h_bytes_per_step=nbytes)

    launch_ms = total_ms / (args.steps * nstages)  # a step is the stage kernel 3x (+ a 100-byte H2D)
    fpcs = flops_per_cell_stage(args.workload)
    achieved_tf = fpcs * ncells / (launch_ms * 1e-3) / 1e12
    hbm_gbs = BYTES_PER_CELL_STAGE[args.workload] * ncells / (launch_ms * 1e-3) / 1e9
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    measured = json.load(open(mp)) if os.path.exists(mp) else {}
    hbm_peak = measured.get("hbm_gbs", 6650.0)
    roofline = dict(bound="fp32" if form == wb.FP32_BULK else "fp64", achieved=achieved_tf, peak=peak,
                    unit="TFLOP/s", frac=achieved_tf / peak, traffic=read_traffic(args.workload),
                    traffic_source=f"not measured live: DRAM bytes read + written per stage launch from one ncu "
                                   f"capture of this command, committed in profiles/stage_kernel_{args.workload}.md",
                    kernel="wenofv::stage_kernel", launch_ms=launch_ms, flops_per_launch=fpcs * ncells,
                    flops_per_cell_stage=fpcs,
                    peak_source=f"FMA throughput of the {'FP32' if form == wb.FP32_BULK else 'FP64'} CUDA-core pipe "
                                f"measured in this run (wenofv_probe_fma_peak)",
                    hbm_view=dict(achieved=hbm_gbs, peak=hbm_peak, unit="GB/s", frac=hbm_gbs / hbm_peak,
                                  bytes_per_cell_stage=BYTES_PER_CELL_STAGE[args.workload],
                                  peak_source="MEASURED_PEAKS.json hbm_gbs (of measured)" if measured else "fallback"))
    out = dict(metric="cell-stage updates/s", value=value, unit="cell-stage updates/s", n_gpus=world,
               steps=args.steps, warmup=args.warmup, ms_per_step=total_ms / args.steps, higher_is_better=True,
               scaling="weak", vs_baseline=None,
               dtype={"fp64": "f64", "fp64_strict": "f64", "fp32_bulk": "f32+f64"}[args.form], data="synthetic",
               config=workload_config(args.workload, args.form, world),
               roofline=roofline, e2e=e2e, gpu_launches=args.steps * nstages, status_flags=flags)
    if fp32:
        fp32["roofline"] = dict(bound="fp64+fp32", achieved=fpcs * ncells / (fp32["launch_ms"] * 1e-3) / 1e12,
                                unit="TFLOP/s", note="counted flops of the FP64 algorithm per launch / launch time; "
                                "the FP32-bulk form mixes both pipes, so no single peak bounds it")
        fp32["speedup_vs_fp64_per_launch"] = launch_ms / fp32["launch_ms"]
        out["fp32_bulk"] = fp32
    out["clocks"] = clk.summary()
    if not args.no_mix and args.workload == "column1024":
        out.update(mixed_workloads(wb, local, dist, world))
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.workload, steps=args.cpu_steps, warmup=0)
    s.close()
    return out


def run_steps(wb, cfg, eq, U0, dt, nsteps, precision):
    """the state after nsteps manual RK steps of fixed dt in the given form"""
    c = wb.Config.from_buffer_copy(cfg)
    c.precision = precision
    with wb.Solver(c, eq) as s:
        s.upload(U0)
        for _ in range(nsteps):
            s.step(dt)
        return s.download()


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def oracle_check(wb, cfg, eq, U0, dt, nsteps, threads):
    """FP64_STRICT against the CPU oracle over the first nsteps steps of the same run: the
    strict form is the oracle's arithmetic bit for bit, so it stands in for the oracle over
    the whole run (the oracle at full size takes seconds per step)"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    strict = run_steps(wb, cfg, eq, U0, dt, nsteps, wb.FP64_STRICT)
    p = O.Problem(nx=cfg.nx, ny=cfg.ny, xl=cfg.xl, xr=cfg.xr, yl=cfg.yl, yr=cfg.yr, bc=cfg.bc, rk=cfg.rk_method,
                  cfl=cfg.cfl, scheme=cfg.scheme, limiter=cfg.pp_limiter, flux=cfg.riemann_flux,
                  recon=cfg.reconstruction, ref_slabs=cfg.ref_slabs, threads=threads, eq_kind=eq.eq_kind,
                  rho10=eq.rho10, rho20=eq.rho20, sound1=eq.sound1, sound2=eq.sound2, gamma=eq.gamma)
    orc = O.Oracle()
    V = U0
    t0 = time.perf_counter()
    for _ in range(nsteps):
        V = orc.step(p, V, dt)
    return dict(steps=nsteps, bit_identical=bool(np.array_equal(strict, V)), oracle_threads=threads,
                oracle_seconds=time.perf_counter() - t0)


def compare_fp32(args, wb, cfg, eq, U0, dt, U64, ncells, nstages, flush, barrier, dist, world, local):
    """FP32-bulk beside FP64: the same steps from the same state and dt, device-timed the same
    way; its error, and the FP64 form's, against the FP64 oracle's arithmetic (FP64_STRICT on the
    device, checked bit for bit against the CPU oracle over a prefix of the same run)"""
    import torch

    cfg32 = wb.Config.from_buffer_copy(cfg)
    cfg32.precision = wb.FP32_BULK
    s = wb.Solver(cfg32, eq)
    s.upload(U0)
    for _ in range(args.warmup):
        s.step(dt)
    s.synchronize()
    stream = torch.cuda.ExternalStream(s.stream())
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            s.step(dt)
            evs[k][1].record(stream)
    s.synchronize()
    torch.cuda.synchronize()
    barrier()
    total_ms = float(np.sum([a.elapsed_time(b) for a, b in evs]))
    total_ms = max_over_ranks(total_ms, dist, local)
    U32 = s.download()
    flags, _ = s.status()
    s.close()
    nsteps = args.warmup + args.steps
    Ustrict = run_steps(wb, cfg, eq, U0, dt, nsteps, wb.FP64_STRICT)
    per = [float(np.abs(U32[v] - Ustrict[v]).sum() / max(np.abs(Ustrict[v]).sum(), 1e-300)) for v in range(U64.shape[0])]
    out = dict(value=world * ncells * nstages * args.steps / (total_ms * 1e-3), unit="cell-stage updates/s",
               ms_per_step=total_ms / args.steps, launch_ms=total_ms / (args.steps * nstages),
               gpu_launches=args.steps * nstages,
               speedup_vs_fp64_per_launch=None,
               rel_l1_vs_oracle=rel_l1(U32, Ustrict), rel_l1_vs_oracle_per_var=per,
               fp64_rel_l1_vs_oracle=rel_l1(U64, Ustrict), rel_l1_vs_fp64=rel_l1(U32, U64),
               min_partial_density=[float(U32[0].min()), float(U32[1].min())] if U32.shape[0] == 4 else None,
               error_note=f"pooled relative L1 of the final state after the same {nsteps} steps from the same "
                          f"initial data and dt, against the FP64 oracle's arithmetic (FP64_STRICT on the device; "
                          f"see oracle_check) and, for the spread of the scheme's own roundoff, the FP64 form's",
               status_flags=flags)
    if not args.no_oracle_check:
        out["oracle_check"] = oracle_check(wb, cfg, eq, U0, dt, 2, os.cpu_count() or 1)
    return out


def mixed_workloads(wb, local, dist, world):
    """bounded versions of the batched ensemble and the serving stream for the default line:
    solves/s, latency percentiles, FP32-bulk against FP64, and both forms' errors against the
    oracle's arithmetic"""
    ens = cases.ensemble(64, seed=4)
    res, _, cells = batch_measure(wb, ens, 50, 3, local, dist, world)
    batch = dict(workload="batched_ensemble_64", instances=64, cells=cells, steps_per_solve=50,
                 grids="U{64,96,128,192,256}^2 and {256x64, 512x128} (seed 4)",
                 solves_per_s=res["fp64"]["solves_per_s"], fp64=res["fp64"], fp32_bulk=res["fp32_bulk"],
                 fp64_strict=res["fp64_strict"], errors=res["errors"],
                 oracle_check=batch_oracle_check(wb, ens, 10, os.cpu_count() or 1))
    reqs = serve_requests(wb, 16, 7, 50, 400, nx_max=1024, ny_max=256)
    sres = serve_measure(wb, reqs, 4.0, 8 << 30, 7, local, dist, world)
    serve = dict(workload="serving_stream_16", requests=16, arrival="Poisson, mean 4 req/s (seed 7)",
                 grids="nx log-uniform 64..1024, ny log-uniform 64..256", steps="uniform 50..400 per request",
                 mix="Euler quadrants / two-phase columns 50/50", hbm_budget_gb=8,
                 solves_per_s=sres["fp64"]["solves_per_s"], p50_latency_s=sres["fp64"]["p50_latency_s"],
                 p99_latency_s=sres["fp64"]["p99_latency_s"], fp64=sres["fp64"], fp32_bulk=sres["fp32_bulk"],
                 errors=sres["errors"])
    return dict(batch=batch, serve=serve)


def _load_package():
    import importlib.util

    spec = importlib.util.spec_from_file_location("wenofv_b200", os.path.join(ROOT, "two-phase-3equation-2d-pal-column_b200", "__init__.py"))
    wb = importlib.util.module_from_spec(spec)
    sys.modules["wenofv_b200"] = wb
    spec.loader.exec_module(wb)
    return wb


def _pctl(x, q):
    return float(np.percentile(np.asarray(x, dtype=np.float64), q)) if len(x) else None


# ---- config 4: batched ensemble ------------------------------------------------------------------
def per_instance_errors(finals, names=("fp64", "fp32_bulk"), ref="fp64_strict"):
    """pooled relative L1 of each instance's final state against the FP64 oracle's arithmetic
    (the strict form), per form: the FP64 form's spread is the scheme's own sensitivity to
    rounding, against which FP32-bulk's error is read"""
    out = {}
    for name in names:
        e = [rel_l1(a, b) for a, b in zip(finals[name], finals[ref]) if a is not None and b is not None]
        out[name] = e
    return out


def summarize_errors(err, bar=1e-5):
    e32, e64 = np.asarray(err["fp32_bulk"]), np.asarray(err["fp64"])
    # an instance "within the scheme's spread": FP32's error at most 10x the FP64 form's
    excused = [(a > bar and a <= 10 * b) for a, b in zip(e32, e64)]
    unexplained = [dict(k=k, fp32=float(a), fp64=float(b)) for k, (a, b, x) in enumerate(zip(e32, e64, excused))
                   if a > bar and not x]
    unexplained.sort(key=lambda r: -r["fp32"])
    return dict(fp32_vs_oracle=dict(median=_pctl(e32, 50), p90=_pctl(e32, 90), max=float(e32.max()) if len(e32) else None,
                                    within_bar=int(np.sum(e32 <= bar)), n=int(len(e32))),
                fp64_vs_oracle=dict(median=_pctl(e64, 50), p90=_pctl(e64, 90), max=float(e64.max()) if len(e64) else None),
                over_bar_explained_by_fp64_spread=int(np.sum(excused)),
                over_bar_unexplained=len(unexplained), unexplained_instances=unexplained[:16],
                bar=bar, note="pooled relative L1 per instance against FP64_STRICT (the oracle's arithmetic, "
                              "bit for bit); an instance over the bar whose FP64-form spread is within 10x of its "
                              "FP32-bulk error is the scheme's own roundoff sensitivity, not FP32's")


def batch_measure(wb, ens, steps, warmup, local, dist, world, autotune=True):
    """one persistent launch per RK stage for all instances, captured step pairs; FP64, FP32-bulk
    and FP64_STRICT on the same inputs (the strict run is the oracle's arithmetic)"""
    import torch

    cells = sum(prm["nx"] * prm["ny"] for _, prm in ens)
    res, finals = {}, {}
    for name, form in (("fp64", wb.FP64), ("fp32_bulk", wb.FP32_BULK), ("fp64_strict", wb.FP64_STRICT)):
        cfgs, eqs = [], []
        for U0, prm in ens:
            c = wb.make_config(prm["nx"], prm["ny"], rk=2, cfl=0.5, scheme=prm["scheme"], flux=1, recon=1, limiter=1,
                               precision=form)
            c.device = local
            cfgs.append(c)
            eqs.append(wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"]))
        b = wb.Batch(cfgs, eqs)
        for k, (U0, _) in enumerate(ens):
            b.upload(k, U0)
        tiling = None
        if autotune and name != "fp64_strict":
            rows, ctas, tune_ms = b.autotune()
            tiling = dict(rows_per_item=rows or "automatic", ctas_per_sm=ctas, threads_per_cta=b.tiling()[2] or "per instance",
                          autotune_best_stage_ms=tune_ms)
        if name != "fp64_strict":
            b.advance(1e9, max_steps=warmup)
            for k, (U0, _) in enumerate(ens):
                b.upload(k, U0)
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        try:
            ns = b.advance(1e9, max_steps=steps)
            failed = []
        except wb.WenofvError:
            ns, failed = None, ["status flags raised"]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, local)
        finals[name] = [b.download(k) for k in range(len(ens))]
        res[name] = dict(value=world * cells * 3 * steps / (ms * 1e-3), unit="cell-stage updates/s",
                         solves_per_s=world * len(ens) / (ms * 1e-3), seconds=ms * 1e-3, tiling=tiling,
                         all_steps_done=bool(ns is not None and int(ns.min()) == int(ns.max()) == steps),
                         failures=failed)
        b.close()
    res["fp64_strict"].pop("tiling")
    err = per_instance_errors(finals)
    res["fp32_bulk"]["speedup_vs_fp64"] = res["fp32_bulk"]["value"] / res["fp64"]["value"]
    res["errors"] = summarize_errors(err)
    return res, err, cells


def batch_oracle_check(wb, ens, steps, threads):
    """FP64_STRICT against the CPU oracle for the first two instances of the batch, solved alone"""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    ok = True
    for U0, prm in ens[:2]:
        p = O.Problem(nx=prm["nx"], ny=prm["ny"], rk=2, cfl=0.5, scheme=prm["scheme"], flux=1, recon=1, limiter=1,
                      threads=threads, rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"],
                      sound2=prm["sound2"])
        V, *_ = O.Oracle().advance(p, U0, t_end=1e9, max_steps=steps)
        cfg = wb.make_config(prm["nx"], prm["ny"], rk=2, cfl=0.5, scheme=prm["scheme"], flux=1, recon=1, limiter=1,
                             precision=wb.FP64_STRICT)
        eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
        with wb.Solver(cfg, eq) as s:
            s.upload(U0)
            s.advance(1e9, max_steps=steps)
            ok = ok and bool(np.array_equal(s.download(), V))
    return dict(instances=2, steps=steps, bit_identical=ok)


def run_batch(args, rank, world, dist):
    """config 4: 256 uneven two-phase instances"""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    wb = _load_package()
    ens = cases.ensemble(args.instances, seed=4)
    res, err, cells = batch_measure(wb, ens, args.steps, args.warmup, local, dist, world)
    res["oracle_check"] = batch_oracle_check(wb, ens, min(args.steps, 20), os.cpu_count() or 1)
    rows = [dict(k=k, nx=prm["nx"], ny=prm["ny"], ratio=round(prm["ratio"], 1), eps=prm["eps"], scheme=prm["scheme"],
                 fp32=err["fp32_bulk"][k], fp64=err["fp64"][k]) for k, (_, prm) in enumerate(ens)]
    for u in res["errors"].get("unexplained_instances", []):
        u.update({key: rows[u["k"]][key] for key in ("nx", "ny", "ratio", "eps", "scheme")})
    rows.sort(key=lambda r: -r["fp32"])
    out = dict(metric="cell-stage updates/s", value=res["fp64"]["value"], unit="cell-stage updates/s", n_gpus=world,
               steps=args.steps, warmup=args.warmup, ms_per_step=res["fp64"]["seconds"] * 1e3 / args.steps,
               higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
               config=dict(workload=f"batched_ensemble_{len(ens)}", instances=len(ens), cells=cells,
                           grids="U{64,96,128,192,256}^2 and {256x64, 512x128} (seed 4)",
                           ic="liquid columns, radius U[0.1,0.3], density ratio U[10,1000], eps in {1e-8,1e-6}",
                           scheme="WENO-JS/WENO-Z mixed", flux="HLLC", reconstruction="characteristic",
                           limiter=True, rk="SSP-RK3", steps_per_solve=args.steps,
                           l2=f"working set {cells * 32 * 3 / 1e6:.0f} MB", parallelism=f"replicas x{world}"),
               solves_per_s=res["fp64"]["solves_per_s"], fp64=res["fp64"], fp32_bulk=res["fp32_bulk"],
               fp64_strict=res["fp64_strict"], errors=res["errors"], oracle_check=res["oracle_check"],
               worst_fp32_instances=rows[:10], gpu_launches=2 * 3 * args.steps)
    return out


# ---- config 5: serving stream --------------------------------------------------------------------
def serve_requests(wb, n, seed, min_steps, max_steps, nx_max=2048, ny_max=512):
    """n requests: Euler quadrants (outflow, conservative) or two-phase columns (periodic,
    characteristic, limiter) 50/50, nx log-uniform 64..nx_max, ny 64..ny_max, steps uniform"""
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        nx = int(round(2 ** rng.uniform(6, np.log2(nx_max)) / 8)) * 8
        ny = int(round(2 ** rng.uniform(6, np.log2(ny_max)) / 8)) * 8
        steps = int(rng.integers(min_steps, max_steps + 1))
        if rng.uniform() < 0.5:
            U0, _ = cases.euler_quadrants(nx, ny, seed=100 + k)
            mk = lambda f, nx=nx, ny=ny: wb.make_config(nx, ny, bc=wb.BC_OUTFLOW, rk=2, cfl=0.4, scheme=1, flux=1,
                                                         recon=0, precision=f)
            eq = wb.make_eq(kind=wb.EQ_EULER, gamma=1.4)
            kind = "euler"
        else:
            U0, prm = cases.point_column(nx, ny, seed=100 + k)
            mk = lambda f, nx=nx, ny=ny: wb.make_config(nx, ny, rk=2, cfl=0.5, scheme=1, flux=1, recon=1, limiter=1,
                                                         precision=f)
            eq = wb.make_eq(rho10=prm["rho10"], rho20=prm["rho20"], sound1=prm["sound1"], sound2=prm["sound2"])
            kind = "two_phase"
        reqs.append((mk, eq, U0, steps, nx * ny, kind))
    return reqs


def serve_stream(wb, reqs, arrivals, form, budget_bytes, local, dist, world):
    """submits the requests at their arrival times (server clock) and polls until all are done"""
    srv = wb.Server(local, hbm_budget_bytes=budget_bytes, max_slots=256)
    if dist is not None:
        dist.barrier()
    n = len(reqs)
    t0 = srv.clock()
    ids, done, failed = [], {}, set()
    k = 0
    while len(done) < n:
        now = srv.clock() - t0
        while k < n and arrivals[k] <= now:
            mk, eq, U0, steps, _, _ = reqs[k]
            cfg = mk(form)
            cfg.device = local
            ids.append(srv.submit(cfg, eq, U0, 1e9, max_steps=steps))
            k += 1
        for j, rid in enumerate(ids):
            if j in done:
                continue
            try:
                got = srv.poll(rid)
            except wb.WenofvError:  # a numerically failed solve is a result too
                got = (None, None)
                failed.add(j)
            if got is not None:
                done[j] = got
        time.sleep(0.0005)
    srv.close()
    ok = [j for j in range(n) if j not in failed]
    lat = [done[j][1].t_done - done[j][1].t_submit for j in ok]
    qwait = [done[j][1].t_admit - done[j][1].t_submit for j in ok]
    span = max(done[j][1].t_done for j in ok) - min(done[j][1].t_submit for j in ok)
    span = max_over_ranks(span, dist, local)
    assert all(done[j][1].steps == reqs[j][3] for j in ok)
    work_ok = sum(reqs[j][3] * reqs[j][4] * 3 for j in ok)
    stats = dict(value=world * work_ok / span, unit="cell-stage updates/s", solves_per_s=world * len(ok) / span,
                 failed_requests=sorted(failed), p50_latency_s=_pctl(lat, 50), p99_latency_s=_pctl(lat, 99),
                 p50_queue_s=_pctl(qwait, 50), makespan_s=span)
    return stats, [done[j][0] for j in range(n)]


def serve_alone_strict(wb, reqs, local):
    """each request solved alone in FP64_STRICT (the oracle's arithmetic)"""
    out = []
    for mk, eq, U0, steps, _, _ in reqs:
        cfg = mk(wb.FP64_STRICT)
        cfg.device = local
        with wb.Solver(cfg, eq) as s:
            s.upload(U0)
            try:
                s.advance(1e9, max_steps=steps)
                out.append(s.download())
            except wb.WenofvError:
                out.append(None)
    return out


def serve_measure(wb, reqs, rate, budget_bytes, seed, local, dist, world, forms=("fp64", "fp32_bulk")):
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    res, finals = {}, {}
    for name in forms:
        form = {"fp64": wb.FP64, "fp32_bulk": wb.FP32_BULK}[name]
        res[name], finals[name] = serve_stream(wb, reqs, arrivals, form, budget_bytes, local, dist, world)
    if "fp32_bulk" in res:
        finals["fp64_strict"] = serve_alone_strict(wb, reqs, local)
        # errors per request kind (results of failed requests are left out)
        by = {"euler": {"fp64": [], "fp32_bulk": [], "req": []}, "two_phase": {"fp64": [], "fp32_bulk": [], "req": []}}
        for j, r in enumerate(reqs):
            a, b, c = finals["fp32_bulk"][j], finals["fp64"][j], finals["fp64_strict"][j]
            if a is None or b is None or c is None:
                continue
            by[r[5]]["fp32_bulk"].append(rel_l1(a, c))
            by[r[5]]["fp64"].append(rel_l1(b, c))
            by[r[5]]["req"].append(j)
        res["errors"] = {}
        for kind, v in by.items():
            if not v["fp64"]:
                continue
            summ = summarize_errors(v)
            for u in summ["unexplained_instances"]:  # k: the request's index in the stream
                j = v["req"][u["k"]]
                nx, ny = reqs[j][2].shape[2], reqs[j][2].shape[1]
                u.update(k=j, nx=int(nx), ny=int(ny), steps=int(reqs[j][3]))
            res["errors"][kind] = summ
        res["fp32_bulk"]["speedup_vs_fp64"] = res["fp32_bulk"]["value"] / res["fp64"]["value"]
    return res


def run_serve(args, rank, world, dist):
    """config 5: Poisson arrivals of mixed Euler / two-phase solves into the continuous-batching
    server at the configured rate, plus a load sweep at rates the GPU sustains"""
    import torch

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    wb = _load_package()
    reqs = serve_requests(wb, args.requests, 5 + rank, args.min_steps, args.max_steps)
    budget = args.hbm_budget_gb << 30
    res = serve_measure(wb, reqs, args.rate, budget, 5 + rank, local, dist, world)
    sweep = []
    for rate in [float(x) for x in args.rates.split(",") if x]:
        r = serve_measure(wb, reqs, rate, budget, 6 + rank, local, dist, world, forms=("fp64",))
        sweep.append(dict(rate=rate, **{k: r["fp64"][k] for k in ("solves_per_s", "p50_latency_s", "p99_latency_s",
                                                                   "p50_queue_s", "value")}))
    out = dict(metric="cell-stage updates/s", value=res["fp64"]["value"], unit="cell-stage updates/s", n_gpus=world,
               steps=args.requests, warmup=0, ms_per_step=None, higher_is_better=True, scaling="weak", vs_baseline=None,
               dtype="f64", data="synthetic",
               config=dict(workload=f"serving_stream_{args.requests}", requests=args.requests,
                           arrival=f"Poisson, mean {args.rate} req/s (seed {5 + rank})",
                           grids="nx log-uniform 64..2048, ny log-uniform 64..512 (multiples of 8)",
                           steps=f"uniform {args.min_steps}..{args.max_steps} per request",
                           mix="Euler quadrants (outflow, conservative WENO-Z/HLLC) and two-phase columns "
                               "(periodic, characteristic WENO-Z/HLLC/limiter), 50/50",
                           hbm_budget_gb=args.hbm_budget_gb, parallelism=f"replicas x{world}",
                           latency="server clock, submission to completion"),
               solves_per_s=res["fp64"]["solves_per_s"], p50_latency_s=res["fp64"]["p50_latency_s"],
               p99_latency_s=res["fp64"]["p99_latency_s"], fp64=res["fp64"], fp32_bulk=res["fp32_bulk"],
               errors=res["errors"], load_sweep=sweep)
    return out


def run_reference_arm(args):
    """the reference's CPU implementation on the same workload and config as the GPU arm.  At
    1024^2 one reference step takes tens of seconds, so the arm times a bounded prefix: at most
    REF_MAX_STEPS steps after at most one warm-up step (the line's steps and warmup say what ran)."""
    REF_MAX_STEPS = 2
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    warmup = min(args.warmup, 1)
    cb = cpu_baseline(args.workload, steps=steps, warmup=warmup, single_core=True)
    return dict(metric="cell-stage updates/s", value=cb["value"], unit="cell-stage updates/s", n_gpus=args.gpus,
                steps=steps, warmup=warmup, ms_per_step=1e3 * cb["seconds"] / steps,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64", data="synthetic",
                impl="reference", config=workload_config(args.workload, args.form, args.gpus),
                requested=dict(steps=args.steps, warmup=args.warmup,
                               note=f"bounded prefix: {steps} timed step(s) after {warmup} warm-up step(s) of the "
                                    f"full-size workload on every reference process"),
                cpu_baseline=dict(value=cb["value"], unit=cb["unit"], cores=cb["cores"], kind=cb["kind"],
                                  sample=cb["sample"], single_core=cb.get("single_core")),
                e2e=dict(value=cb["value"], unit=cb["unit"], h2d_bytes_per_step=0, d2h_bytes_per_step=0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="column1024", choices=sorted(FLOP_KEYS) + ["batch256", "serve"])
    ap.add_argument("--instances", type=int, default=256, help="batch256: instances")
    ap.add_argument("--requests", type=int, default=32, help="serve: requests")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: mean arrival rate, requests/s")
    ap.add_argument("--min-steps", type=int, default=50, help="serve: fewest steps of a request")
    ap.add_argument("--max-steps", type=int, default=2000, help="serve: most steps of a request")
    ap.add_argument("--hbm-budget-gb", type=int, default=150, help="serve: HBM budget of the server")
    ap.add_argument("--rates", default="1,2,4", help="serve: arrival rates (req/s) of the load sweep")
    ap.add_argument("--no-mix", action="store_true", help="default line: skip the batch and serve objects")
    ap.add_argument("--form", default="fp64", choices=["fp64", "fp64_strict", "fp32_bulk"])
    ap.add_argument("--cpu-steps", type=int, default=1, help="timed reference steps of the cpu_baseline leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-bulk comparison of the FP64 form")
    ap.add_argument("--no-oracle-check", action="store_true", help="skip the CPU oracle check of the strict form")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference_arm(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if args.workload == "batch256":
        out = run_batch(args, rank, world, dist)
    elif args.workload == "serve":
        out = run_serve(args, rank, world, dist)
    else:
        out = run_ours(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
