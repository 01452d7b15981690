"""Generates the golden fixtures of tests/golden/ from the compiled reference solver.

Run from the repository root after `make -C oracle ref` (needs the reference checkout
only at build time):  python tests/golden/make_golden.py

Each case runs the unmodified reference (oracle/_ref/wenofv_ref, src/WENOFV.cpp with its
4-rank x-slab decomposition) on a small periodic two-phase grid and stores, as float64:
U0 (initial averages, the reference's own or injected), rhs (one assembleRHS of U0),
U (after `steps` RK steps with the CFL time step, or after the run() loop to t_end) and
dts (the time steps taken).  These fixtures pin the oracle and the GPU path in tests that
run where the reference is absent.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import Problem, run_reference  # noqa: E402
import cases  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, testcase, nx, ny, scheme, flux, recon, limiter, rk, steps, t_end, injected liquid column)
CASES = [
    ("smooth_js_cons_llf_rk3", 0, 32, 16, 0, 0, 0, 0, 2, 5, 0.0, False),
    ("smooth_z_char_llf_rk3_settings", 0, 32, 16, 1, 0, 1, 0, 2, 5, 0.0, False),
    ("smooth_z_char_hllc_rk2", 0, 24, 20, 1, 1, 1, 0, 1, 4, 0.0, False),
    ("smooth_js_cons_hllc_rk1_tend", 0, 16, 16, 0, 1, 0, 0, 0, 0, 0.01, False),
    ("sharp_z_char_hllc_lim_rk3", 2, 40, 24, 1, 1, 1, 1, 2, 8, 0.0, False),
    ("sharp_js_cons_llf_lim_rk3", 2, 40, 24, 0, 0, 0, 1, 2, 8, 0.0, False),
    ("column_z_char_hllc_lim_rk3", 2, 48, 32, 1, 1, 1, 1, 2, 6, 0.0, True),
    ("column_js_cons_llf_lim_rk3", 2, 48, 32, 0, 0, 0, 1, 2, 6, 0.0, True),
    ("sharp_z_prim_hllc_lim_rk3", 2, 40, 24, 1, 1, 2, 1, 2, 8, 0.0, False),
    ("smooth_js_prim2_llf_rk3", 0, 32, 16, 0, 0, 3, 0, 2, 5, 0.0, False),
    ("column_z_prim2_hllc_lim_rk3", 2, 48, 32, 1, 1, 3, 1, 2, 6, 0.0, True),
    ("smooth_exp_cons_llf_rk3", 0, 32, 16, 2, 0, 0, 0, 2, 5, 0.0, False),
    ("sharp_exp_char_hllc_lim_rk3", 2, 40, 24, 2, 1, 1, 1, 2, 8, 0.0, False),
    ("column_exp_char_hllc_lim_rk3", 2, 48, 32, 2, 1, 1, 1, 2, 6, 0.0, True),
    ("column_exp_prim_hllc_lim_rk3", 2, 48, 32, 2, 1, 2, 1, 2, 6, 0.0, True),
    ("smooth_prim3_llf_rk3", 0, 32, 16, 1, 0, 4, 0, 2, 5, 0.0, False),
    ("sharp_prim3_hllc_lim_rk3", 2, 40, 24, 1, 1, 4, 1, 2, 8, 0.0, False),
    ("column_prim3_hllc_lim_rk3", 2, 48, 32, 0, 1, 4, 1, 2, 6, 0.0, True),
]
# cases with the gravity source of assembleSourceTerm: name -> (the test case it sees, g_g0)
GRAVITY = {"column_gravity_z_char_hllc_lim_rk3": (6, 9.81)}
CASES.append(("column_gravity_z_char_hllc_lim_rk3", 2, 48, 32, 1, 1, 1, 1, 2, 6, 0.0, True))

PARAMS = {0: dict(rho10=1.2, rho20=1.0, sound1=1.0, sound2=1.0),
          2: dict(rho10=1000.0, rho20=1.0, sound1=70.0, sound2=70.0)}


def main(only=()):
    """Regenerates every case, or only the named ones (the index keeps the others)."""
    index = {}
    if only:
        with open(os.path.join(OUT, "index.json")) as f:
            index = json.load(f)
    for (name, tc, nx, ny, scheme, flux, recon, lim, rk, steps, t_end, column) in CASES:
        if only and name not in only:
            continue
        prm = dict(PARAMS[tc])
        U0 = None
        if column:
            U0, cp = cases.liquid_column(nx, ny, seed=11)
            prm = dict(rho10=cp["rho10"], rho20=cp["rho20"], sound1=cp["sound1"], sound2=cp["sound2"])
        source_case, g = GRAVITY.get(name, (-1, 0.0))
        p = Problem(nx=nx, ny=ny, rk=rk, cfl=0.5, scheme=scheme, flux=flux, recon=recon,
                    limiter=lim, ref_slabs=4, gravity=g, **prm)
        r = run_reference(p, testcase=tc, U0=U0, steps=steps, t_end=t_end, want_rhs=True, source_case=source_case)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), U0=r.U0, rhs=r.rhs, U=r.U, dts=r.dts)
        index[name] = dict(testcase=tc, nx=nx, ny=ny, scheme=scheme, flux=flux, recon=recon,
                           limiter=lim, rk=rk, steps=steps, t_end=t_end, cfl=0.5, ref_slabs=4, gravity=g,
                           nsteps_taken=int(len(r.dts)), **prm)
        print(name, "steps", len(r.dts), "|U|max", float(np.abs(r.U).max()))
    with open(os.path.join(OUT, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
