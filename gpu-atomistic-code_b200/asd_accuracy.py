"""Error of the FP32 and fused-FP64 forms against the FP64 plain form as the run lengthens.

All three forms start from the same spins and, at finite temperature, draw the same Philox
noise (the FP32 form evaluates it in single precision).  At each checkpoint the script reports
max |dS| over all spin components and, for the long-range workloads, max |dH| of the total
field relative to its largest component.  Deterministic (T = 0) runs from random spins relax
chaotically for the first ~1/(lambda gamma H_exch) of simulated time, so small per-step rounding
differences grow there; the growth curve, not one number, describes a form's accuracy.

    python asd_accuracy.py --workload northstar --checkpoints 100,1000,10000
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import asd_b200 as A
import asd_lattice as LT


def workload(name):
    if name == "northstar":
        s = LT.sc_ferromagnet((128, 128, 64), pbc=(0, 0, 0), dipole=True)
        return [s], dict(integrator=A.HEUN, dt=1e-16, update=1)
    if name == "sc128_fft":
        return [LT.sc_fft(128)], dict(integrator=A.HEUN, dt=1e-16)
    if name == "bct2_64":
        return [LT.bct2_antiferromagnet(64, layout="csr", T=0.0)], dict(integrator=A.HEUN, dt=1e-16)
    if name == "sc16":
        return [LT.sc_ferromagnet(16)], dict(integrator=A.HEUN, dt=1e-16)
    if name == "film_rk4":
        return [LT.film_dia(256, 256, 4, dipole=True)], dict(integrator=A.RK4, dt=5e-16, update=1)
    raise ValueError(f"unknown workload {name}")


def run(name, checkpoints, seed=0):
    systems, kw = workload(name)
    n = sum(s.nspins for s in systems)
    S0 = LT.random_spins(n, seed)
    lr = systems[0].lr != A.LR_NONE
    forms = {"fp32": A.RunParams(precision=A.FP32, flags=A.FLAG_COMPENSATED, **kw),
             "fp64_fused": A.RunParams(precision=A.FP64_FUSED, **kw),
             "fp64_plain": A.RunParams(precision=A.FP64_PLAIN, **kw)}
    if lr:
        del forms["fp64_fused"]          # the fused FP64 form has no long-range field
    hs = {k: A.Handle(p, systems) for k, p in forms.items()}
    for h in hs.values():
        h.set_spins(S0)
    rows, done, t0 = [], 0, time.time()
    for c in sorted(checkpoints):
        for h in hs.values():
            h.step(c - done)
        done = c
        ref = hs["fp64_plain"].get_spins()
        row = {"steps": c}
        href = hs["fp64_plain"].get_field() if lr else None
        for k in [f for f in forms if f != "fp64_plain"]:
            row[f"max_abs_dS_{k}"] = float(np.abs(hs[k].get_spins() - ref).max())
            if lr:
                hk = hs[k].get_field()
                row[f"max_rel_dH_{k}"] = float(np.abs(hk - href).max() / np.abs(href).max())
        rows.append(row)
    for h in hs.values():
        h.close()
    return {"workload": name, "nspins": n, "T_K": float(systems[0].temperature), "wall_s": time.time() - t0,
            "rows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="northstar")
    ap.add_argument("--checkpoints", default="100,1000,10000")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    print(json.dumps(run(args.workload, [int(x) for x in args.checkpoints.split(",")], args.seed)))


if __name__ == "__main__":
    main()
