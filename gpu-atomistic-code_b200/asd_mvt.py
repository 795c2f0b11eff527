"""Magnetisation-versus-temperature driver (the reference's sim::MvT, src/mvt.cpp:21-476).

The reference loops over temperatures one at a time: equilibrate, then average |m_s| with a
RunningStat until the change of the mean and the variance fall below tolerances
(src/mvt.cpp:178-331, 258-275), copying spins to the host every `update` steps.  Here all
temperatures are replicas of one handle advancing together; |m_s| is pushed into running
statistics on the device (asd_sample_magnetisation), and the host reads the statistics only
every `check_every` samples to test convergence.

    python asd_mvt.py [--replicas 96] [--equil 20000] [--average 20000] [--update 100]
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

import asd_b200 as A
import asd_lattice as LT


def run_mvt(reps, equil, average, update=100, convmean=1e-4, convvar=1e-4, precision=A.FP32, seed=1,
            check_every=10, spins=None, dt=1e-16):
    """Returns mean |m_s|, its standard error (sqrt(var/n), uncorrelated-sample estimate), the
    sample count per replica and sublattice, and the steps run."""
    flags = A.FLAG_COMPENSATED if precision == A.FP32 else 0
    with A.Handle(A.RunParams(precision=precision, seed=seed, dt=dt, flags=flags, update=update), reps) as h:
        n = sum(r.nspins for r in reps)
        h.set_spins(spins if spins is not None else np.tile([0.0, 0.0, 1.0], (n, 1)))
        h.step(equil)
        h.reset_magnetisation_stats()
        steps = equil
        nsamp = max(1, average // update)
        for k in range(nsamp):
            h.step(update)
            h.sample_magnetisation()
            steps += update
            if (k + 1) % check_every == 0 and k + 1 >= 2 * check_every:
                st = h.magnetisation_stats()
                dmean = np.abs(st[..., 1] - st[..., 3])
                if np.all(dmean < convmean) and np.all(st[..., 2] < convvar):
                    break
        st = h.magnetisation_stats()
    mean = st[..., 1]
    sem = np.sqrt(st[..., 2] / np.maximum(st[..., 0], 1))
    return mean, sem, st[..., 0], steps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--replicas", type=int, default=96)
    ap.add_argument("--equil", type=int, default=20000)
    ap.add_argument("--average", type=int, default=20000)
    ap.add_argument("--update", type=int, default=100)
    ap.add_argument("--tmax", type=float, default=None, help="highest temperature (default 1.2 x 104 K)")
    ap.add_argument("--seed", type=int, default=4)
    args = ap.parse_args()
    reps, L, Ts = LT.replica_batch(args.replicas, seed=args.seed, Tmax=args.tmax)
    t0 = time.time()
    mean, sem, cnt, steps = run_mvt(reps, args.equil, args.average, args.update, convmean=0.0, convvar=0.0)
    wall = time.time() - t0
    rows = [{"edge": int(l), "T_K": float(t), "m": float(mean[r, 0]), "sem": float(sem[r, 0]), "samples": int(cnt[r, 0])}
            for r, (l, t) in enumerate(zip(L, Ts))]
    # temperature where <|m|> of the largest replicas crosses 0.5 (a finite-size Tc estimate)
    big = [row for row in rows if row["edge"] == max(L)]
    tc = None
    for a, b in zip(big, big[1:]):
        if a["m"] >= 0.5 > b["m"]:
            tc = a["T_K"] + (a["m"] - 0.5) * (b["T_K"] - a["T_K"]) / (a["m"] - b["m"])
    print(json.dumps({"steps": steps, "wall_s": wall, "nspins": int(sum(r.nspins for r in reps)),
                      "tc_half_m_K": tc, "rows": rows}))


if __name__ == "__main__":
    main()
