"""Magnetisation-versus-temperature driver (the reference's sim::MvT, src/mvt.cpp:21-476).

The reference loops over temperatures one at a time: equilibrate, then average |m_s| with a
RunningStat until the change of the mean and the variance fall below tolerances
(src/mvt.cpp:178-331, 258-275), copying spins to the host every `update` steps.  Here all
temperatures are replicas of one handle advancing together; |m_s| is pushed into running
statistics on the device (asd_sample_magnetisation), and the host reads the statistics only
every `check_every` samples to test convergence.

    python asd_mvt.py [--replicas 96] [--equil 20000] [--average 20000] [--update 100]
    torchrun --nproc-per-node N asd_mvt.py ...   (temperatures split over N GPUs, rows gathered to rank 0)
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

import asd_b200 as A
import asd_lattice as LT
import asd_replicas as R


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


def compare(args):
    """M(T) of the FP32 form against the FP64 plain form on the same replicas and seeds: at finite
    T the trajectories decorrelate, so the check is statistical, per replica
    z = (m32 - m64) / sqrt(sem32^2 + sem64^2), with the share of |z| < 2 reported."""
    edges = tuple(int(e) for e in args.edges.split(","))
    reps, L, Ts = LT.replica_batch(args.replicas, edges=edges, seed=args.seed, Tmax=args.tmax)
    out = {}
    for name, prec in (("fp32", A.FP32), ("fp64_plain", A.FP64_PLAIN)):
        t0 = time.time()
        mean, sem, cnt, steps = run_mvt(reps, args.equil, args.average, args.update, convmean=0.0, convvar=0.0,
                                        precision=prec, seed=args.seed)
        out[name] = (mean[:, 0], sem[:, 0], time.time() - t0)
    m32, s32, w32 = out["fp32"]
    m64, s64, w64 = out["fp64_plain"]
    z = (m32 - m64) / np.sqrt(np.maximum(s32 ** 2 + s64 ** 2, 1e-300))
    hot = Ts > 0
    rows = [{"edge": int(l), "T_K": float(t), "m_fp32": float(a), "sem_fp32": float(b), "m_fp64": float(c),
             "sem_fp64": float(d), "z": float(e)} for l, t, a, b, c, d, e in zip(L, Ts, m32, s32, m64, s64, z)]
    print(json.dumps({"steps": steps, "wall_s_fp32": w32, "wall_s_fp64_plain": w64,
                      "within_2sigma": float(np.mean(np.abs(z[hot]) < 2.0)), "max_abs_z": float(np.abs(z[hot]).max()),
                      "rows": rows}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--replicas", type=int, default=96)
    ap.add_argument("--equil", type=int, default=20000)
    ap.add_argument("--average", type=int, default=20000)
    ap.add_argument("--update", type=int, default=100)
    ap.add_argument("--tmax", type=float, default=None, help="highest temperature (default 1.2 x 104 K)")
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--edges", default="16,24,32,48,64", help="replica edge lengths to draw from")
    ap.add_argument("--compare-fp64", action="store_true",
                    help="also run the FP64 plain form and report (m32 - m64) / sqrt(sem32^2 + sem64^2)")
    args = ap.parse_args()
    if args.compare_fp64:
        compare(args)
        return
    reps, L, Ts = LT.replica_batch(args.replicas, seed=args.seed, Tmax=args.tmax)
    # under torchrun each rank (one GPU) runs its share of the temperatures
    dist = None
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    rank = dist.get_rank() if dist else 0
    mine = R.shard([r.nspins for r in reps], rank, world)
    t0 = time.time()
    mean, sem, cnt, steps = run_mvt([reps[g] for g in mine], args.equil, args.average, args.update, convmean=0.0,
                                    convvar=0.0)
    wall = R.allmax(time.time() - t0, dist)
    part = [{"edge": int(L[g]), "T_K": float(Ts[g]), "m": float(mean[k, 0]), "sem": float(sem[k, 0]),
             "samples": int(cnt[k, 0])} for k, g in enumerate(mine)]
    rows = R.gather_rows(part, mine, dist, len(reps))
    if dist:
        dist.destroy_process_group()
    if rows is None:
        return
    # temperature where <|m|> of the largest replicas crosses 0.5 (a finite-size Tc estimate)
    big = [row for row in rows if row["edge"] == max(L)]
    tc = None
    for a, b in zip(big, big[1:]):
        if a["m"] >= 0.5 > b["m"]:
            tc = a["T_K"] + (a["m"] - 0.5) * (b["T_K"] - a["T_K"]) / (a["m"] - b["m"])
    print(json.dumps({"steps": steps, "wall_s": wall, "ranks": world, "nspins": int(sum(r.nspins for r in reps)),
                      "tc_half_m_K": tc, "rows": rows}))


if __name__ == "__main__":
    main()
