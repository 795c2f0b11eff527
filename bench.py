#!/usr/bin/env python
"""Benchmark of the sLLG step: spin-updates/s on one B200 (or N replicas on N GPUs).

Default workload ("sc128x128x64_dipole"): the 1M-spin exchange + dipolar lattice, simple cubic
128x128x64 (1,048,576 spins), open boundaries, nearest-neighbour exchange in CSR (SELL-32 on
the device) plus the point-dipole field by zero-padded FFT on the 256x256x128 mesh, refreshed
every step, Heun, T=0, FP32 state with FP64 renormalisation.  Other workloads (--workload):
bct2_64 (BCT-2 64^3 cells, 26 neighbours, full 3x3 tensors, T=300 K), bct2_64_dia, sc16,
replicas96, sc128_fft, film_rk4.  Prints one JSON line (rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import re
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "gpu-atomistic-code_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

FLUSH_BYTES = 256 << 20     # twice the B200's 126 MB L2
METRIC = "spin-updates/s on 1 B200: FP32 batched vs FP64 plain at stated err vs FP64"
PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def pinned(n):
    """A float64 numpy array of n elements in page-locked host memory (cudaHostAlloc, portable)."""
    import ctypes
    import numpy as np
    rt = ctypes.CDLL("libcudart.so.12")
    p = ctypes.c_void_p()
    rc = rt.cudaHostAlloc(ctypes.byref(p), ctypes.c_size_t(8 * max(n, 1)), ctypes.c_uint(1))
    if rc != 0:
        raise RuntimeError(f"cudaHostAlloc failed ({rc})")
    arr = np.frombuffer((ctypes.c_double * max(n, 1)).from_address(p.value), dtype=np.float64)[:n]
    return arr, (rt, p)


def ncu_traffic(workload, kernel):
    """Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel` on
    `workload` from the committed ncu table profiles/dram_traffic.csv (columns workload, kernel
    prefix, bytes, source capture), or None."""
    path = os.path.join(REPO, "profiles", "dram_traffic.csv")
    if not os.path.exists(path):
        return None
    import csv
    with open(path) as f:
        for row in csv.DictReader(f):
            if row["workload"] == workload and kernel.startswith(row["kernel"]):
                return float(row["bytes"])
    return None


def make_workload(name):
    import asd_b200 as A
    import asd_lattice as LT
    if name == "bct2_64":
        s = LT.bct2_antiferromagnet(64, layout="csr", T=300.0)
        return [s], dict(integrator=A.HEUN, dt=1e-16), {"lattice": "bct2 64x64x64 cells", "nspins": s.nspins,
                                                         "neighbours": 26, "tensor": "full 3x3", "exchange": "CSR",
                                                         "integrator": "heun", "T_K": 300.0}
    if name == "bct2_64_dia":
        s = LT.bct2_antiferromagnet(64, layout="dia", T=300.0)
        return [s], dict(integrator=A.HEUN, dt=1e-16), {"lattice": "bct2 64^3 cells", "nspins": s.nspins,
                                                         "exchange": "DIA", "integrator": "heun", "T_K": 300.0}
    if name == "sc16":
        s = LT.sc_ferromagnet(16, T=300.0)
        return [s], dict(integrator=A.HEUN, dt=1e-16), {"lattice": "sc 16^3", "nspins": s.nspins, "T_K": 300.0}
    if name == "replicas96":
        reps, L, Ts = LT.replica_batch(96)
        return reps, dict(integrator=A.HEUN, dt=1e-16), {"lattice": "96 sc replicas, edges U{16..64} seed 4",
                                                          "nspins": int(sum(r.nspins for r in reps)),
                                                          "T_K": "0..1.2*104"}
    if name == "sc128_fft":
        s = LT.sc_fft(128)
        return [s], dict(integrator=A.HEUN, dt=1e-16), {"lattice": "sc 128^3 open, pad 256^3", "nspins": s.nspins,
                                                         "field": "dipole+exchange via R2C/C2R FFT", "T_K": 0.0}
    if name == "sc128x128x64_dipole":
        s = LT.sc_ferromagnet((128, 128, 64), pbc=(0, 0, 0), dipole=True)
        return [s], dict(integrator=A.HEUN, dt=1e-16, update=1), {"lattice": "sc 128x128x64 open", "nspins": s.nspins,
                                                                   "field": "CSR NN exchange + FFT dipole every step",
                                                                   "T_K": 0.0}
    if name == "film_rk4":
        s = LT.film_dia(1024, 1024, 4)
        return [s], dict(integrator=A.RK4, dt=5e-16, update=1), {"lattice": "film 1024x1024x4", "nspins": s.nspins,
                                                                  "exchange": "DIA J1+J2", "integrator": "rk4"}
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, max, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.out = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.out.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- reference arm
# The reference's CPU step cannot evaluate the dipole field here (its FFT path needs FFTW3, which
# is absent), so the sc 128x128x64 dipole lattice runs on the FP64 restatement with the long-range field by
# threaded FFT (oracle/fft_oracle.py, pinned against the direct-sum oracle); lattices without a
# long-range field run the reference's own llgCPU compiled from source.  Neither loads the
# product library: the sc 128x128x64 CSR comes from a numpy builder that is bit-exact with the
# reference's exchunitcell, the BCT-2 CSR from the reference's exchunitcell itself.
NS_DIM = (128, 128, 64)
REF_STEP_CAP = 60          # at most this many timed CPU steps per run (~1.3 s each at 1M spins, 8 cores)


def cpu_port_sc128x128x64(steps, warmup, workers=None):
    """FFT restatement on the sc 128x128x64 dipole lattice: (spin-updates/s, seconds, spins, threads, steps)."""
    sys.path[:0] = [REPO]
    from oracle import fft_oracle as F
    s = F.sc_dipole_system(NS_DIM)
    o = F.FFTOracle(s, dt=1e-16, update=1, workers=workers)
    o.set_spins(F.random_spins(s.nspins, 0))
    o.step(warmup)
    secs = o.timed_steps(steps)
    return s.nspins * steps / secs, secs, s.nspins, o.workers, steps


def _ref_worker(args):
    """One process: the reference llgCPU on the BCT-2 lattice, CSR from the reference's exchunitcell."""
    cells, steps, warmup, seed = args
    sys.path[:0] = [REPO, PKG]
    import numpy as np
    from asd_lattice import _bct2_bonds           # bond list only (numpy); no library call
    from oracle import oracle as O
    ba, bt, bv, bj = _bct2_bonds(np.random.default_rng(2))
    xadj, adj, val = O.ref_exchunitcell((cells,) * 3, (1, 1, 1), [1.5, 1.5],
                                        [(a, b, v, np.asarray(j).reshape(3, 3)) for a, b, v, j in zip(ba, bt, bv, bj)])
    from types import SimpleNamespace as NS
    mats = [NS(mu=1.5, lam=0.01, gamma=1.0, k1u=-1e-23, k1u_dir=(0.0, 0.0, 1.0), sublattice=q) for q in (0, 1)]
    s = NS(nspins=2 * cells ** 3, materials=mats, atom=None, exch=2, full=True, xadj=xadj, adjncy=adj, csr_val=val,
           temperature=300.0, site_field=None)
    r = O.RefLLGCPU(s, seed=(seed, seed + 100))
    rng = np.random.default_rng(seed)
    z = rng.uniform(-1, 1, s.nspins)
    ph = rng.uniform(0, 2 * np.pi, s.nspins)
    r.set_spins(np.stack([np.sqrt(1 - z * z) * np.cos(ph), np.sqrt(1 - z * z) * np.sin(ph), z], 1))
    r.step(warmup)
    t0 = time.perf_counter()
    r.step(steps)
    return s.nspins, steps, time.perf_counter() - t0


def cpu_reference(cells, steps, warmup, procs):
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(cells, steps, warmup, 1 + k) for k in range(procs)])
    wall = max(r[2] for r in res)
    total = sum(r[0] * r[1] for r in res)
    return total / wall, res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    base = {"metric": METRIC, "unit": "spin-updates/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic"}
    k = max(1, min(args.steps, REF_STEP_CAP))
    if args.workload == "sc128x128x64_dipole":
        rate, secs, n, thr, k = cpu_port_sc128x128x64(k, min(args.warmup, 2))
        sample = (f"FP64 restatement of the reference's Heun step (oracle/fft_oracle.py: CSR exchange, dipole by "
                  f"threaded FFT on the 256x256x128 mesh, pinned against the direct-sum oracle) on the same "
                  f"sc 128x128x64 open lattice and initial spins, {k} timed steps of the whole lattice "
                  f"({secs:.1f} s), {thr} threads")
        kind = "port"
        cfg = {"workload": "sc128x128x64_dipole", "lattice": "sc 128x128x64 open", "nspins": n,
               "field": "CSR NN exchange + FFT dipole every step", "T_K": 0.0, "integrator": "heun",
               "same_config": True}
    elif args.workload == "bct2_64":
        procs = os.cpu_count() or 1
        k = max(1, min(args.steps, 30))
        rate, res = cpu_reference(64, k, min(args.warmup, 2), procs)
        secs = max(r[2] for r in res)
        n, thr = res[0][0], procs
        sample = (f"reference llgCPU (src/llgCPU.cpp, compiled from source) on the same BCT-2 64^3-cell lattice "
                  f"({n} spins, 26 nbrs, full 3x3 CSR from the reference's exchunitcell, T=300 K), one "
                  f"independent replica per process x {procs} processes, {k} timed steps each ({secs:.1f} s)")
        kind = "reference"
        cfg = {"workload": "bct2_64", "nspins_per_process": n, "processes": procs, "same_config": True}
    else:
        print(json.dumps({"impl": "reference", "unavailable": f"no CPU reference arm for workload {args.workload}"}))
        return
    line = dict(base, value=rate, ms_per_step=1e3 * secs / k, config=cfg, steps_run=k,
                cpu_baseline={"value": rate, "unit": "spin-updates/s", "cores": thr, "kind": kind, "sample": sample},
                e2e={"value": rate, "unit": "spin-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import numpy as np
    import asd_b200 as A
    import asd_lattice as LT

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    else:
        try:
            import ctypes
            ctypes.CDLL("libcudart.so.12").cudaSetDevice(local)
        except OSError:
            pass

    streamed = args.workload.endswith("_streamed")      # keep every tensor in the matrix stream
    systems, kw, cfg = make_workload(args.workload[: -len("_streamed")] if streamed else args.workload)
    n = sum(s.nspins for s in systems)
    S0 = LT.random_spins(n, 0)
    flags = A.FLAG_COMPENSATED | (0 if args.launch_shape else A.FLAG_AUTOTUNE) | \
        (A.FLAG_STREAMED_EXCHANGE if streamed else 0)
    p32 = A.RunParams(precision=A.FP32, seed=1 + rank, flags=flags, **kw)
    h = A.Handle(p32, systems)
    if args.launch_shape:
        blk, stg = (int(x) for x in args.launch_shape.split(","))
        h.set_launch_shape(blk, stg)
    if args.layout:
        h.set_device_layout(A.EXCH_DIA if args.layout == "dia" else A.EXCH_CSR)
    h.set_spins(S0)
    h.step(args.warmup)
    h.sync()

    def barrier():
        if dist:
            import torch
            t = torch.zeros(1, device="cuda")
            dist.all_reduce(t)
            torch.cuda.synchronize()

    def allmax(v):
        if not dist:
            return v
        import torch
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # timed region: every step starts with a cold L2 (an untimed 256 MB device write, twice the
    # L2) and is bracketed by its own CUDA events; the graph-replayed, L2-resident rate is
    # reported beside it
    barrier()
    with ClockSampler(local) as clk:
        ms, launches = h.time_steps_cold(args.steps, FLUSH_BYTES)
    barrier()
    ms = allmax(ms)
    value = n * world * args.steps / (ms * 1e-3)
    ms_warm, _ = h.time_steps(args.steps)
    ms_warm = allmax(ms_warm)

    # dominant kernel: per-launch CUDA-event time of the fused stage kernel, cold L2 per launch
    # every kernel of the step timed launch by launch with a cold L2; the dominant one (largest
    # summed time) carries the roofline, the others are listed beside it
    ks = h.time_kernels(max(4, min(args.steps, 20)), FLUSH_BYTES)
    peak, peak_kind = hbm_peak()
    achieved = ks["bytes"] / (ks["avg_ms"] * 1e-3) / 1e9 if ks["avg_ms"] > 0 else None
    traffic = ncu_traffic(args.workload, ks["name"])
    kernels = [{"kernel": k["name"], "avg_ms": k["avg_ms"], "launches": k["count"], "alg_bytes_per_launch": k["bytes"],
                "achieved_gbs": k["bytes"] / (k["avg_ms"] * 1e-3) / 1e9 if k["avg_ms"] > 0 else None,
                "frac": (k["bytes"] / (k["avg_ms"] * 1e-3) / 1e9 / peak) if k["avg_ms"] > 0 else None,
                "traffic": ncu_traffic(args.workload, k["name"])} for k in ks["kernels"]]

    # end to end through the C ABI with host buffers: upload spins, per step set the
    # applied field (H2D) + step + magnetisation read-back (D2H), download spins
    nsub_out = h.nrep * h.nsub * 3
    he = A.Handle(p32, systems)
    if args.launch_shape:
        he.set_launch_shape(blk, stg)
    he.step(1)
    he.sync()
    # host buffers in page-locked memory: spins in and out, the applied field, the magnetisation
    s_in, k1 = pinned(3 * n)
    s_out, k2 = pinned(3 * n)
    f_in, k3 = pinned(3)
    m_out, k4 = pinned(nsub_out)
    s_in[:] = S0.reshape(-1)
    f_in[:] = 0.0
    he.magnetisation(m_out)
    barrier()
    t0 = time.perf_counter()
    he.set_spins(s_in)
    for k in range(args.steps):
        he.set_applied(f_in)
        he.step(1)
        he.magnetisation(m_out)
    he.get_spins(s_out)
    e2e_s = allmax(time.perf_counter() - t0)
    barrier()
    he.close()
    for rt, ptr in (k1, k2, k3, k4):
        rt.cudaFreeHost(ptr)
    e2e = {"value": n * world * args.steps / e2e_s, "unit": "spin-updates/s",
           "h2d_bytes_per_step": (24 * n + 24 * args.steps) / args.steps,
           "d2h_bytes_per_step": (24 * n + 8 * nsub_out * args.steps) / args.steps,
           "calls_per_step": "asd_set_applied + asd_step(1) + asd_magnetisation", "host_buffers": "pinned"}

    # FP64 plain form on the same input; the FP32 and fused FP64 forms' errors against it on the
    # same noise, and the fused FP64 form's throughput
    plain = None
    err = None
    fused64 = None
    if not args.no_plain:
        pp = A.RunParams(precision=A.FP64_PLAIN, seed=1 + rank, **kw)
        hp = A.Handle(pp, systems)
        hp.set_spins(S0)
        kp = max(3, args.steps // 2)
        hp.step(min(3, kp))
        hp.sync()
        msp, lp = hp.time_steps_cold(kp, FLUSH_BYTES)
        msp = allmax(msp)
        plain = {"value": n * world * kp / (msp * 1e-3), "ms_per_step": msp / kp, "steps": kp, "gpu_launches": lp}
        hp.close()
        p64 = A.RunParams(precision=A.FP64_FUSED, seed=1 + rank, flags=A.FLAG_AUTOTUNE, **kw)
        hf = A.Handle(p64, systems)
        hf.set_spins(S0)
        hf.step(3)
        hf.sync()
        msf, lf = hf.time_steps_cold(kp, FLUSH_BYTES)
        msf = allmax(msf)
        hf.close()
        ne = args.err_steps
        hs = {k: A.Handle(pr, systems) for k, pr in (("fp32", p32), ("fp64_fused", p64), ("plain", pp))}
        for hh in hs.values():
            hh.set_spins(S0)
            hh.step(ne)
        ref = hs["plain"].get_spins()
        e32 = float(np.abs(hs["fp32"].get_spins() - ref).max())
        e64 = float(np.abs(hs["fp64_fused"].get_spins() - ref).max())
        for hh in hs.values():
            hh.close()
        err = {"max_abs_dS": e32, "steps": ne, "vs": "FP64 plain form, same initial spins and same Philox noise"}
        fused64 = {"value": n * world * kp / (msf * 1e-3), "ms_per_step": msf / kp, "steps": kp, "gpu_launches": lf,
                   "max_abs_dS_vs_fp64_plain": e64, "err_steps": ne,
                   "speedup_vs_fp64_plain": (msp / msf)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            if args.workload == "sc128x128x64_dipole":
                rate, secs, nn, thr, k = cpu_port_sc128x128x64(args.cpu_steps, 1)
                cpu = {"value": rate, "unit": "spin-updates/s", "cores": thr, "kind": "port",
                       "sample": f"FP64 restatement (oracle/fft_oracle.py: CSR exchange, dipole by threaded FFT) on "
                                 f"the same sc 128x128x64 lattice and spins, {k} whole-lattice steps "
                                 f"({secs:.1f} s), {thr} threads"}
            else:
                k = max(1, min(args.cpu_steps, 60))
                rate, res = cpu_reference(64, k, 1, 1) if args.workload == "bct2_64" else (None, None)
                if rate is None:
                    raise RuntimeError(f"no CPU baseline for workload {args.workload}")
                cpu = {"value": rate, "unit": "spin-updates/s", "cores": 1, "kind": "reference",
                       "sample": f"reference llgCPU (src/llgCPU.cpp compiled from source) on the same BCT-2 64^3-cell "
                                 f"lattice ({res[0][0]} spins, CSR from the reference's exchunitcell, T=300 K), "
                                 f"{k} steps ({res[0][2]:.1f} s), 1 thread (the reference has no threading)"}
        except Exception as e:  # the checkers are built by __graft_entry__.build()
            cpu = {"value": None, "unit": "spin-updates/s", "cores": None, "kind": "port",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "spin-updates/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict({"workload": args.workload}, **cfg, parallelism=f"replicas x{world}",
                               l2="L2 flushed before every timed step (256 MB device write, untimed); "
                                  "steps timed one by one with CUDA events",
                               state="FP32 hi+lo spins, FP64 renormalisation", launch_shape=h.tuning()),
                "value_l2_resident": n * world * args.steps / (ms_warm * 1e-3),
                "e2e": e2e,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                             "kernel": ks["name"], "kernel_avg_ms": ks["avg_ms"],
                             "alg_bytes_per_launch": ks["bytes"], "peak_source": peak_kind},
                "kernels": kernels,
                "cpu_baseline": cpu, "clocks": clk.summary(), "gpu_launches": launches,
                "fp64_plain": plain, "error_vs_fp64": err, "fp64_fused": fused64,
                "speedup_vs_fp64_plain": (value / plain["value"]) if plain else None}
        print(json.dumps(line), flush=True)
    h.close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sc128x128x64_dipole")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=8,
                    help="whole-lattice steps of the CPU baseline (sc 128x128x64 dipole lattice: ~1.3 s each on 8 cores)")
    ap.add_argument("--err-steps", type=int, default=100)
    ap.add_argument("--layout", default="", choices=["", "sell", "dia"],
                    help="device layout of the exchange matrix instead of the autotuner's choice")
    ap.add_argument("--launch-shape", default="",
                    help="block,staging for the fused stage kernel instead of the autotuner's choice "
                         "(staging 0 none, 1 words, 2 words+spins)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
