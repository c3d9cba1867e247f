"""Benchmark: cell-solves/s of the per-cell chemistry + Tgas BDF solve on B200.

Workload (N=1 line): the uneven-stiffness batching workload -- the
primordial3 network (cooling H2, CONT, CHEM; heating COMPRESS, CHEM; H2
opacity RIPAMONTI; gamma EXACT; evolve_T) on 262,144 cells per GPU at
rtol 1e-6, run as the captured hydro loop of the reference's collapse
driver: each step is one call -- tff of the current state, densities x 1.01,
dt = 0.01 tff, then the solve of every cell -- captured once as a CUDA graph
and replayed. Seeded synthetic inputs (n_H log-uniform in [1, 1e14] cm^-3,
Tgas in [50, 5000] K, x_H2 in [1e-6, 0.5], x_e in [1e-8, 1e-2]; no dataset
exists for this path). A step is 262,144 cell-solves.

  value     device-timed cell-solves/s of the K timed steps (inputs resident
            in HBM; each step's graph replay timed with CUDA events on its
            stream; an L2 flush of 256 MB is written between steps, outside
            the steps' events)
  e2e       the same loop through the public API: each call of
            krome_solve_cells on pinned host arrays timed on the host, its
            host->device and device->host copies inside; the caller's
            host-side compression between calls is not timed (as in the
            reference arm's loop)
  roofline  the solve kernel against the FP64 pipe: algorithmic flops from
            the per-cell CVODE counters the kernel writes x the network's
            counted work per rhs evaluation, over the kernel's event time;
            the peak is this GPU's DFMA rate measured live
  cpu_baseline  the reference's own krome_solve_cells (compiled from its
            sources with OpenMP, oracle/_ref) on the host cores, on the first
            cells of the same batch through the same loop
  forms     (N = 1) the kernel forms, each on its own workload, each with
            the reference's CPU solve of (a sample of) the same cells:
            small      the plain method's small workload: 4,096 primordial
                       cells, analytic Jacobian, dense LU, one solve
            batching   the batching workload itself (262,144 primordial3
                       cells, the hydro loop's first calls) with each
                       launch form: one lane / one warp per cell, each on
                       a persistent work-queue grid or a plain grid
            adjoint    the differentiation workload: 65,536 primordial cells
                       (cooling ATOMIC, H2; heating CHEM, COMPRESS; rtol 1e-6),
                       the plain solve, the recording solve and the reverse
                       sweep of the discrete adjoint (gradients of x_H2 and
                       Tgas w.r.t. n0, T0 and every ln k), device-timed; the
                       CPU's gradient is central differences
            precision  the precision workload: 131,072 galaxy_ism cells, the
                       Newton matrix factored in FP64 and in FP32 (FP64
                       refactor after Newton failures): cell-solves/s, the
                       FP64 refactors, and each form's error against the
                       rtol 1e-12 FP64 solve (the fraction of cells whose
                       abundances above atol/rtol and Tgas are within
                       10 rtol, the median and p99 of the cell's largest
                       relative error)
            large_network  the large-network workload: Semenov (655 species,
                       5,639 reactions, grain-surface chemistry), fixed Tgas,
                       the sparse-LU block-per-cell kernel on the first cells
                       of the seeded 16,384-cell batch: cell-solves/s, its
                       algorithmic bytes and DRAM traffic against the HBM peak
            large_network_cloud  the second large network on the same
                       kernel: the reference's dark-cloud chemistry (452
                       species, 4,429 reactions), 2,048 seeded cells

``python bench.py --gpus N --steps K --warmup W [--impl reference]``; with
N > 1 each rank (torchrun) solves its own 262,144 cells (weak scaling: no
collective on the data path; the max-over-ranks time is the job's).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

NETWORK = "primordial3"
RTOL = 1e-6
# DRAM bytes (read + write) the solve kernel moves per cell-solve in a
# hydro-loop call: one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum) of the third call of a 3-call primordial3 collapse
# loop on 65,536 cells, 10.31 + 9.53 GB in one launch; the traffic grows
# with the cells solved, so a launch of this benchmark moves this x its cells
TRAFFIC_PER_CELL_SOLVE = 19.84e9 / 65536
from krome_x_b200.krome import STAT_NAMES  # the per-cell counters' columns


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=262144, help="cells per GPU")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--cpu-cells", type=int, default=8192,
                    help="cells of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--large-cells", type=int, default=SEMENOV_CELLS,
                    help="cells of the large-network form (the workload's "
                         "batch is 16,384; the default is a seeded subset "
                         "that keeps the run within minutes)")
    ap.add_argument("--large-cpu-cells", type=int, default=512,
                    help="cells of the large-network form's CPU baseline")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the adjoint and precision forms")
    # one solve of a workload, outside the benchmark's timing: the command a
    # profiler wraps to capture a single kernel launch
    ap.add_argument("--case", default=None, metavar="NETWORK",
                    help="run one workload of NETWORK and print its time")
    ap.add_argument("--case-cells", type=int, default=65536)
    ap.add_argument("--calls", type=int, default=1,
                    help="--case: steps of the collapse loop")
    ap.add_argument("--layout", default="lane", choices=["lane", "warp"])
    ap.add_argument("--kernel", default="persistent",
                    choices=["persistent", "plain"])
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--lu32", action="store_true")
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--dt", type=float, default=None,
                    help="--case: every cell's time step")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_seed(rank):
    """each rank draws its own cells (weak scaling: one shard per rank, no
    exchange between ranks)"""
    return 1000 + rank


def job_times(values, dev, world):
    """the job's times: per entry the max over ranks of the local times
    (an all_reduce MAX; nothing on one rank)"""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=dev)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def job_rate(units_per_rank, world, seconds):
    """whole-job throughput: the units all ranks processed over the job's
    time"""
    return units_per_rank * world / seconds


def inputs(ncell, seed):
    from krome_x_b200 import netinfo, workloads
    info = netinfo.load(NETWORK)
    n, T, dt, par = workloads.primordial3(ncell, info, seed=seed)
    return info, n, T, dt, par


def options(net):
    # JAC_AUTO with Tgas evolved resolves to the difference-quotient
    # Jacobian, dense LU, as the reference; the persistent work-queue
    # kernel, one lane per cell
    return net.options(evolve_T=1, jac="auto", linsol="auto", rtol=RTOL,
                       atol_n=1e-20, atol_T=1e-6, kernel="persistent",
                       layout=1, lane_minb=2)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms"""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_flops(stats_sum, flops, N, ncells_solved):
    """W = (nfe + nfeDQ) F_rhs + nsetups (2/3 N^3 + N^2) + nni (2N^2 + 2N)
    + nst 14 N: the rhs evaluations at the network's counted work, the
    dense LU factorizations and solves, and the per-step vector work
    (CVODE's predictor, corrector and norms at a mean order of 3)"""
    s = dict(zip(STAT_NAMES, stats_sum))
    rhs = (s["nfe"] + s["nfeDQ"]) * flops["rhs_flops"]
    lu = s["nsetups"] * (2.0 / 3.0 * N ** 3 + N ** 2)
    sol = s["nni"] * (2.0 * N * N + 2.0 * N)
    vec = s["nst"] * 14.0 * N
    special = (s["nfe"] + s["nfeDQ"]) * flops["rhs_special"]
    return rhs + lu + sol + vec, special / max(ncells_solved, 1)


# ---------------------------------------------------------------------------
# the CPU legs: the reference's krome_solve_cells on the host cores

def _cpu_solver(key):
    """the reference's own library for a network (kind 'reference') or,
    where it was not built, the CPU oracle ('port')"""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc
    try:
        return orc.Reference(key), "reference"
    except (FileNotFoundError, OSError):
        return orc.Oracle(key), "port"


def _cpu_loop(args):
    """the collapse loop on the host, on the first `ncell` cells of rank
    0's seeded batch of `total` cells (the GPU arm's own first cells); run
    in a spawned process (one generated network per process)"""
    ncell, total, warm, steps, threads = args
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from krome_x_b200 import workloads
    info, n, T, dt, par = inputs(total, seed=rank_seed(0))
    n, T, dt, par = (np.ascontiguousarray(a[:ncell]) for a in (n, T, dt, par))
    opts = dict(evolve_T=1, jac=0, linsol=0, rtol=RTOL, atol_n=1e-20,
                atol_T=1e-6)
    solver, kind = _cpu_solver(NETWORK)
    secs = 0.0
    failed = 0
    for step in range(warm + steps):
        dt = workloads.hydro_step_info(n, par, info)
        t0 = time.perf_counter()
        out = solver.solve(n, T, dt, par, threads=threads, **opts)
        el = time.perf_counter() - t0
        ok = out["flags"] == 0
        n[ok] = out["n"][ok]
        T[ok] = out["T"][ok]
        if step >= warm:
            secs += el
            failed += int((~ok).sum())
    return dict(kind=kind, seconds=secs, cells=ncell, steps=steps,
                failed=failed)


def cpu_leg(ncell, total, warm, steps):
    import multiprocessing as mp
    threads = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(1) as pool:
        r = pool.map(_cpu_loop, [(ncell, total, warm, steps, threads)])[0]
    r["threads"] = threads
    r["value"] = r["cells"] * r["steps"] / r["seconds"]
    return r


def _cpu_once(args):
    """one solve of a form's workload on the host: the first `ncell` cells
    of the seeded batch of `total` cells the GPU form solves, best of
    `reps` (spawned process)"""
    key, total, ncell, seed, opts, threads, reps = args
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from krome_x_b200 import netinfo, workloads
    info = netinfo.load(key)
    n, T, dt, par = workloads.GENERATORS[key](total, info, seed=seed)
    n, T, dt, par = (np.ascontiguousarray(a[:ncell]) for a in (n, T, dt, par))
    solver, kind = _cpu_solver(key)
    best, failed = None, 0
    for _ in range(reps):
        t0 = time.perf_counter()
        out = solver.solve(n, T, dt, par, threads=threads, **opts)
        el = time.perf_counter() - t0
        best = el if best is None else min(best, el)
        failed = int((out["flags"] != 0).sum())
    return dict(kind=kind, seconds=best, cells=ncell, failed=failed)


def cpu_form(key, total, ncell, seed, opts, reps=1):
    """a form's CPU baseline: the reference's krome_solve_cells (OpenMP over
    cells, every host core) on the first ncell cells of the form's batch"""
    import multiprocessing as mp
    threads = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(1) as pool:
        r = pool.map(_cpu_once, [(key, total, ncell, seed, dict(opts),
                                  threads, reps)])[0]
    return {"value": r["cells"] / r["seconds"], "unit": "cell-solves/s",
            "cores": threads, "kind": r["kind"], "seconds": r["seconds"],
            "failed_cells": r["failed"],
            "sample": "the first %d cells of the form's seeded %d-cell batch, "
                      "one solve%s" % (ncell, total,
                                       ", best of %d" % reps if reps > 1 else "")}


def run_reference(args, rank):
    if rank != 0:
        return
    r = cpu_leg(args.cpu_cells, args.cells, args.warmup, args.steps)
    line = {
        "impl": "reference",
        "metric": "cell-solves/s", "value": r["value"],
        "unit": "cell-solves/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * r["seconds"] / r["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "primordial3 captured hydro loop (collapse "
                               "driver: tff, n x1.01, dt = 0.01 tff), rtol 1e-6",
                   "network": NETWORK, "cells_per_gpu": args.cells,
                   "sample_cells": r["cells"]},
        "cpu_baseline": {"value": r["value"], "unit": "cell-solves/s",
                         "cores": r["threads"], "kind": r["kind"],
                         "sample": "the first %d cells of the GPU arm's seeded "
                                   "%d-cell batch x %d loop calls (after %d "
                                   "warm-up calls)"
                                   % (r["cells"], args.cells, r["steps"],
                                      args.warmup)},
        "e2e": {"value": r["value"], "unit": "cell-solves/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# this library's leg

def _events(torch):
    e = torch.cuda.Event(enable_timing=True)
    e.record()
    return e


def adjoint_form(torch, dev, reps=3, cpu=True):
    """the discrete adjoint's cost on the differentiation workload"""
    from krome_x_b200 import autograd, krome, netinfo, workloads
    key, N = "primordial", 65536
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial(N, info, seed=0)
    net = krome.load(key)
    o = workloads.OPTIONS[key]
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"])
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    sp = info["species"]
    w = np.array([{"H": 1, "H+": 1, "H-": 1, "H2": 2, "H2+": 2, "HD": 1}
                  .get(x, 0) for x in sp], dtype=float)
    nH = t(n @ w)
    best = None
    for _ in range(reps):
        nd, Td = t(n), t(T)
        fl = torch.zeros(N, dtype=torch.int32, device=dev)
        cur = torch.zeros(1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        e0 = _events(torch)
        net.solve_device(nd, Td, t(dt), t(par), fl, opts=opts, cursor=cur)
        e1 = _events(torch)
        torch.cuda.synchronize()
        plain = e0.elapsed_time(e1)
        n0, T0 = t(n).requires_grad_(), t(T).requires_grad_()
        m = torch.zeros(net.nrea, dtype=torch.float64, device=dev,
                        requires_grad=True)
        torch.cuda.synchronize()
        e0 = _events(torch)
        nout, Tout, flags = autograd.solve(net, n0, T0, m, t(dt), t(par), opts)
        e1 = _events(torch)
        loss = (nout[:, sp.index("H2")] / nH).sum() + Tout.sum()
        e2 = _events(torch)
        loss.backward()
        e3 = _events(torch)
        torch.cuda.synchronize()
        rec, rev = e0.elapsed_time(e1), e2.elapsed_time(e3)
        r = (plain, rec, rev, int((flags != 0).sum()))
        if best is None or r[1] + r[2] < best[1] + best[2]:
            best = r
    plain, rec, rev, failed = best
    # the memory-bounded form: tapes of 4 GB at most (chunks of cells
    # recorded through one buffer, recomputed in the backward)
    budget = 4 * 2 ** 30
    n0, T0 = t(n).requires_grad_(), t(T).requires_grad_()
    m = torch.zeros(net.nrea, dtype=torch.float64, device=dev,
                    requires_grad=True)
    torch.cuda.synchronize()
    e0 = _events(torch)
    nout, Tout, flags = autograd.solve(net, n0, T0, m, t(dt), t(par), opts,
                                       max_tape_bytes=budget)
    e1 = _events(torch)
    loss = (nout[:, sp.index("H2")] / nH).sum() + Tout.sum()
    e2 = _events(torch)
    loss.backward()
    e3 = _events(torch)
    torch.cuda.synchronize()
    bounded = {"tape_bytes_max": budget,
               "forward_ms": e0.elapsed_time(e1),
               "backward_ms": e2.elapsed_time(e3),
               "gradient_over_forward":
                   (e0.elapsed_time(e1) + e2.elapsed_time(e3)) / plain}
    out = {"workload": "primordial, 65,536 cells, rtol 1e-6, outputs x_H2 "
                       "and Tgas, inputs n0, T0 and all %d ln k" % net.nrea,
           "plain_forward_ms": plain, "recording_forward_ms": rec,
           "reverse_sweep_ms": rev, "reverse_over_forward": rev / plain,
           "gradient_over_forward": (rec + rev) / plain,
           "failed_cells": failed, "reps": reps,
           "memory_bounded": bounded,
           "full_tape_bytes": N * autograd.DEFAULT_TAPE_CAP * 8}
    if cpu:
        # the reference has no adjoint: its gradient is central differences,
        # 2 (nspec + 1 + nrea) forward solves per cell
        cb = cpu_form(key, N, 4096, 0, o)
        nfd = 2 * (net.nspec + 1 + net.nrea)
        cb["fd_solves_per_gradient"] = nfd
        cb["gradient_cells_per_s"] = cb["value"] / nfd
        out["cpu_baseline"] = cb
        out["gpu_gradient_cells_per_s"] = N / ((rec + rev) * 1e-3)
    return out


def precision_form(torch, dev, cpu=True):
    """FP64 and FP32 Newton-matrix factorisations on the precision workload,
    against the rtol 1e-12 FP64 solve"""
    from krome_x_b200 import krome, netinfo, workloads
    key, N = "galaxy_ism", 131072
    info = netinfo.load(key)
    n, T, dt, par = workloads.galaxy_ism(N, info, seed=0)
    net = krome.load(key)
    o = workloads.OPTIONS[key]
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)

    def run(rtol, lu32):
        opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=rtol,
                           atol_n=o["atol_n"], atol_T=o["atol_T"], lu32=lu32,
                           max_steps=2000000)
        nd, Td = t(n), t(T)
        fl = torch.zeros(N, dtype=torch.int32, device=dev)
        st = torch.zeros((N, len(STAT_NAMES)), dtype=torch.int64, device=dev)
        cur = torch.zeros(1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        e0 = _events(torch)
        net.solve_device(nd, Td, t(dt), t(par), fl, opts=opts, stats=st,
                         cursor=cur)
        e1 = _events(torch)
        torch.cuda.synchronize()
        return (nd.cpu().numpy(), Td.cpu().numpy(), fl.cpu().numpy(),
                st.cpu().numpy(), e0.elapsed_time(e1))
    ref = run(1e-12, 0)

    def error(res):
        nn, TT, fl, _, _ = res
        ok = (fl == 0) & (ref[2] == 0)
        big = np.abs(ref[0][ok]) > o["atol_n"] / o["rtol"]
        with np.errstate(all="ignore"):
            rel = np.where(big, np.abs(nn[ok] - ref[0][ok]) / np.abs(ref[0][ok]),
                           0.0).max(axis=1)
        relT = np.abs(TT[ok] - ref[1][ok]) / np.abs(ref[1][ok])
        e = np.maximum(rel, relT)
        return {"cells_within_10rtol": float((e <= 10 * o["rtol"]).mean()),
                "median_rel_err": float(np.median(e)),
                "p99_rel_err": float(np.quantile(e, 0.99)),
                "failed_cells": int((fl != 0).sum())}
    out = {"workload": "galaxy_ism, 131,072 cells, rtol 1e-6, dt 3.15e11 s",
           "reference": "the FP64 solve at rtol 1e-12 on the GPU",
           "reference_ms": ref[4]}
    if cpu:
        out["cpu_baseline"] = cpu_form(key, N, 8192, 0, o)
    for name, lu32 in (("fp64", 0), ("lu32", 1)):
        runs = [run(o["rtol"], lu32) for _ in range(3)]
        best = min(runs, key=lambda r: r[4])
        d = {"cell_solves_per_s": N / (best[4] * 1e-3), "ms": best[4]}
        d.update(error(best))
        if lu32:
            d["fp64_refactors"] = int(best[3][:, STAT_NAMES.index("nlu64")].sum())
            d["cells_with_refactor"] = int(
                (best[3][:, STAT_NAMES.index("nlu64")] > 0).sum())
        out[name] = d
    return out


# the large-network form: DRAM bytes (read + write) of its solve kernel per
# integration step, from one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum) of `python bench.py --case semenov --case-cells 148 --dt
# 3.15e9` (154,747 steps: 2.29 + 6.27 GB); the per-cell workspace (~600 KB)
# stays in L2
SEMENOV_DRAM_PER_STEP = 8.57e9 / 154747
SEMENOV_CELLS = 2048
SEMENOV_BATCH = 16384


def large_network_form(torch, dev, ncell=SEMENOV_CELLS, cpu_cells=512):
    """the sparse-LU path on the large-network workload: Semenov (655
    species, 5,639 reactions), fixed Tgas, one launch of the block-per-cell
    kernel over a seeded subset of the 16,384-cell batch"""
    from krome_x_b200 import krome, netinfo, workloads
    key = "semenov"
    info = netinfo.load(key)
    n, T, dt, par = workloads.semenov(SEMENOV_BATCH, info, seed=0)
    n, T, dt, par = (np.ascontiguousarray(a[:ncell]) for a in (n, T, dt, par))
    net = krome.load(key)
    opts = net.options(**workloads.OPTIONS[key])
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    nd, Td = t(n), t(T)
    fl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    st = torch.zeros((ncell, len(STAT_NAMES)), dtype=torch.int64, device=dev)
    cur = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    e0 = _events(torch)
    net.solve_device(nd, Td, t(dt), t(par), fl, opts=opts, stats=st,
                     cursor=cur)
    e1 = _events(torch)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    S = st.cpu().numpy()
    steps = int(S[:, STAT_NAMES.index("nst")].sum())
    dram = SEMENOV_DRAM_PER_STEP * steps
    io = ncell * 8 * (2 * net.nspec + net.npar + 2)
    # the sparse path's algorithmic bytes: per Newton matrix the Jacobian and
    # the factors written and read, per Newton iteration the factors read,
    # per rhs the rates and two state vectors:
    # B = nsetups 8 (nnzJ + 2 nnzLU) + nni 8 nnzLU + nfe 8 (nrea + 2 nspec)
    tot = dict(zip(STAT_NAMES, S.sum(axis=0).astype(float)))
    nnz_j, nnz_lu = info["nnz_j"], info["nnz_lu"]
    alg = 8.0 * (tot["nsetups"] * (nnz_j + 2 * nnz_lu) + tot["nni"] * nnz_lu
                 + (tot["nfe"] + tot["nfeDQ"]) * (net.nrea + 2 * net.nspec))
    peak, peak_source = _hbm_peak()
    mass = np.asarray(info["mass_g"])
    out = nd.cpu().numpy()
    return {"workload": "Semenov (655 species, 5,639 reactions), fixed Tgas, "
                        "rtol 1e-6, dt 3.15e13 s, sparse LU; the first %d "
                        "cells of the seeded 16,384-cell batch" % ncell,
            "cell_solves_per_s": ncell / (ms * 1e-3), "ms": ms,
            "failed_cells": int((fl != 0).sum().item()),
            "mean_steps_per_cell": steps / ncell,
            "mass_conservation_max_rel": float(
                np.abs(out @ mass / (n @ mass) - 1).max()),
            "hbm": {"achieved_gbs": dram / (ms * 1e-3) / 1e9,
                    "peak_gbs": peak, "peak_source": peak_source,
                    "frac": dram / (ms * 1e-3) / 1e9 / peak,
                    "traffic_bytes": dram,
                    "traffic_source": "ncu DRAM bytes per integration step "
                                      "x the steps taken",
                    "algorithmic_bytes": alg,
                    "algorithmic_gbs": alg / (ms * 1e-3) / 1e9,
                    "algorithmic_frac": alg / (ms * 1e-3) / 1e9 / peak,
                    "algorithmic_bytes_formula":
                        "nsetups 8 (nnzJ + 2 nnzLU) + nni 8 nnzLU + nfe 8 "
                        "(nrea + 2 nspec), nnzJ %d, nnzLU %d, counters of "
                        "this launch" % (nnz_j, nnz_lu),
                    "cell_io_bytes": io},
            "cpu_baseline": cpu_form(key, SEMENOV_BATCH, cpu_cells, 0,
                                     workloads.OPTIONS[key])
            if cpu_cells > 0 else None}


def cloud_form(torch, dev, ncell=2048, cpu_cells=512):
    """the sparse path on the second large network: the reference's
    gas-phase dark-cloud chemistry (452 species, 4,429 reactions), fixed
    Tgas, one launch over the seeded 2,048-cell batch"""
    from krome_x_b200 import krome, netinfo, workloads
    key = "cloud"
    info = netinfo.load(key)
    n, T, dt, par = workloads.cloud(ncell, info, seed=0)
    net = krome.load(key)
    opts = net.options(**workloads.OPTIONS[key])
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    nd, Td = t(n), t(T)
    fl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    st = torch.zeros((ncell, len(STAT_NAMES)), dtype=torch.int64, device=dev)
    cur = torch.zeros(1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    e0 = _events(torch)
    net.solve_device(nd, Td, t(dt), t(par), fl, opts=opts, stats=st,
                     cursor=cur)
    e1 = _events(torch)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    tot = dict(zip(STAT_NAMES, st.cpu().numpy().sum(axis=0).astype(float)))
    nnz_j, nnz_lu = info["nnz_j"], info["nnz_lu"]
    alg = 8.0 * (tot["nsetups"] * (nnz_j + 2 * nnz_lu) + tot["nni"] * nnz_lu
                 + (tot["nfe"] + tot["nfeDQ"]) * (net.nrea + 2 * net.nspec))
    peak, peak_source = _hbm_peak()
    mass = np.asarray(info["mass_g"])
    out = nd.cpu().numpy()
    return {"workload": "cloud (452 species, 4,429 reactions), fixed Tgas, "
                        "rtol 1e-6, dt 3.15e13 s, sparse LU; %d seeded cells"
                        % ncell,
            "cell_solves_per_s": ncell / (ms * 1e-3), "ms": ms,
            "failed_cells": int((fl != 0).sum().item()),
            "mean_steps_per_cell": tot["nst"] / ncell,
            "mass_conservation_max_rel": float(
                np.abs(out @ mass / (n @ mass) - 1).max()),
            "hbm": {"algorithmic_bytes": alg,
                    "algorithmic_gbs": alg / (ms * 1e-3) / 1e9,
                    "peak_gbs": peak, "peak_source": peak_source,
                    "algorithmic_frac": alg / (ms * 1e-3) / 1e9 / peak,
                    "algorithmic_bytes_formula":
                        "nsetups 8 (nnzJ + 2 nnzLU) + nni 8 nnzLU + nfe 8 "
                        "(nrea + 2 nspec), nnzJ %d, nnzLU %d" % (nnz_j, nnz_lu)},
            "cpu_baseline": cpu_form(key, ncell, cpu_cells, 0,
                                     workloads.OPTIONS[key])
            if cpu_cells > 0 else None}


def batching_form(torch, dev, ncell=262144, calls=3):
    """the batching workload itself (262,144 primordial3 cells of rank 0's
    seeded batch, the captured hydro loop's first `calls` calls: the first,
    stiffest solve from the initial conditions, then hydro steps) with each
    launch form: one lane or one warp per cell, each as a persistent
    work-queue grid or a plain one-cell-per-lane (warp) grid; device-timed,
    every form from the same inputs"""
    from krome_x_b200 import krome, workloads
    info, n, T, dt, par = inputs(ncell, seed=rank_seed(0))
    net = krome.load(NETWORK)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    out = {"workload": "primordial3, %d cells, the hydro loop's first %d "
                       "calls (tff, n x1.01, dt = 0.01 tff; the first call "
                       "from the initial conditions), rtol 1e-6"
                       % (ncell, calls)}
    for layout in ("lane", "warp"):
        for kernel in ("persistent", "plain"):
            o = net.options(evolve_T=1, jac="auto", linsol="auto", rtol=RTOL,
                            atol_n=1e-20, atol_T=1e-6, kernel=kernel,
                            layout=1 if layout == "lane" else 0, lane_minb=2)
            nd, Td, pd = t(n), t(T), t(par)
            dtd = t(dt)
            fl = torch.zeros(ncell, dtype=torch.int32, device=dev)
            cur = torch.zeros(1, dtype=torch.int32, device=dev)
            per_call, failed = [], 0
            for c in range(calls):
                torch.cuda.synchronize()
                e0 = _events(torch)
                if c == 0:
                    net.solve_device(nd, Td, dtd, pd, fl, opts=o, cursor=cur)
                else:  # the collapse step and the solve on the device arrays
                    r = net._lib.krome_b200_hydro_step(
                        ncell, nd.data_ptr(), Td.data_ptr(), dtd.data_ptr(),
                        pd.data_ptr(), net.npar, net.params.index("tff"),
                        1.01, 0.01, fl.data_ptr(), None, cur.data_ptr(),
                        o._h, None)
                    assert r == 0, r
                e1 = _events(torch)
                torch.cuda.synchronize()
                per_call.append(e0.elapsed_time(e1))
                failed += int((fl != 0).sum().item())
            ms = sum(per_call)
            out["%s_%s" % (layout, kernel)] = {
                "cell_solves_per_s": calls * ncell / (ms * 1e-3), "ms": ms,
                "ms_per_call": per_call, "failed_cell_solves": failed}
    out["persistent_lane_over_plain_warp"] = (
        out["lane_persistent"]["cell_solves_per_s"]
        / out["warp_plain"]["cell_solves_per_s"])
    out["persistent_over_plain_lane_layout"] = (
        out["lane_persistent"]["cell_solves_per_s"]
        / out["lane_plain"]["cell_solves_per_s"])
    out["persistent_over_plain_warp_layout"] = (
        out["warp_persistent"]["cell_solves_per_s"]
        / out["warp_plain"]["cell_solves_per_s"])
    return out


def small_form(torch, dev, reps=5, cpu=True):
    """the plain method on its small CPU-runnable workload: 4,096 primordial
    cells (cooling ATOMIC, H2; heating CHEM, COMPRESS), dt = 3.15e10 s,
    rtol 1e-6, the analytic (hybrid) Jacobian, dense LU; device-timed, best
    of reps, beside the reference's krome_solve_cells on the same cells"""
    from krome_x_b200 import krome, netinfo, workloads
    key, N = "primordial", 4096
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial(N, info, seed=rank_seed(0))
    net = krome.load(key)
    o = workloads.OPTIONS[key]
    opts = net.options(**o)
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    best, failed = None, 0
    for _ in range(reps):
        nd, Td = t(n), t(T)
        fl = torch.zeros(N, dtype=torch.int32, device=dev)
        cur = torch.zeros(1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        e0 = _events(torch)
        net.solve_device(nd, Td, t(dt), t(par), fl, opts=opts, cursor=cur)
        e1 = _events(torch)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
        failed = int((fl != 0).sum().item())
    out = {"workload": "primordial, 4,096 cells, dt 3.15e10 s, rtol 1e-6, "
                       "analytic Jacobian, dense LU",
           "cell_solves_per_s": N / (best * 1e-3), "ms": best,
           "failed_cells": failed, "reps": reps}
    if cpu:
        out["cpu_baseline"] = cpu_form(key, N, N, rank_seed(0), o, reps=3)
    return out


def _hbm_peak():
    """the HBM roofline: the measured copy bandwidth of MEASURED_PEAKS.json,
    else the pool's earlier measurement (6.65 TB/s), and which"""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s, an earlier measurement)"


def run_ours(args, rank, world, local):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from krome_x_b200 import krome, workloads
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    net = krome.load(NETWORK)
    info, n, T, dt, par = inputs(args.cells, seed=rank_seed(rank))
    ncell = args.cells
    opts = options(net)
    flops = json.loads((ROOT / "krome_x_b200" / "networks"
                        / ("net_%s.flops.json" % NETWORK)).read_text())
    N = net.nspec + 1

    # ---- device-resident arrays and the captured hydro step ----
    n_d = torch.from_numpy(n).to(dev)
    T_d = torch.from_numpy(T).to(dev)
    dt_d = torch.from_numpy(dt).to(dev)
    par_d = torch.from_numpy(np.ascontiguousarray(par)).to(dev)
    flags_d = torch.zeros(ncell, dtype=torch.int32, device=dev)
    stats_d = torch.zeros((ncell, len(STAT_NAMES)), dtype=torch.int64,
                          device=dev)
    stream = torch.cuda.Stream(device=dev)
    graph = net.hydro_graph(n_d, T_d, dt_d, par_d, flags_d, opts,
                            stats=stats_d, stream=stream)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    stats_acc = torch.zeros(len(STAT_NAMES), dtype=torch.int64, device=dev)
    fails = torch.zeros(1, dtype=torch.int64, device=dev)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            graph.launch()
    torch.cuda.synchronize()
    peak = net.fp64_peak()

    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kst = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ken = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for k in range(args.steps):
            flush.zero_()
            kst[k].record(stream)
            graph.launch()
            ken[k].record(stream)
            stats_acc += stats_d.sum(0)
            fails += (flags_d != 0).sum()
        ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    # the timed steps are the graph replays (the hydro step: compression
    # and the solve), each bracketed by events on the launching stream; the
    # L2 flush and the counter sums between them are not steps
    bracket = ev0.elapsed_time(ev1) / 1e3
    kernel_s = sum(a.elapsed_time(b) for a, b in zip(kst, ken)) / 1e3
    bracket, kernel_s = job_times([bracket, kernel_s], dev, world)
    elapsed = kernel_s
    stats_sum = stats_acc.cpu().numpy().astype(float)
    n_failed = int(fails.item())
    value = job_rate(args.steps * ncell, world, elapsed)
    W, special = algorithmic_flops(stats_sum, flops, N, args.steps * ncell)
    achieved = W / kernel_s / 1e12
    graph.free()

    # ---- end to end through the public API (pinned host arrays) ----
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
    info2, n2, T2, dt2, par2 = inputs(ncell, seed=rank_seed(rank))
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    n2, T2, dt2, par2 = pin(n2), pin(T2), pin(dt2), pin(par2)
    fl2 = pin(np.zeros(ncell, dtype=np.intc))
    import ctypes
    D = ctypes.POINTER(ctypes.c_double)
    args_c = (ncell, n2.ctypes.data_as(D), T2.ctypes.data_as(D),
              dt2.ctypes.data_as(D), par2.ctypes.data_as(D), net.npar, None,
              fl2.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), opts._h)

    def public_step():
        # the caller's hydro update, then the reference-facing call:
        # krome_solve_cells on host arrays, in place (a failed cell keeps
        # its input), timed from the call to its return (the reference
        # arm's loop times its solve calls the same way)
        dt2[:] = workloads.hydro_step_info(n2, par2, info2)
        t0 = time.perf_counter()
        net._lib.krome_solve_cells(*args_c)
        el = time.perf_counter() - t0
        return el, int((fl2 != 0).sum())

    for _ in range(args.warmup):
        public_step()
    if world > 1:
        dist.barrier()
    e2e_s, e2e_failed = 0.0, 0
    for _ in range(e2e_steps):
        el, f = public_step()
        e2e_s += el
        e2e_failed += f
    e2e_s, = job_times([e2e_s], dev, world)
    e2e_value = job_rate(e2e_steps * ncell, world, e2e_s)
    h2d = n.nbytes + T.nbytes + dt.nbytes + par.nbytes
    d2h = n.nbytes + T.nbytes + 4 * ncell

    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        cpu_forms = not args.no_cpu_baseline
        forms = {"small": small_form(torch, dev, cpu=cpu_forms),
                 "batching": batching_form(torch, dev, ncell),
                 "adjoint": adjoint_form(torch, dev, cpu=cpu_forms),
                 "precision": precision_form(torch, dev, cpu=cpu_forms),
                 "large_network": large_network_form(
                     torch, dev, args.large_cells,
                     args.large_cpu_cells if cpu_forms else 0),
                 "large_network_cloud": cloud_form(
                     torch, dev, cpu_cells=512 if cpu_forms else 0)}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_leg(args.cpu_cells, args.cells, args.warmup, args.steps)
        cpu = {"value": r["value"], "unit": "cell-solves/s",
               "cores": r["threads"], "kind": r["kind"],
               "sample": "the first %d cells of the timed %d-cell batch "
                         "x %d loop calls (after %d warm-up calls), the "
                         "reference's krome_solve_cells with OpenMP over "
                         "cells" % (r["cells"], ncell, r["steps"],
                                    args.warmup)}
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    s = dict(zip(STAT_NAMES, (stats_sum / (args.steps * ncell)).round(3)))
    line = {
        "metric": "cell-solves/s", "value": value, "unit": "cell-solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded primordial3 collapse cells)",
        "config": {"workload": "primordial3 captured hydro loop (collapse "
                               "driver: tff, n x1.01, dt = 0.01 tff), rtol 1e-6, "
                               "persistent lane-per-cell kernel",
                   "network": NETWORK, "cells_per_gpu": ncell,
                   "global_cells": ncell * world, "parallelism": "dp%d" % world,
                   "l2": "256 MB flush buffer written between steps",
                   "timed": "each step's graph replay between CUDA events "
                            "on its stream (the flush and the counter sums "
                            "between steps excluded)",
                   "ms_per_step_with_flush": 1e3 * bracket / args.steps,
                   "failed_cell_solves": n_failed,
                   "counters_per_cell_solve": s},
        "e2e": {"value": e2e_value, "unit": "cell-solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "steps": e2e_steps, "failed_cell_solves": e2e_failed,
                "timed": "each krome_solve_cells call on pinned host arrays "
                         "(its copies inside; the caller's host-side "
                         "compression between calls outside, as in the "
                         "reference arm)"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": TRAFFIC_PER_CELL_SOLVE * ncell,
                     "traffic_unit": "bytes per launch (ncu, scaled from "
                                     "65,536 cells by the cells solved)",
                     "peak_source": "measured live: DFMA chains over all SMs",
                     "work": "per cell-solve %.4g flops (special functions "
                             "counted 1 each: %.4g per cell-solve)"
                             % (W / (args.steps * ncell), special)},
        "gpu_launches": 2 * args.steps,
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if forms is not None:
        line["forms"] = forms
    print(json.dumps(line), flush=True)


def run_case(args):
    """--case: one workload through the public API, timed on the host (a
    profiler's capture target; not a benchmark line). With --calls > 1 the
    collapse driver's hydro loop on the host arrays; with --adjoint the
    discrete adjoint through the torch.autograd wrapper."""
    from krome_x_b200 import krome, netinfo, workloads
    info = netinfo.load(args.case)
    n, T, dt, par = workloads.GENERATORS[args.case](args.case_cells, info,
                                                    seed=args.seed)
    if args.dt is not None:
        dt[:] = args.dt
    o = workloads.OPTIONS[args.case]
    net = krome.load(args.case)
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel=args.kernel,
                       layout=0 if args.layout == "warp" else 1,
                       lu32=int(args.lu32), max_steps=o.get("max_steps", 100000))
    out = {"case": args.case, "cells": args.case_cells, "calls": args.calls}
    if args.adjoint:
        import torch
        from krome_x_b200 import autograd
        dev = torch.device("cuda:0")
        t = lambda x: torch.tensor(x, dtype=torch.float64, device=dev)
        n0, T0 = t(n).requires_grad_(), t(T).requires_grad_()
        m = torch.zeros(net.nrea, dtype=torch.float64, device=dev,
                        requires_grad=True)
        t0 = time.perf_counter()
        nout, Tout, flags = autograd.solve(net, n0, T0, m, t(dt), t(par), opts)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        (nout[:, info["species"].index("H2")].sum() + Tout.sum()).backward()
        torch.cuda.synchronize()
        out.update(forward_s=t1 - t0, reverse_s=time.perf_counter() - t1,
                   failed=int((flags != 0).sum()))
    else:
        failed = 0
        t0 = time.perf_counter()
        for c in range(args.calls):
            if c > 0:
                dt = workloads.hydro_step_info(n, par, info)
            r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
            n, T = r.n, r.Tgas
            failed += int((r.flags != 0).sum())
        el = time.perf_counter() - t0
        out.update(seconds=el, cell_solves_per_s=args.case_cells * args.calls / el,
                   failed=failed)
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.case is not None:
        run_case(args)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
