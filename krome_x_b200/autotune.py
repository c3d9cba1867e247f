"""Pick the solve kernel's launch shape by measurement.

The batched solve has four shapes that trade occupancy, register budget,
local-memory footprint and load balance, and the best one depends on the
network (its rhs size, N) and on the batch (how uneven the cells' stiffness
is):

  layout         0 one warp per cell (the LU row-per-lane in registers),
                 1 one lane per cell (private LU, warp-served Jacobians)
  lane_minb      2, 3, 4: the lane kernel's register budget (resident
                 128-thread blocks per SM it is compiled for)
  blocks_per_sm  the persistent grid's blocks per SM (0: the occupancy
                 limit; fewer resident lanes keep their state in L2)
  queue_chunk    cells per work-queue pop (warp layout)

``tune(net, n, Tgas, dt, par, opts)`` solves a sample of the caller's own
cells (at most `sample` of them, spread over the batch) with every candidate,
times each on the device (CUDA events, best of `reps`), and returns the
options with the fastest shape set (a copy of `opts`). Every candidate must
give the same flags as the default shape on the sample, or it is discarded.
Results are cached in memory and, if `cache` names a file, in that JSON file
keyed by network, GPU name, the solve options and the batch size class, so a
code that calls the solver every hydro step tunes once.
"""
import json
import os
from pathlib import Path

import numpy as np

from . import krome

# the shapes tried (layout, lane_minb, blocks_per_sm, queue_chunk)
CANDIDATES = (
    (1, 2, 0, 1), (1, 3, 0, 1), (1, 4, 0, 1), (1, 2, 1, 1), (1, 3, 1, 1),
    (0, 2, 0, 1), (0, 2, 0, 4),
)
KEYS = ("layout", "lane_minb", "blocks_per_sm", "queue_chunk")
# the options that change the work, part of the cache key
WORK_KEYS = ("evolve_T", "jac", "rtol", "atol_n", "atol_T", "lu32",
             "max_steps")

_memo = {}


def _size_class(ncell):
    return int(2 ** round(np.log2(max(ncell, 1))))


def cache_key(net, opts, ncell, gpu):
    work = ",".join("%s=%g" % (k, opts[k]) for k in WORK_KEYS)
    return "%s|%s|%s|%d" % (net.key, gpu, work, _size_class(ncell))


def _copy_opts(net, opts):
    o = net.options()
    for k in WORK_KEYS + KEYS + ("kernel", "clip_negative", "max_err_fails",
                                 "max_conv_fails", "max_restarts"):
        o[k] = opts[k]
    return o


def _sample(ncell, sample):
    if ncell <= sample:
        return np.arange(ncell)
    return np.linspace(0, ncell - 1, sample).round().astype(int)


def time_candidates(net, n, Tgas, dt, par, opts, candidates=CANDIDATES,
                    sample=16384, reps=2):
    """[(candidate, ms or None)] for each candidate on the sample (None:
    rejected, its flags differ from the default shape's)"""
    import torch
    dev = torch.device("cuda:0")
    idx = _sample(n.shape[0], sample)
    P = np.asarray(par, dtype=float)
    Ps = P[idx] if P.ndim == 2 else P
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64,
                               device=dev)
    n_s, T_s, dt_s, P_s = t(n[idx]), t(Tgas[idx]), t(dt[idx]), t(Ps)
    N = len(idx)

    def run(c):
        o = _copy_opts(net, opts)
        for k, v in zip(KEYS, c):
            o[k] = v
        o["kernel"] = 1
        best, flags = None, None
        for _ in range(reps):
            nd, Td = n_s.clone(), T_s.clone()
            fl = torch.zeros(N, dtype=torch.int32, device=dev)
            cur = torch.zeros(1, dtype=torch.int32, device=dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            net.solve_device(nd, Td, dt_s, P_s, fl, opts=o, cursor=cur)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
            flags = fl.cpu().numpy()
        return best, flags
    base_ms, base_flags = run(candidates[0])
    out = [(candidates[0], base_ms)]
    for c in candidates[1:]:
        ms, fl = run(c)
        out.append((c, ms if np.array_equal(fl, base_flags) else None))
    return out


def choose(timings):
    """the fastest accepted candidate"""
    ok = [(ms, c) for c, ms in timings if ms is not None]
    return min(ok)[1]


def tune(net, n, Tgas, dt, par, opts=None, cache=None, sample=16384,
         reps=2, candidates=CANDIDATES):
    """a copy of opts with the fastest launch shape for this batch"""
    import torch
    opts = net._options(opts)
    n = np.asarray(n, dtype=float)
    gpu = torch.cuda.get_device_name(0)
    key = cache_key(net, opts, n.shape[0], gpu)
    best = _memo.get(key)
    path = Path(cache) if cache else None
    if best is None and path is not None and path.exists():
        best = json.loads(path.read_text()).get(key)
    if best is None:
        timings = time_candidates(net, n, np.asarray(Tgas, float),
                                  np.asarray(dt, float), par, opts,
                                  candidates, sample, reps)
        best = list(choose(timings))
        if path is not None:
            data = json.loads(path.read_text()) if path.exists() else {}
            data[key] = best
            tmp = path.with_suffix(".tmp")
            tmp.write_text(json.dumps(data, indent=1))
            os.replace(tmp, path)
    _memo[key] = list(best)
    o = _copy_opts(net, opts)
    for k, v in zip(KEYS, best):
        o[k] = v
    return o
