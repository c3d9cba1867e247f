"""Run one solve of a benchmark workload from the command line.

    python -m krome_x_b200.run primordial3 65536 [--layout lane|warp]
        [--kernel persistent|plain] [--seed 5] [--calls 1]

Draws the seeded workload (krome_x_b200.workloads), solves it through the
C ABI (krome_b200_solve_batch) and prints the elapsed time, the cell-solves
per second and the failed cells; with --calls > 1 it runs that many steps
of the collapse driver's hydro loop on the host arrays. Used to profile a
single kernel launch (ncu -k ... python -m krome_x_b200.run ...).
"""
import argparse
import time

from . import krome, netinfo, workloads


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("network")
    ap.add_argument("cells", type=int)
    ap.add_argument("--layout", default="lane", choices=["lane", "warp"])
    ap.add_argument("--kernel", default="persistent",
                    choices=["persistent", "plain"])
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--calls", type=int, default=1)
    ap.add_argument("--lane-minb", type=int, default=2)
    a = ap.parse_args(argv)
    info = netinfo.load(a.network)
    n, T, dt, par = workloads.GENERATORS[a.network](a.cells, info, seed=a.seed)
    o = workloads.OPTIONS[a.network]
    net = krome.load(a.network)
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel=a.kernel, layout=0 if a.layout == "warp" else 1,
                       lane_minb=a.lane_minb)
    failed = 0
    t0 = time.perf_counter()
    for c in range(a.calls):
        if c > 0:
            dt = workloads.hydro_step_info(n, par, info)
        r = net.solve_batch(n, T, dt, par, opts=opts, check=False)
        n, T = r.n, r.Tgas
        failed += int((r.flags != 0).sum())
    el = time.perf_counter() - t0
    print("%s %d cells x %d calls: %.3f s, %.0f cell-solves/s, failed %d"
          % (a.network, a.cells, a.calls, el, a.cells * a.calls / el, failed))


if __name__ == "__main__":
    main()
