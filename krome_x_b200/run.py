"""Run one solve of a benchmark workload from the command line.

    python -m krome_x_b200.run primordial3 65536 [--layout lane|warp]
        [--kernel persistent|plain] [--seed 5] [--calls 1] [--lu32]
    python -m krome_x_b200.run primordial 8192 --adjoint
    python -m krome_x_b200.run semenov 148 --dt 3.15e9

Draws the seeded workload (krome_x_b200.workloads), solves it through the
C ABI (krome_b200_solve_batch) and prints the elapsed time, the cell-solves
per second and the failed cells; with --calls > 1 it runs that many steps
of the collapse driver's hydro loop on the host arrays. With --adjoint it
runs the discrete adjoint through the torch.autograd wrapper instead (the
recording forward solve and the reverse sweep, gradients of sum(n_H2) +
sum(Tgas)). --dt replaces every cell's time step (a shorter solve of the
same cells, e.g. to profile the large networks' kernel). Used to profile a single kernel launch (ncu -k ... python -m
krome_x_b200.run ...).
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
    ap.add_argument("--lu32", action="store_true")
    ap.add_argument("--adjoint", action="store_true")
    ap.add_argument("--dt", type=float, default=None)
    a = ap.parse_args(argv)
    info = netinfo.load(a.network)
    n, T, dt, par = workloads.GENERATORS[a.network](a.cells, info, seed=a.seed)
    if a.dt is not None:
        dt[:] = a.dt
    o = workloads.OPTIONS[a.network]
    net = krome.load(a.network)
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel=a.kernel, layout=0 if a.layout == "warp" else 1,
                       lane_minb=a.lane_minb, lu32=int(a.lu32),
                       max_steps=o.get("max_steps", 100000))
    if a.adjoint:
        return adjoint(a, net, opts, info, n, T, dt, par)
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


def adjoint(a, net, opts, info, n, T, dt, par):
    import torch
    from . import autograd
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
    t2 = time.perf_counter()
    print("%s %d cells adjoint: forward %.3f s, reverse sweep %.3f s, "
          "failed %d, finite gradients %s"
          % (a.network, a.cells, t1 - t0, t2 - t1, int((flags != 0).sum()),
             bool(torch.isfinite(m.grad).all())))


if __name__ == "__main__":
    main()
