"""Parity of the benchmark's own workloads with the oracle.

* The batching workload as the benchmark runs it: primordial3 cells through
  the captured hydro step (krome_b200_graph_*: tff of the current state,
  densities x 1.01, dt = 0.01 tff, the persistent lane kernel), ten calls
  in a row on 4,096 cells of the benchmark's seeded batch. Each call is
  compared with the oracle solving the same inputs -- the state the graph
  started the call from, times 1.01 (an exact product on both sides), with
  the dt and tff the captured step wrote -- so every call is held to the
  parity bar on its own, at the noise floor of one call of the loop
  (tests/golden/noise_floor.py).
* Config 0 at its full size: 4,096 primordial cells with the analytic
  Jacobian, one solve."""
import numpy as np
import pytest

from conftest import assert_at_floor, parity
from krome_x_b200 import krome, netinfo, workloads
from oracle import Oracle

pytestmark = pytest.mark.gpu


def test_hydro_loop_matches_the_oracle_call_by_call():
    import torch
    key, ncell, calls = "primordial3", 4096, 10
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial3(ncell, info, seed=1000)
    o = workloads.OPTIONS[key]
    net = krome.load(key)
    # the benchmark's options: JAC_AUTO (difference quotients with Tgas
    # evolved), dense LU, the persistent lane-per-cell kernel
    opts = net.options(evolve_T=1, jac="auto", linsol="auto", rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"],
                       kernel="persistent", layout=1)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    n_d, T_d, dt_d, par_d = t(n), t(T), t(dt), t(par)
    fl = torch.zeros(ncell, dtype=torch.int32, device=dev)
    st = torch.zeros((ncell, 10), dtype=torch.int64, device=dev)
    g = net.hydro_graph(n_d, T_d, dt_d, par_d, fl, opts, stats=st)
    orc = Oracle(key)
    steps = []
    for c in range(calls):
        n0, T0 = n_d.cpu().numpy(), T_d.cpu().numpy()
        with torch.cuda.stream(g.stream):
            g.launch()
        torch.cuda.synchronize()
        ref = orc.solve(n0 * 1.01, T0, dt_d.cpu().numpy(), par_d.cpu().numpy(),
                        **o)
        m = parity(n_d.cpu().numpy(), T_d.cpu().numpy(), fl.cpu().numpy(),
                   ref["n"], ref["T"], ref["flags"], o["rtol"])
        assert_at_floor(m, "primordial3/hydro/4096/1000")
        # the same CVODE decisions: mean step counts within 3 %
        g_nst = st.cpu().numpy()[:, 0].mean()
        c_nst = ref["stats"][:, 0].mean()
        assert abs(g_nst - c_nst) <= 0.03 * c_nst + 0.5, (c, g_nst, c_nst)
        steps.append(g_nst)
    g.free()
    # the loop reaches the benchmark's steady state: later calls are short
    assert steps[-1] < steps[0]


def test_config0_full_batch_matches_the_oracle():
    key = "primordial"
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial(4096, info, seed=0)
    o = workloads.OPTIONS[key]
    assert o["jac"] == 1  # the analytic Jacobian of config 0
    net = krome.load(key)
    opts = net.options(evolve_T=o["evolve_T"], jac="analytic", linsol="dense",
                       rtol=o["rtol"], atol_n=o["atol_n"], atol_T=o["atol_T"])
    r = net.solve_batch(n, T, dt, par, opts=opts, check=False, stats=True)
    ref = Oracle(key).solve(n, T, dt, par, **o)
    m = parity(r.n, r.Tgas, r.flags, ref["n"], ref["T"], ref["flags"], o["rtol"])
    assert_at_floor(m, "primordial/config0/4096/0")
    g, c = r.stats.mean(axis=0), ref["stats"].mean(axis=0)
    for i in (0, 1, 3, 4, 5):  # nst nfe nje nsetups nni
        assert abs(g[i] - c[i]) <= 0.03 * c[i] + 0.5, (i, g, c)
