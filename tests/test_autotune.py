"""The launch-shape autotuner (krome_x_b200.autotune)."""
import json

import numpy as np
import pytest

from conftest import parity
from krome_x_b200 import autotune, krome, netinfo, workloads


def test_choose_takes_the_fastest_accepted_shape():
    t = [((1, 2, 0, 1), 10.0), ((1, 3, 0, 1), 7.0), ((1, 4, 0, 1), None),
         ((0, 2, 0, 1), 9.0)]
    assert autotune.choose(t) == (1, 3, 0, 1)
    # a rejected shape never wins, however fast it was
    t[2] = ((1, 4, 0, 1), None)
    assert autotune.choose(t) != (1, 4, 0, 1)


def test_cache_key_covers_the_work_options_and_the_batch_size_class():
    net = krome.load("primordial3")
    a = net.options(rtol=1e-6)
    b = net.options(rtol=1e-8)
    k = lambda o, nc: autotune.cache_key(net, o, nc, "B200")
    assert k(a, 100000) != k(b, 100000)
    assert k(a, 100000) == k(a, 120000)      # same power-of-two class
    assert k(a, 100000) != k(a, 1000)
    # the launch shape itself is not part of the key
    c = net.options(rtol=1e-6, lane_minb=4)
    assert k(a, 100000) == k(c, 100000)


def test_sample_spreads_over_the_batch():
    s = autotune._sample(1000, 10)
    assert len(s) == 10 and s[0] == 0 and s[-1] == 999
    assert (np.diff(s) > 0).all()
    np.testing.assert_array_equal(autotune._sample(5, 10), np.arange(5))


@pytest.mark.gpu
def test_tuned_shape_solves_like_the_default(tmp_path, monkeypatch):
    key = "primordial3"
    info = netinfo.load(key)
    n, T, dt, par = workloads.primordial3(8192, info, seed=17)
    net = krome.load(key)
    o = workloads.OPTIONS[key]
    opts = net.options(evolve_T=o["evolve_T"], jac=o["jac"], rtol=o["rtol"],
                       atol_n=o["atol_n"], atol_T=o["atol_T"])
    cache = tmp_path / "tune.json"
    tuned = autotune.tune(net, n, T, dt, par, opts, cache=str(cache),
                          sample=4096)
    entry = json.loads(cache.read_text())
    assert len(entry) == 1
    shape = tuple(int(tuned[k]) for k in autotune.KEYS)
    assert shape in autotune.CANDIDATES
    a = net.solve_batch(n, T, dt, par, opts=opts, check=False)
    b = net.solve_batch(n, T, dt, par, opts=tuned, check=False)
    m = parity(b.n, b.Tgas, b.flags, a.n, a.Tgas, a.flags, o["rtol"])
    assert m["flags_equal"] == 1.0 and m["frac"] >= 0.95, m
    # a second tuning of the same kind of batch reads the cache
    autotune._memo.clear()
    monkeypatch.setattr(autotune, "time_candidates",
                        lambda *a, **k: pytest.fail("re-timed"))
    again = autotune.tune(net, n, T, dt, par, opts, cache=str(cache),
                          sample=4096)
    assert tuple(int(again[k]) for k in autotune.KEYS) == shape
