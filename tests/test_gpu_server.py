"""Serving loop (cgfd_server_*): continuous admission by HBM budget, same-grid batching,
overlapping problems of different grids and media, p50/p99 latency.

Tolerance of the alone-vs-mix check: 0 (bitwise). A request computes the same arithmetic
whether it runs alone, as one shot of a same-grid batch or beside other problems on other
streams, so its seismograms must be identical.
"""
import dataclasses
import time

import numpy as np
import pytest

from cgfd_b200 import Simulation, Server, problem_bytes, synth, CgfdError, CGFD_PREC_FP16_WAVE, CGFD_PREC_U16_COEF
from helpers import small_problem

pytestmark = pytest.mark.gpu


def _with_sources(p, seed, n=1):
    rng = np.random.default_rng(seed)
    src = synth.dc_sources(p.coord, p.ni, p.nj, n, rng, depth_range=(600.0, 1200.0), fc_range=(2.5, 4.0),
                           stf_length=p.nt_total * p.dt)
    return dataclasses.replace(p, src=src)


def _solo(p):
    s = Simulation(p)
    s.run()
    out = s.seismograms()
    s.close()
    return out


@pytest.mark.parametrize("medium,precision,nshot", [("iso", 0, 1), ("vti", 0, 3), ("aniso", CGFD_PREC_U16_COEF, 2),
                                                     ("iso", CGFD_PREC_FP16_WAVE, 2)])
def test_problem_bytes_matches_device(medium, precision, nshot):
    p = small_problem(medium, nsteps=10, nsrc=0)
    p.precision = precision
    shots = [_with_sources(p, 10 + n).src for n in range(nshot)]
    resident, peak = problem_bytes(p, shots)
    sim = Simulation(p, shots=shots)
    assert sim.device_bytes() == resident
    assert peak >= resident


def test_alone_equals_in_mix():
    base_a = small_problem("iso", ni=48, nj=44, nk=36, nsteps=90, nsrc=0, seed=1)
    base_b = small_problem("vti", ni=40, nj=36, nk=30, nsteps=70, nsrc=0, seed=2)
    base_c = small_problem("aniso", ni=36, nj=40, nk=30, nsteps=60, nsrc=0, seed=3)
    base_c.precision = CGFD_PREC_FP16_WAVE
    reqs = [_with_sources(base_a, 100), _with_sources(base_a, 101), _with_sources(base_b, 102),
            _with_sources(base_c, 103), _with_sources(base_a, 104, n=2), _with_sources(base_b, 105)]
    late = [_with_sources(base_a, 106), _with_sources(base_c, 107)]
    alone = [_solo(p) for p in reqs + late]

    with Server(max_active=3, max_batch=2, steps_per_slice=7) as srv:
        ids = [srv.submit(p) for p in reqs]
        # the late requests arrive while the first ones are on the device
        t0 = time.time()
        while srv.stats()["active"] == 0 and time.time() - t0 < 60:
            time.sleep(0.002)
        assert srv.stats()["active"] > 0
        ids += [srv.submit(p) for p in late]
        res = [srv.wait(i, timeout=300) for i in ids]
        st = srv.stats()
    for n, (a, r) in enumerate(zip(alone, res)):
        assert r is not None and r.shape == a.shape, n
        assert np.array_equal(a, r), f"request {n}: max diff {np.abs(a - r).max()}"
    assert st["completed"] == len(ids) and st["failed"] == 0
    assert st["batches"] < len(ids)  # same-grid requests shared batches
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    assert st["cell_stages_per_s"] > 0 and st["hbm_peak"] <= st["hbm_budget"]
    assert st["hbm_in_use"] == 0


def test_hbm_budget_admission():
    """A budget that fits one request at a time: requests run one after another, a request
    larger than the budget fails with CGFD_ERR_NOMEM and the others still complete."""
    small = small_problem("iso", nsteps=30, nsrc=0, seed=4)
    big = small_problem("iso", ni=64, nj=64, nk=48, nsteps=30, nsrc=0, seed=5)
    r1, r2 = _with_sources(small, 200), _with_sources(small, 201)
    rb = _with_sources(big, 202)
    _, peak = problem_bytes(r1)
    _, peak_big = problem_bytes(rb)
    assert peak_big > int(peak * 1.5)
    with Server(hbm_budget=int(peak * 1.5), max_active=4, max_batch=1) as srv:
        i1, ib, i2 = srv.submit(r1), srv.submit(rb), srv.submit(r2)
        a = srv.wait(i1, timeout=120)
        with pytest.raises(CgfdError) as e:
            srv.wait(ib, timeout=120)
        assert e.value.code == -3
        b = srv.wait(i2, timeout=120)
        st = srv.stats()
    assert np.array_equal(a, _solo(r1)) and np.array_equal(b, _solo(r2))
    assert st["completed"] == 2 and st["failed"] == 1
    assert st["hbm_peak"] <= int(peak * 1.5)
