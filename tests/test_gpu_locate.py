"""Sources and stations given by physical coordinates (loc_coord_type 1, flag_coord 1): the
product's device location (nearest grid point, containing cell, 101^3 sampling; depth below
the free surface converted through the top quads) against the oracle's restatement and the
reference's own location code run on the same GPU (oracle/_ref/ref_harness).
Bars: located indices equal; per-station relative L2 of the seismograms <= 1e-4."""
import dataclasses
import os
import tempfile

import numpy as np
import pytest

from cgfd_b200 import Simulation
from cgfd_b200.abi import Stations
from oracle.oracle import Oracle, locate_points
from golden import ref_io
from helpers import small_problem, per_station_rel_l2

pytestmark = pytest.mark.gpu


def trilinear(coord, i0, j0, k0, f):
    out = np.zeros(3)
    for kk in (0, 1):
        for jj in (0, 1):
            for ii in (0, 1):
                w = (f[0] if ii else 1 - f[0]) * (f[1] if jj else 1 - f[1]) * (f[2] if kk else 1 - f[2])
                out += w * coord[:, k0 + 3 + kk, j0 + 3 + jj, i0 + 3 + ii]
    return out


def coordinate_problem(medium="iso", seed=0):
    p = small_problem(medium, nsteps=60, nsrc=1)
    rng = np.random.default_rng(seed)
    c = p.coord
    # the source at a random point of an interior cell, by (x, y, z)
    i0, j0, k0 = p.src.loc[0].astype(int)
    xyz = trilinear(c, int(i0), int(j0), int(k0), rng.uniform(0.05, 0.95, 3)).astype(np.float32)
    src = dataclasses.replace(p.src, loc=xyz[None, :], loc_coord_type=1, loc_3dim=0)
    # stations: 5 on the free surface by (x, y, depth 0), 3 buried by (x, y, z)
    loc, fd = [], []
    for n in range(5):
        i, j = rng.integers(8, p.ni - 9), rng.integers(8, p.nj - 9)
        f = rng.uniform(0.1, 0.9, 2)
        top = trilinear(c, i, j, p.nk - 2, (f[0], f[1], 1.0))
        loc.append([top[0], top[1], 0.0]); fd.append(1)
    for n in range(3):
        i, j, k = rng.integers(8, p.ni - 9), rng.integers(8, p.nj - 9), rng.integers(5, p.nk - 6)
        loc.append(trilinear(c, i, j, k, rng.uniform(0.1, 0.9, 3))); fd.append(0)
    sta = Stations(loc=np.array(loc, np.float32), flag_depth=np.array(fd, np.int32),
                   flag_coord=np.ones(len(loc), np.int32), names=[f"c{n}" for n in range(len(loc))])
    return dataclasses.replace(p, src=src, sta=sta)


@pytest.mark.parametrize("medium", ["iso", "vti"])
def test_coordinate_location_matches_oracle(medium):
    p = coordinate_problem(medium, seed=3)
    sim, orc = Simulation(p), Oracle(p)
    sim.run()
    orc.run()
    s, r = sim.seismograms(), orc.seismograms()
    assert s.shape == r.shape and s.shape[0] == 8
    assert per_station_rel_l2(s, r) <= 1e-4
    # the stations' located cells agree with the oracle's location
    idx, inc = locate_points(p.coord, p.sta.loc, p.sta.flag_depth)
    idx = idx.copy()
    idx[inc < 0] -= 1
    import ctypes as C
    from cgfd_b200 import lib
    ijk = np.zeros((8, 3), np.int32)
    ii = np.zeros(8, np.int32)
    assert lib().cgfd_station_info(sim.h, ii.ctypes.data, ijk.ctypes.data) == 0
    assert np.array_equal(ijk, idx[ii])


@pytest.mark.skipif(not os.path.exists(ref_io.HARNESS), reason="oracle/_ref/ref_harness not built")
def test_coordinate_location_matches_reference():
    p = coordinate_problem("iso", seed=5)
    with tempfile.TemporaryDirectory() as d:
        ref = ref_io.run(p, d, 60)
    p.metric = ref["metric"]
    sim = Simulation(p)
    sim.run(60)
    rs = ref["seismo"][:, :, :60]
    assert rs.shape[0] == 8 and np.abs(rs).max() > 0
    assert per_station_rel_l2(sim.seismograms()[:, :, :60], rs) <= 1e-4
