"""Batched sources on one grid (cgfd_batch_create): each shot of a batch equals the same
source run alone (bitwise: identical arithmetic per shot), and the oracle within 1e-4."""
import numpy as np
import pytest

from cgfd_b200 import Simulation, synth
from oracle.oracle import Oracle
from helpers import small_problem, per_station_rel_l2

pytestmark = pytest.mark.gpu


def _shots(p, n, seed):
    rng = np.random.default_rng(seed)
    return [synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(600.0, 1200.0), fc_range=(2.5, 4.0),
                             stf_length=p.nt_total * p.dt) for _ in range(n)]


@pytest.mark.parametrize("medium", ["iso", "aniso"])
def test_batch_equals_individual_runs(medium):
    p = small_problem(medium, nsteps=40, nsrc=0)
    shots = _shots(p, 3, 5)
    b = Simulation(p, shots=shots)
    b.run()
    bs = b.seismograms()
    assert bs.shape == (3, 9, 9, p.nt_total)
    for n, s in enumerate(shots):
        p.src = s
        one = Simulation(p)
        one.run()
        assert np.array_equal(one.seismograms(), bs[n])
        assert np.array_equal(one.wavefield(), b.wavefield(n))
    # shot 1 against the oracle
    p.src = shots[1]
    o = Oracle(p)
    o.run()
    assert per_station_rel_l2(bs[1], o.seismograms()) <= 1e-4


def test_batch_validation():
    p = small_problem("iso", nsteps=4, nsrc=0)
    shots = _shots(p, 2, 1)
    s = Simulation(p, shots=shots)
    with pytest.raises(Exception):
        s.set_bulk_variant(0)


def test_shot_groups_agree_and_autotune_picks_one():
    """The block order of a batch (shot groups of 1, 2 or every shot; strips of tile rows
    sized by the group) changes no result: every group gives the same seismograms and final
    wavefields bitwise. The autotuner then picks a group and returns the batch to step 0."""
    p = small_problem("iso", nsteps=30, nsrc=0)
    shots = _shots(p, 5, 9)
    ref = None
    for g in (5, 1, 2):
        b = Simulation(p, shots=shots)
        b.set_shot_group(g)
        assert b.shot_group == g
        b.run()
        out = (b.seismograms(), [b.wavefield(n) for n in range(5)])
        b.close()
        if ref is None:
            ref = out
        else:
            assert np.array_equal(out[0], ref[0])
            for n in range(5):
                assert np.array_equal(out[1][n], ref[1][n])
    b = Simulation(p, shots=shots)
    b.autotune(2)
    assert b.shot_group in (4, 5)
    assert b.step == 0
    b.run()
    assert np.array_equal(b.seismograms(), ref[0])
    b.close()
