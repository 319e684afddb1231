"""Run-to-run determinism of the time loop: two simulations of the same problem must give
bitwise-identical wavefields and seismograms (tolerance: exact).

Every cell is written by exactly one thread per stage and the source injection of a single
source touches each point once, so nothing in the arithmetic is order-dependent; a difference
means a synchronisation fault. The grid (128 x 128 x 64, CFS-PML 10, free surface) gives each
column two z chunks of the bulk kernel and two resident blocks per SM, the setting in which a
shared-memory slot of the TMA ring was once refilled while a load of it was still in flight
(it showed up within 5-30 steps as small differences between repeated runs).
"""
import numpy as np
import pytest

from cgfd_b200 import Simulation, synth, CGFD_PREC_FP32, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE

pytestmark = pytest.mark.gpu


def _problem(medium):
    return synth.make_problem(128, 128, 64, 50.0, 120, dt=None, medium=medium, npml=10, nsrc=1, sta_grid=(4, 4),
                              fc=4.0, seed=41, src_depth=(1500.0, 1500.0), center_src=True)


@pytest.mark.parametrize("medium,precision", [("iso", CGFD_PREC_FP32), ("vti", CGFD_PREC_FP32),
                                              ("aniso", CGFD_PREC_FP32), ("vti", CGFD_PREC_U16_COEF),
                                              ("aniso", CGFD_PREC_FP16_WAVE)])
def test_repeated_runs_are_identical(medium, precision):
    p = _problem(medium)
    p.precision = precision
    out = []
    for _ in range(2):
        s = Simulation(p)
        s.run()
        out.append((s.wavefield(), s.seismograms()))
        s.close()
    assert np.abs(out[0][1]).max() > 0
    assert np.array_equal(out[0][0], out[1][0]), "final wavefields differ between identical runs"
    assert np.array_equal(out[0][1], out[1][1]), "seismograms differ between identical runs"


def test_repeated_batched_runs_are_identical():
    """A batch of 3 shots (shot-fastest block order, coefficient tiles shared through L2)."""
    p = _problem("vti")
    rng = np.random.default_rng(5)
    shots = [synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(800.0, 2000.0), fc_range=(3.0, 4.0),
                              stf_length=p.nt_total * p.dt) for _ in range(3)]
    out = []
    for _ in range(2):
        s = Simulation(p, shots=shots)
        s.run()
        out.append(s.seismograms())
        s.close()
    assert np.abs(out[0]).max() > 0
    assert np.array_equal(out[0], out[1]), "batched seismograms differ between identical runs"
