"""The FP64 build of the kernels (CGFD_PREC_FP64: wavefield, coefficients, PML auxiliaries and
arithmetic in double, direct-load bulk kernel) against the FP64 oracle (the CPU restatement
instantiated in double) on the same inputs.

Both take the same float inputs (metrics, medium). The FP64 build also takes the library's
float setup tables (source time function samples, smoothing weights, CFS-PML profiles,
free-surface matrices, station weights: the reference computes and stores them in float),
while the FP64 oracle rebuilds some of them in double, so the two differ by those tables'
float rounding: per-station relative L2 <= 2e-6 (bar written here), far below the FP32
path's own distance from FP64 (1e-6 .. 1e-5) and the 16-bit modes' (1e-5 .. 1e-3). The
second test checks the FP64 build as the reference of the precision study: the FP32 path's
error measured against it equals its error against the FP64 oracle.
"""
import numpy as np
import pytest

from cgfd_b200 import Simulation, CgfdError, CGFD_PREC_FP32, CGFD_PREC_FP64, CGFD_PREC_U16_COEF
from oracle.oracle import Oracle
from helpers import small_problem, random_wavefield, rel_l2, per_station_rel_l2

pytestmark = pytest.mark.gpu


def _problem(medium, **kw):
    return small_problem(medium, ni=56, nj=52, nk=40, nsteps=240, npml=8, sta_grid=(4, 4), seed=7, **kw)


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_fp64_build_matches_fp64_oracle(medium):
    p = _problem(medium)
    orc = Oracle(p, fp64=True)
    orc.run()
    ref = orc.seismograms()
    p.precision = CGFD_PREC_FP64
    sim = Simulation(p)
    sim.run()
    s = sim.seismograms()
    assert np.abs(ref).max() > 0
    assert per_station_rel_l2(s, ref) <= 2e-6
    assert rel_l2(sim.wavefield(), orc.wavefield()) <= 2e-6
    pg = sim.peak_motion()
    for q in range(15):
        assert rel_l2(pg[q], orc.peak_motion()[q]) <= 2e-6, q


@pytest.mark.parametrize("medium", ["iso", "aniso"])
def test_fp64_build_two_steps_from_random_state(medium):
    """Every pair direction of one step in double, PML and free surface: the update agrees with
    the FP64 oracle to double rounding (max |diff| <= 1e-12 x max |ref| per component)."""
    p = small_problem(medium, nsrc=0, sta_grid=None, nsteps=12)
    p.precision = CGFD_PREC_FP64
    w0 = random_wavefield(p, seed=3)
    sim = Simulation(p)
    sim.set_step(3)
    sim.set_wavefield(w0)
    orc = Oracle(p, fp64=True)
    orc.set_step(3)
    orc.set_wavefield(w0)
    sim.run(2)
    orc.run(2)
    w, r = sim.wavefield(), orc.wavefield()
    for c in range(9):
        scale = float(np.abs(r[c]).max())
        # the read-back rounds to float: the bar is float rounding of the result
        assert float(np.abs(w[c] - r[c]).max()) <= 2e-7 * scale, c


def test_fp64_build_is_the_precision_reference():
    p = _problem("vti")
    orc = Oracle(p, fp64=True)
    orc.run()
    ref_orc = orc.seismograms()
    p.precision = CGFD_PREC_FP64
    s64 = Simulation(p)
    s64.run()
    ref_gpu = s64.seismograms()
    for prec in (CGFD_PREC_FP32, CGFD_PREC_U16_COEF):
        p.precision = prec
        sim = Simulation(p)
        sim.run()
        s = sim.seismograms()
        e_orc, e_gpu = rel_l2(s, ref_orc), rel_l2(s, ref_gpu)
        assert abs(e_orc - e_gpu) <= 0.1 * e_orc + 2e-7, (prec, e_orc, e_gpu)


def test_fp64_build_runs_the_direct_kernel_only():
    p = _problem("iso")
    p.precision = CGFD_PREC_FP64
    sim = Simulation(p)
    with pytest.raises(CgfdError) as e:
        sim.set_bulk_variant(1)
    assert e.value.code == -5
    assert sim.device_bytes() == __import__("cgfd_b200").problem_bytes(p)[0]
