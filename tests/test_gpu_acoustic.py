"""Acoustic media (CGFD_MEDIUM_ACOUSTIC_ISO, sv_curv_col_ac_iso_gpu.cu): the CUDA path through the
C ABI against the CPU oracle and against the reference's own acoustic solver code
(oracle/_ref/ref_harness).

Fields Vx Vy Vz P (P in the Txx slot); components 4-8 of every array stay exactly 0. Velocities
and pressure differ by orders of magnitude, so every bar is taken per group (velocities,
pressure). Tolerances as for the elastic path: random-state steps max |diff| <= 2e-5 x max |ref|
per component; seismograms and wavefields after 60-120 steps per-station / field relative L2
<= 1e-4 against the reference and the oracle (the oracle itself is within 2e-5 of the
reference); FP64 build against the FP64 oracle within float rounding of the read-back
(2e-7 x max |ref| per component).
"""
import os
import tempfile

import numpy as np
import pytest

from cgfd_b200 import Simulation, CgfdError, CGFD_PREC_FP64, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE
from oracle.oracle import Oracle, metric_fp32
from golden import ref_io
from golden.cases import golden_problem
from helpers import small_problem, random_wavefield, rel_l2, per_station_rel_l2

pytestmark = pytest.mark.gpu

V, P = slice(0, 3), slice(3, 4)
IN = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))  # physical points


def phys(w):
    """Physical points of a [9, nz, ny, nx] wavefield. The read-back returns ghosts as 0, while the
    oracle's and the reference's state keep the free-surface pressure image in the ghost planes."""
    return w[IN]


def _ac_wavefield(p, seed):
    w = random_wavefield(p, seed=seed)
    w[4:] = 0.0
    return w


def _compare_fields(w, ref, tol=2e-5):
    w, ref = phys(w), phys(ref)
    for c in range(9):
        scale = float(np.abs(ref[c]).max())
        err = float(np.abs(w[c] - ref[c]).max())
        assert err <= tol * max(scale, 1e-30), f"component {c}: max err {err:.3e} vs scale {scale:.3e}"
    assert not np.any(w[4:]), "components 4-8 of an acoustic wavefield must stay 0"


def _check_groups(s, r, w, wr, tol):
    w, wr = phys(w), phys(wr)
    assert np.abs(r[:, V]).max() > 0 and np.abs(r[:, P]).max() > 0
    assert per_station_rel_l2(s[:, V], r[:, V]) <= tol
    assert per_station_rel_l2(s[:, P], r[:, P]) <= tol
    assert rel_l2(w[V], wr[V]) <= tol
    assert rel_l2(w[P], wr[P]) <= tol
    assert not np.any(s[:, 4:]) and not np.any(w[4:])


@pytest.mark.parametrize("free_top", [1, 0])
@pytest.mark.parametrize("it0", [0, 3, 6])
def test_random_field_steps(free_top, it0):
    """Two steps from a smooth random state: every pair/stage direction, CFS-PML on every face,
    the free-surface pressure image and the low-order top rows."""
    p = small_problem("ac", nsrc=0, sta_grid=None, nsteps=12, free_top=free_top)
    w0 = _ac_wavefield(p, it0)
    sim, orc = Simulation(p), Oracle(p)
    sim.set_step(it0)
    orc.set_step(it0)
    sim.set_wavefield(w0)
    orc.set_wavefield(w0)
    for _ in range(2):
        sim.run(1)
        orc.run(1)
        _compare_fields(sim.wavefield(), orc.wavefield())


def test_seismograms_against_oracle():
    """Force and pressure sources, stations on the free surface, 80 steps."""
    p = small_problem("ac", nsteps=80, nsrc=2)
    sim, orc = Simulation(p), Oracle(p)
    sim.run()
    orc.run()
    _check_groups(sim.seismograms(), orc.seismograms(), sim.wavefield(), orc.wavefield(), 1e-4)
    for q in range(15):
        assert rel_l2(sim.peak_motion()[q], orc.peak_motion()[q]) <= 1e-4, q


@pytest.mark.skipif(not os.path.exists(ref_io.HARNESS), reason="oracle/_ref/ref_harness not built")
def test_oracle_and_product_match_reference():
    """The reference's own acoustic solver (sv_curv_col_ac_iso_onestage and its kernels, built
    unmodified) on the ac_small golden case."""
    p, nsteps = golden_problem("ac_small")
    with tempfile.TemporaryDirectory() as d:
        ref = ref_io.run(p, d, nsteps)
    assert rel_l2(metric_fp32(p.coord)[:, 3:-3, 3:-3, 3:-3], ref["metric"][:, 3:-3, 3:-3, 3:-3]) < 1e-6
    p.metric = ref["metric"]
    orc = Oracle(p)
    orc.run(nsteps)
    sim = Simulation(p)
    sim.run(nsteps)
    rs = ref["seismo"][:, :, :nsteps]
    _check_groups(orc.seismograms()[:, :, :nsteps], rs, orc.wavefield(), ref["wave"], 2e-5)
    _check_groups(sim.seismograms()[:, :, :nsteps], rs, sim.wavefield(), ref["wave"], 1e-4)
    for q in range(15):
        assert rel_l2(orc.peak_motion()[q], ref["pg"][q]) <= 2e-5, q
        assert rel_l2(sim.peak_motion()[q], ref["pg"][q]) <= 1e-4, q


@pytest.mark.skipif(not os.path.exists(ref_io.HARNESS), reason="oracle/_ref/ref_harness not built")
def test_long_run_with_interior_tiles_matches_reference():
    """600 steps on 96x88x64 (CFS-PML 10, free surface, two force + pressure sources, 25 stations
    3 grid points below the flat surface, where the pressure is 0): tiles without any PML face and
    z chunks below the top planes run. Stations and the pressure field stay within 1e-4 of the
    reference's own acoustic solver. By step 600 the velocity field has decayed ~230x from its
    peak and float rounding dominates it (the reference's own float run is ~2e-4 from the FP64
    build of the product): its bar is 3x the reference's distance from the FP64 build."""
    from oracle.oracle import metric_fp32 as mfp32
    p = small_problem("ac", ni=96, nj=88, nk=64, nsteps=600, npml=10, nsrc=2, sta_grid=(5, 5), seed=21)
    p.sta.loc[:, 2] = 3.0
    with tempfile.TemporaryDirectory() as d:
        ref = ref_io.run(p, d, 600, timeout=1200)
    assert rel_l2(mfp32(p.coord)[:, 3:-3, 3:-3, 3:-3], ref["metric"][:, 3:-3, 3:-3, 3:-3]) < 1e-6
    p.metric = ref["metric"]
    sim = Simulation(p)
    sim.run(600)
    p.precision = CGFD_PREC_FP64
    sim64 = Simulation(p)
    sim64.run(600)
    s, r = sim.seismograms()[:, :, :600], ref["seismo"][:, :, :600]
    w, wr, w64 = phys(sim.wavefield()), phys(ref["wave"]), phys(sim64.wavefield())
    assert np.abs(r[:, V]).max() > 0 and np.abs(r[:, P]).max() > 0
    assert per_station_rel_l2(s[:, V], r[:, V]) <= 1e-4
    assert per_station_rel_l2(s[:, P], r[:, P]) <= 1e-4
    assert rel_l2(w[P], wr[P]) <= 1e-4
    assert rel_l2(w[V], wr[V]) <= max(1e-4, 3.0 * rel_l2(wr[V], w64[V]))
    assert rel_l2(w64[P], wr[P]) <= 1e-4
    assert not np.any(s[:, 4:]) and not np.any(w[4:])


def test_zchunk_graph_and_batch_invariance():
    """z chunks, graph replay and batching change nothing (bitwise)."""
    p = small_problem("ac", nsteps=16, nk=40, nsrc=1)
    ref = Simulation(p)
    ref.run()
    for nzc in (3, 7, 64):
        s = Simulation(p)
        s.set_zchunk(nzc)
        s.set_graph_mode(nzc != 7)
        s.run()
        assert np.array_equal(s.wavefield(), ref.wavefield())
        assert np.array_equal(s.seismograms(), ref.seismograms())
    b = Simulation(p, shots=[p.src, p.src])
    b.run()
    for shot in range(2):
        assert np.array_equal(b.wavefield(shot), ref.wavefield())


def test_tma_and_direct_stage_kernels_agree():
    """The TMA-pipelined stage kernel (default) and the direct-load one: the same arithmetic on
    the same values, every direction pair, PML and free surface; 1e-6 x max |w| per component of
    the wavefield, 2e-5 per station (FMA contraction differs between the two compiled kernels)."""
    p = small_problem("ac", nsteps=20, nsrc=2, ni=70, nj=52, nk=44)
    a = Simulation(p)
    a.run()
    b = Simulation(p)
    b.set_bulk_variant(0)
    b.run()
    wa, wb = phys(a.wavefield()), phys(b.wavefield())
    for c in range(4):
        assert np.abs(wa[c] - wb[c]).max() <= 1e-6 * np.abs(wb[c]).max(), c
    assert per_station_rel_l2(a.seismograms()[:, :4], b.seismograms()[:, :4]) <= 2e-5


def test_fp64_build_matches_fp64_oracle():
    p = small_problem("ac", nsrc=0, sta_grid=None, nsteps=12)
    p.precision = CGFD_PREC_FP64
    w0 = _ac_wavefield(p, 5)
    sim, orc = Simulation(p), Oracle(p, fp64=True)
    sim.set_step(5)
    orc.set_step(5)
    sim.set_wavefield(w0)
    orc.set_wavefield(w0)
    sim.run(2)
    orc.run(2)
    # the read-back rounds to float: the bar is float rounding of the result
    _compare_fields(sim.wavefield(), orc.wavefield(), tol=2e-7)


def test_autotune_and_unsupported_modes():
    p = small_problem("ac", nsteps=12)
    s = Simulation(p)
    c = s.autotune(steps=2)
    assert 1 <= c <= p.nk
    s.run()
    ref = Simulation(p)
    ref.run()
    assert np.array_equal(s.wavefield(), ref.wavefield())
    for prec in (CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE):
        p.precision = prec
        with pytest.raises(CgfdError):
            Simulation(p)
