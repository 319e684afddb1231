"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on the same inputs.

Tolerances (FP32 both sides, different summation order and FMA contraction):
  - single/few-step random-wavefield updates: max |diff| <= 2e-5 * max |ref| per component
  - seismograms after tens of steps: per-station relative L2 <= 1e-4 (the path's bar)
"""
import numpy as np
import pytest

from cgfd_b200 import Simulation
from oracle.oracle import Oracle
from helpers import small_problem, random_wavefield, rel_l2, per_station_rel_l2

pytestmark = pytest.mark.gpu


def _compare_fields(w, ref, tol=2e-5):
    for c in range(9):
        scale = float(np.abs(ref[c]).max())
        err = float(np.abs(w[c] - ref[c]).max())
        assert err <= tol * max(scale, 1e-30), f"component {c}: max err {err:.3e} vs scale {scale:.3e}"


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
@pytest.mark.parametrize("it0", [0, 3, 6])
def test_random_field_steps(medium, it0):
    """Two steps from a smooth random state: every pair/stage direction, PML, free surface."""
    p = small_problem(medium, nsrc=0, sta_grid=None, nsteps=12)
    w0 = random_wavefield(p, seed=it0)
    sim = Simulation(p)
    sim.set_step(it0)
    sim.set_wavefield(w0)
    orc = Oracle(p)
    orc.set_step(it0)
    orc.set_wavefield(w0)
    for _ in range(2):
        sim.run(1)
        orc.run(1)
        _compare_fields(sim.wavefield(), orc.wavefield())


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_seismograms_small(medium):
    """Point source + stations over 60 steps: per-station rel L2 <= 1e-4."""
    p = small_problem(medium, nsteps=60)
    sim = Simulation(p)
    sim.run()
    orc = Oracle(p)
    orc.run()
    s, r = sim.seismograms(), orc.seismograms()
    assert s.shape == r.shape and s.shape[0] == 9
    assert np.abs(r).max() > 0
    assert per_station_rel_l2(s, r) <= 1e-4
    assert rel_l2(sim.wavefield(), orc.wavefield()) <= 1e-4


def test_no_free_surface_pml_top():
    """All six faces CFS-PML (no free surface): bulk kernel covers every plane."""
    p = small_problem("iso", free_top=0, nsrc=0, sta_grid=None, nsteps=4)
    w0 = random_wavefield(p, seed=11)
    sim, orc = Simulation(p), Oracle(p)
    sim.set_wavefield(w0)
    orc.set_wavefield(w0)
    sim.run(3)
    orc.run(3)
    _compare_fields(sim.wavefield(), orc.wavefield())


def test_graph_and_direct_launch_identical():
    p = small_problem("iso", nsteps=20)
    a = Simulation(p)
    a.run()
    b = Simulation(p)
    b.set_graph_mode(0)
    b.run()
    assert np.array_equal(a.seismograms(), b.seismograms())
    assert np.array_equal(a.wavefield(), b.wavefield())


def test_zchunk_invariance():
    """Results do not depend on the z-chunk of the bulk kernel (bitwise)."""
    p = small_problem("iso", nsteps=10, nk=40)
    ref = None
    for nzc in (3, 7, 64):
        s = Simulation(p)
        s.set_zchunk(nzc)
        s.run()
        w = s.wavefield()
        if ref is None:
            ref = w
        else:
            assert np.array_equal(w, ref)


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_tma_and_direct_bulk_variants_agree(medium):
    """The TMA-pipelined bulk kernel and the direct-load variant compute the same update."""
    p = small_problem(medium, nsteps=16, ni=70, nj=45, nk=33)
    a = Simulation(p)
    a.run()
    b = Simulation(p)
    b.set_bulk_variant(0)
    b.run()
    wa, wb = a.wavefield(), b.wavefield()
    for c in range(9):
        scale = float(np.abs(wb[c]).max())
        assert float(np.abs(wa[c] - wb[c]).max()) <= 1e-6 * max(scale, 1e-30)


@pytest.mark.parametrize("medium", ["iso", "aniso"])
def test_peak_motion_matches_oracle(medium):
    """Free-surface PGV/PGA/PGD (PG_calcu_gpu) over a point-source run, every component."""
    p = small_problem(medium, nsteps=60)
    sim, orc = Simulation(p), Oracle(p)
    sim.run()
    orc.run()
    a, b = sim.peak_motion(), orc.peak_motion()
    assert a.shape == (15, p.nj + 6, p.ni + 6)
    for q in range(15):
        assert np.abs(b[q]).max() > 0
        assert rel_l2(a[q], b[q]) <= 1e-4, q
    assert not a[:, :3].any() and not a[:, :, :3].any()  # ghost points stay 0


def test_peak_motion_needs_free_surface():
    from cgfd_b200 import CgfdError
    p = small_problem("iso", free_top=0, nsrc=0, sta_grid=None, nsteps=4)
    sim = Simulation(p)
    with pytest.raises(CgfdError) as e:
        sim.peak_motion()
    assert e.value.code == -5


@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_tile_shapes_agree(medium):
    """The two tile shapes of the TMA bulk kernel (cgfd_set_tile_shape) compute the same update:
    the same per-cell arithmetic on a different thread-block tiling (within 1e-6 of the
    per-component maximum: the compiler may contract multiply-adds differently per
    instantiation)."""
    p = small_problem(medium, nsteps=16, ni=70, nj=45, nk=33)
    a = Simulation(p)
    a.set_tile_shape(0)
    assert a.tile_shape == 0
    a.run()
    b = Simulation(p)
    b.set_tile_shape(1)
    assert b.tile_shape == 1
    b.run()
    wa, wb = a.wavefield(), b.wavefield()
    assert np.abs(wa).max() > 0
    for c in range(9):
        scale = float(np.abs(wa[c]).max())
        assert float(np.abs(wa[c] - wb[c]).max()) <= 1e-6 * max(scale, 1e-30), c
    sa, sb = a.seismograms(), b.seismograms()
    assert per_station_rel_l2(sb, sa) <= 1e-6


def test_autotune_picks_a_chunk_and_resets_state():
    """cgfd_autotune times the tile-shape and z-chunk candidates on the problem itself, keeps the
    fastest pair and returns the problem to step 0 with a zero wavefield: the following run
    equals a run of a fresh problem (bitwise when the default shape won)."""
    p = small_problem("iso", nsteps=30)
    a = Simulation(p)
    default_chunk = a.zchunk
    c = a.autotune(2)  # both tile shapes x the z-chunk candidates, and the default tiling
    assert c in (8, 10, 12, 14, 16, 20, 24, 32, 48, 64, 96, p.nk - 4, default_chunk)
    assert a.zchunk == c and a.step == 0
    assert a.tile_shape in (0, 1)
    a.run()
    b = Simulation(p)
    b.run()
    if a.tile_shape == b.tile_shape:  # results do not depend on the chunk length (bitwise)
        assert np.array_equal(a.seismograms(), b.seismograms())
        assert np.array_equal(a.wavefield(), b.wavefield())
    else:  # nor on the tile shape (up to multiply-add contraction)
        assert per_station_rel_l2(a.seismograms(), b.seismograms()) <= 1e-6
    with pytest.raises(Exception):
        a.autotune(2)  # only before the first step
