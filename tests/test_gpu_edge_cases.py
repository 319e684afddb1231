"""Edge cases of the time loop against the oracle, through the C ABI.

Tolerances (FP32 both sides, different summation order and FMA contraction):
  - random-state steps: max |diff| <= 2e-5 x max |ref| per component
  - runs with sources: per-station relative L2 <= 1e-4, wavefield relative L2 <= 1e-4

Covered: grids smaller than one 32 x 8 tile and ragged in every direction (down to the
8-point minimum, which is also the minimum depth of the 4-plane free-surface slab), CFS-PML
on some faces only or none and thick PML, force sources (cmp_type 1) and the reference's
cmp_type 3 = force-only reading (src_t.cu:437-441), moment tensors given directly
(mechanism_type 0), every wavelet (src_t.cu:873-903), sampled source time functions
(stf_given 1, Lagrange-interpolated at the global step, src_t.cu:683), sources whose 7^3
smoothing stencil the grid edge clips, overlapping sources, sources outside the grid, stations
on edges and corners (io_funcs.cu:1624-1666), and a batch mixing force and moment shots.
"""
import dataclasses

import numpy as np
import pytest

from cgfd_b200 import Simulation, synth, WAVELETS
from cgfd_b200.abi import Sources, Stations
from oracle.oracle import Oracle
from helpers import small_problem, random_wavefield, rel_l2, per_station_rel_l2

pytestmark = pytest.mark.gpu


def _compare_fields(w, ref, tol=2e-5):
    for c in range(9):
        scale = float(np.abs(ref[c]).max())
        err = float(np.abs(w[c] - ref[c]).max())
        assert err <= tol * max(scale, 1e-30), f"component {c}: max err {err:.3e} vs scale {scale:.3e}"


def _steps_vs_oracle(p, nsteps=3, seed=0, it0=0):
    w0 = random_wavefield(p, seed=seed)
    sim, orc = Simulation(p), Oracle(p)
    for x in (sim, orc):
        x.set_step(it0)
        x.set_wavefield(w0)
    for _ in range(nsteps):
        sim.run(1)
        orc.run(1)
        _compare_fields(sim.wavefield(), orc.wavefield())


def _compare_run(p):
    sim, orc = Simulation(p), Oracle(p)
    sim.run()
    orc.run()
    s, r = sim.seismograms(), orc.seismograms()
    assert s.shape == r.shape
    assert np.isfinite(s).all()
    assert np.abs(r).max() > 0
    assert per_station_rel_l2(s, r) <= 1e-4
    assert rel_l2(sim.wavefield(), orc.wavefield()) <= 1e-4
    return s


def _sources(locs, cmp_type=2, wavelet="ricker", fc=4.0, stf_len=None, stf_given=0, dt=0.01, nt=40,
             seed=0, mechanism_type=0, t_start=0.0):
    """Sources at 0-based grid indices (z = grid index, loc_3dim 0) with seeded components."""
    rng = np.random.default_rng(seed)
    n = len(locs)
    loc = np.asarray(locs, np.float32).reshape(n, 3)
    cmp = np.zeros((n, 9), np.float32)
    cmp[:, 0:3] = rng.uniform(-1, 1, (n, 3)) * 1e12
    cmp[:, 3:9] = rng.uniform(-1, 1, (n, 6)) * 1e16
    coefs = np.zeros((n, 10), np.float32)
    coefs[:, 0] = fc
    coefs[:, 1] = 1.2 / fc
    if wavelet in ("gaussian", "gaussian_deriv"):
        coefs[:, 0] = 0.25 / fc  # a: the Gaussian width (s)
        coefs[:, 1] = 1.0 / fc
    src = Sources(loc=loc, t_start=np.full(n, t_start, np.float32), cmp_type=cmp_type,
                  mechanism_type=mechanism_type, loc_coord_type=0, loc_3dim=0)
    if stf_given == 0:
        src.wavelet = np.full(n, WAVELETS[wavelet], np.int32)
        src.wavelet_coefs = coefs
        src.cmp = cmp
        src.stf_length = float(stf_len)
    else:
        sdt = dt * 0.7  # not a multiple of the time step: the interpolation matters
        t = np.arange(nt) * sdt
        u = (t - 1.2 / fc) * 2 * np.pi * fc
        ricker = (1 - u * u / 2) * np.exp(-u * u / 4)
        vals = ricker[None, :, None] * cmp[:, None, :]
        src.stf_given, src.stf_dt, src.stf_nt = 1, float(sdt), int(nt)
        src.cmp_values = np.ascontiguousarray(vals, np.float32)
    return src


def _stations(ni, nj, nk):
    """Corners and edges of the top plane (depth 0), a fractional edge point, and buried
    stations at the bottom plane and at a side face (1-based index, flag_depth 0)."""
    loc = [(1, 1, 0), (ni, 1, 0), (1, nj, 0), (ni, nj, 0), (ni - 0.5, (nj + 1) / 2, 0.0),
           ((ni + 1) / 2, 1.25, 0.0), ((ni + 1) / 2, (nj + 1) / 2, 1.0), (1, (nj + 1) / 2, nk / 2 + 0.3)]
    flag_depth = [1, 1, 1, 1, 1, 1, 0, 0]
    return Stations(loc=np.asarray(loc, np.float32), flag_depth=np.asarray(flag_depth, np.int32),
                    names=[f"e{n}" for n in range(len(loc))])


# ---- grids -----------------------------------------------------------------------------

@pytest.mark.parametrize("shape", [(13, 8, 9), (20, 11, 8), (33, 9, 12), (40, 17, 10)])
@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_ragged_small_grids(shape, medium):
    """Grids below one tile, ragged in x, y and z, with free surface and 2-layer PML."""
    ni, nj, nk = shape
    p = small_problem(medium, ni=ni, nj=nj, nk=nk, npml=2, nsrc=0, sta_grid=None, nsteps=6)
    _steps_vs_oracle(p, nsteps=3, seed=sum(shape))


@pytest.mark.parametrize("shape", [(8, 8, 8), (37, 10, 8)])
def test_minimum_grid_no_free_surface(shape):
    """The 8-point minimum with PML on all six faces (no free surface)."""
    ni, nj, nk = shape
    p = small_problem("iso", ni=ni, nj=nj, nk=nk, npml=2, free_top=0, nsrc=0, sta_grid=None, nsteps=6)
    _steps_vs_oracle(p, nsteps=3, seed=3)


# ---- partial CFS-PML ---------------------------------------------------------------------

def _pml_faces(p, faces, n):
    f = synth.pml_all(n, ref_vel=6500.0)[0][0]
    pml = [[None, None], [None, None], [None, None]]
    for a, side in faces:
        pml[a][side] = dict(f)
    p.pml = pml
    return p


@pytest.mark.parametrize("faces,free_top", [
    ((), 1),                                   # no PML at all
    (((0, 0), (0, 1)), 1),                     # x faces only
    (((0, 1),), 1),                            # one x face
    (((1, 0), (2, 0)), 1),                     # y0 and the bottom
    (((2, 0),), 1),                            # bottom only
    (((2, 1),), 0),                            # top PML only, no free surface
    (((0, 0), (1, 1), (2, 0), (2, 1)), 0),     # mixed, top PML
])
@pytest.mark.parametrize("medium", ["iso", "aniso"])
def test_partial_pml(faces, free_top, medium):
    p = small_problem(medium, ni=44, nj=38, nk=30, npml=6, free_top=free_top, nsrc=0, sta_grid=None, nsteps=6)
    _pml_faces(p, faces, 6)
    _steps_vs_oracle(p, nsteps=3, seed=len(faces) + 7 * free_top)


def test_thick_pml():
    """14-layer PML on a 40 x 36 x 30 grid: most tiles are PML tiles, the interior is thin."""
    p = small_problem("vti", ni=40, nj=36, nk=30, npml=14, nsrc=0, sta_grid=None, nsteps=6)
    _steps_vs_oracle(p, nsteps=3, seed=14)


# ---- sources and stations ----------------------------------------------------------------

@pytest.mark.parametrize("cmp_type", [1, 2, 3])
@pytest.mark.parametrize("medium", ["iso", "vti"])
def test_force_and_moment_sources(cmp_type, medium):
    p = small_problem(medium, ni=40, nj=36, nk=30, nsrc=0, sta_grid=None, nsteps=50)
    locs = [(20, 18, 18), (11.3, 24.6, 22.2)]
    p.src = _sources(locs, cmp_type=cmp_type, stf_len=p.nt_total * p.dt, dt=p.dt, seed=cmp_type)
    p.sta = _stations(p.ni, p.nj, p.nk)
    _compare_run(p)


def test_cmp_type_3_is_force_only():
    """cmp_type 3 injects the forces only (the reference's reading): same result as cmp_type 1
    with the same components, bitwise."""
    p = small_problem("iso", ni=40, nj=36, nk=30, nsrc=0, nsteps=30)
    locs = [(20, 18, 18)]
    out = []
    for ct in (1, 3):
        p.src = _sources(locs, cmp_type=ct, stf_len=p.nt_total * p.dt, dt=p.dt, seed=5)
        s = Simulation(p)
        s.run()
        out.append(s.seismograms())
    assert np.abs(out[0]).max() > 0
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("wavelet", list(WAVELETS))
def test_every_wavelet(wavelet):
    p = small_problem("iso", ni=40, nj=36, nk=30, nsrc=0, nsteps=50)
    p.src = _sources([(20, 18, 19.4)], cmp_type=2, wavelet=wavelet, fc=4.0, stf_len=p.nt_total * p.dt,
                     dt=p.dt, seed=11, t_start=0.0013)
    _compare_run(p)


@pytest.mark.parametrize("medium", ["iso", "aniso"])
def test_sampled_stf_edge_and_overlapping_sources(medium):
    """Sampled source time functions on sources at the grid's edges and corners (smoothing
    stencil clipped), two sources on one point, one starting later, one just outside."""
    p = small_problem(medium, ni=40, nj=36, nk=30, nsrc=0, nsteps=50)
    locs = [(0, 18, 15), (39, 35, 29), (20, 0, 0), (1.4, 33.6, 27.8), (20, 18, 15), (20, 18, 15), (-2, 10, 10)]
    src = _sources(locs, cmp_type=2, stf_given=1, dt=p.dt, nt=60, seed=13)
    src.t_start = np.asarray([0, 0, 0, 0, 0, 3.5 * p.dt, 0], np.float32)
    p.src = src
    p.sta = _stations(p.ni, p.nj, p.nk)
    _compare_run(p)


def test_edge_sources_with_wavelets_and_force():
    p = small_problem("vti", ni=40, nj=36, nk=30, nsrc=0, nsteps=40)
    p.src = _sources([(0, 0, 29), (39, 0, 1), (2, 34, 28.6)], cmp_type=1, stf_len=p.nt_total * p.dt, dt=p.dt,
                     seed=17)
    p.sta = _stations(p.ni, p.nj, p.nk)
    _compare_run(p)


def test_batch_mixes_force_and_moment_shots():
    """One batch: a force shot, a moment shot (strike/dip/rake), a sampled-STF shot. Each shot
    equals its own oracle run."""
    p = small_problem("iso", ni=44, nj=40, nk=32, nsrc=0, nsteps=40, sta_grid=(3, 3))
    rng = np.random.default_rng(3)
    shots = [_sources([(22, 20, 20)], cmp_type=1, stf_len=p.nt_total * p.dt, dt=p.dt, seed=1),
             synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(700.0, 1000.0), fc_range=(3.0, 4.0),
                              stf_length=p.nt_total * p.dt),
             _sources([(10, 30, 25), (30, 8, 22)], cmp_type=2, stf_given=1, dt=p.dt, nt=50, seed=2)]
    b = Simulation(p, shots=shots)
    b.run()
    bs = b.seismograms()
    for n, s in enumerate(shots):
        q = dataclasses.replace(p, src=s)
        o = Oracle(q)
        o.run()
        r = o.seismograms()
        assert np.abs(r).max() > 0
        assert per_station_rel_l2(bs[n], r) <= 1e-4, n
