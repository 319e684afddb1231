"""Visco-elastic media (CGFD_MEDIUM_VISCO_ISO, generalized Maxwell body; sv_curv_col_vis_iso_gpu.cu,
md_vis_GMB_cal_Y): the CUDA path through the C ABI against the reference's own visco-elastic
solver code, built unmodified (oracle/_ref/ref_harness: md_vis_GMB_cal_Y, sv_curv_col_vis_iso_dvh2dvz,
sv_curv_col_vis_iso_onestage, sv_curv_col_vis_iso_free_gpu in the reference's time loop).

Bars: the GMB fit (solved here in FP64, by the reference in float) within 3e-5 of the reference's
weights and 1e-5 of its unrelaxed moduli (measured 3e-6 / 1.2e-7); seismograms and wavefields
per-station / field relative L2 <= 2e-5 after 160 steps (measured 1.5e-6).
"""
import os
import tempfile

import numpy as np
import pytest

from cgfd_b200 import Simulation, CgfdError, visco_gmb
from golden import ref_io
from helpers import small_problem, rel_l2, per_station_rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(ref_io.HARNESS), reason="oracle/_ref/ref_harness not built")]

IN = (slice(None), slice(3, -3), slice(3, -3), slice(3, -3))


def _ref(p, nsteps):
    with tempfile.TemporaryDirectory() as d:
        return ref_io.run(p, d, nsteps)


def test_gmb_fit_matches_reference():
    p = small_problem("vis", nsteps=4, nsrc=1)
    ref = _ref(p, 1)
    m = p.medium[IN]
    lu, mu, yl, ym, wl = visco_gmb(p.visco, m[1], m[2], m[3], m[4])
    g = ref["gmb"]["fields"][IN]
    nm = p.visco["nmaxwell"]
    assert np.allclose(wl, ref["gmb"]["wl"], rtol=1e-6)
    e_l = np.abs(lu - g[0].ravel()).max() / np.abs(g[0]).max()
    e_m = np.abs(mu - g[1].ravel()).max() / np.abs(g[1]).max()
    e_yl = max(np.abs(yl[n] - g[2 + n].ravel()).max() / np.abs(g[2 + n]).max() for n in range(nm))
    e_ym = max(np.abs(ym[n] - g[2 + nm + n].ravel()).max() / np.abs(g[2 + nm + n]).max() for n in range(nm))
    print(f"gmb fit: lambda {e_l:.2e} mu {e_m:.2e} Ylam {e_yl:.2e} Ymu {e_ym:.2e}")
    assert e_l <= 1e-5 and e_m <= 1e-5
    assert e_yl <= 3e-5 and e_ym <= 3e-5


@pytest.mark.parametrize("free_top", [1, 0])
def test_seismograms_and_wavefield_match_reference(free_top):
    """Two sources, CFS-PML on every face (and the top without the free surface), 160 steps."""
    nsteps = 160
    p = small_problem("vis", nsteps=nsteps, nsrc=2, free_top=free_top, ni=44, nj=40, nk=36)
    if not free_top:
        p.sta.loc[:, 2] = 3.0
    ref = _ref(p, nsteps)
    p.metric = ref["metric"]
    sim = Simulation(p)
    sim.run(nsteps)
    s, r = sim.seismograms()[:, :, :nsteps], ref["seismo"][:, :, :nsteps]
    w, wr = sim.wavefield()[IN], ref["wave"][IN]
    es = per_station_rel_l2(s, r)
    ew = rel_l2(w, wr)
    print(f"visco free_top={free_top}: stations {es:.2e} wavefield {ew:.2e} max|ref| {np.abs(wr).max():.2e}")
    assert np.abs(r).max() > 0
    assert es <= 2e-5
    assert ew <= 2e-5


def test_attenuation_is_active():
    """The same problem with Q raised 1000x runs closer to the elastic medium, and the visco-elastic
    run decays: the memory variables are coupled in."""
    nsteps = 120
    p = small_problem("vis", nsteps=nsteps, nsrc=1)
    a = Simulation(p)
    a.run(nsteps)
    p2 = small_problem("vis", nsteps=nsteps, nsrc=1)
    p2.medium[3:] *= 1000.0
    b = Simulation(p2)
    b.run(nsteps)
    pe = small_problem("iso", nsteps=nsteps, nsrc=1)
    e = Simulation(pe)
    e.run(nsteps)
    d_vis = rel_l2(a.seismograms(), e.seismograms())
    d_hiq = rel_l2(b.seismograms(), e.seismograms())
    print(f"visco vs elastic {d_vis:.2e}, high-Q visco vs elastic {d_hiq:.2e}")
    assert d_hiq < 0.2 * d_vis


def test_unsupported_modes():
    p = small_problem("vis", nsteps=8, nsrc=1)
    s = Simulation(p)
    with pytest.raises(CgfdError):
        s.set_bulk_variant(1)
    with pytest.raises(CgfdError):
        Simulation(p, shots=[p.src, p.src])
