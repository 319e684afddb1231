"""Line receivers and slices (the io_line_keep / io_slice_nc_put outputs of the time loop),
through the C ABI and through the drop-in CLI.

- Line receivers sample w_pre at grid points at the start of every step: at the surface grid
  points of stations given by integer index (trilinear weight 1 at corner 0) they equal the
  station seismograms bitwise, and at interior points they equal the wavefield read back
  step by step, bitwise (both are copies of the same device values).
- Slices hold the full x / y / z planes of w_pre of every step in a device ring: bitwise equal
  to the wavefield read back at that step; steps outside the ring are refused.
- The CLI writes <line>.no<n>.<cmp>.sac per line receiver and slicex_i<i>/slicey_j<j>/
  slicez_k<k>_px0_py0_pz0.nc record files (time, 9 components) as the reference names them;
  their contents equal the oracle's wavefield within the path's 1e-4 bar.
"""
import os
import subprocess

import numpy as np
import pytest

from cgfd_b200 import Simulation, CgfdError, formats, synth
from oracle.oracle import Oracle
from helpers import small_problem

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpu-cgfd3d-elastic_b200", "_build", "cgfd3d_b200")
CMPS = ["Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy"]


def test_line_receivers_equal_stations_and_wavefield():
    p = small_problem("iso", nsteps=20)
    sim = Simulation(p)
    nsta = sim.num_stations
    ijk = np.zeros((nsta, 3), np.int32)
    sim_idx = np.zeros(nsta, np.int32)
    import ctypes as C
    from cgfd_b200 import lib
    lib().cgfd_station_info(sim.h, sim_idx.ctypes.data, ijk.ctypes.data)
    interior = np.array([[5, 7, 3], [20, 18, 12], [p.ni - 1, p.nj - 1, p.nk - 1]], np.int32)
    sim.set_line_receivers(np.concatenate([ijk, interior]))
    states = []
    for it in range(p.nt_total - 1):
        states.append(sim.wavefield())
        sim.run(1)
    lines = sim.line_seismograms()
    sta = sim.seismograms()
    assert np.abs(sta).max() > 0
    assert np.array_equal(lines[:nsta, :, :p.nt_total - 1], sta[:, :, :p.nt_total - 1])
    for r, (i, j, k) in enumerate(interior):
        got = lines[nsta + r, :, :p.nt_total - 1]
        want = np.stack([s[:, k + 3, j + 3, i + 3] for s in states], axis=1)
        assert np.array_equal(got, want)


def test_line_receivers_reject_points_outside():
    p = small_problem("iso", nsteps=4, nsrc=0, sta_grid=None)
    sim = Simulation(p)
    with pytest.raises(CgfdError):
        sim.set_line_receivers([[p.ni, 0, 0]])


@pytest.mark.parametrize("precision", [0, 5])
def test_slices_equal_wavefield_each_step(precision):
    p = small_problem("vti", nsteps=12)
    p.precision = precision
    sim = Simulation(p)
    ix, iy, iz = [3, 17], [10], [0, p.nk - 1, 9]
    sim.set_slices(ix, iy, iz, ring_steps=4)
    states = []
    for it in range(7):
        states.append(sim.wavefield())
        sim.run(1)
    for it in range(3, 7):  # the ring holds the last 4 steps
        x, y, z = sim.slices(it)
        w = states[it][:, 3:-3, 3:-3, 3:-3]  # [9, nk, nj, ni]
        for s, i in enumerate(ix):
            assert np.array_equal(x[s], w[:, :, :, i])
        for s, j in enumerate(iy):
            assert np.array_equal(y[s], w[:, :, j, :])
        for s, k in enumerate(iz):
            assert np.array_equal(z[s], w[:, k, :, :])
    assert np.abs(states[6]).max() > 0
    for bad in (2, 7):
        with pytest.raises(CgfdError):
            sim.slices(bad)


def test_cli_lines_and_slices_match_oracle(tmp_path):
    nsteps = 24
    p = small_problem("iso", nsteps=nsteps)
    extra = {"receiver_line": [{"name": "L1", "grid_index_start": [3, 5, p.nk], "grid_index_incre": [4, 0, 0],
                                "grid_index_count": 12},
                               {"name": "V", "grid_index_start": [20, 18, 1], "grid_index_incre": [0, 0, 7],
                                "grid_index_count": 6}],
             "slice": {"x_index": [11, 1000], "y_index": [19], "z_index": [p.nk, 5]}}
    par = formats.write_case(str(tmp_path), p, nsteps, extra=extra)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p.metric = synth.metrics(p.coord)  # the CLI's FP64 metric
    orc = Oracle(p)
    states = []
    for it in range(p.nt_total):
        states.append(orc.wavefield())
        orc.run(1)
    out = os.path.join(str(tmp_path), "output")
    # line receivers inside the grid: L1 points 0..9 (x 2, 6, .., 38), V points 0..4 (k 0, 7, .., 28)
    pts = [("L1", n, 2 + 4 * n, 4, p.nk - 1) for n in range(10)] + [("V", n, 19, 17, 7 * n) for n in range(5)]
    assert not os.path.exists(os.path.join(out, "L1.no10.Vx.sac"))
    assert not os.path.exists(os.path.join(out, "V.no5.Vx.sac"))
    for name, n, i, j, k in pts:
        for c, cn in enumerate(CMPS):
            hdr, data = formats.read_sac(os.path.join(out, f"{name}.no{n}.{cn}.sac"))
            want = np.array([s[c, k + 3, j + 3, i + 3] for s in states], np.float64)
            assert hdr["npts"] == p.nt_total
            den = max(np.linalg.norm(want), 1e-3 * np.abs(np.array(states)[:, c]).max() * np.sqrt(p.nt_total), 1e-30)
            assert np.linalg.norm(data - want) <= 1e-4 * den, (name, n, cn)
    from scipy.io import netcdf_file
    files = {"slicex_i11": ("k", "j"), "slicey_j19": ("k", "i"), f"slicez_k{p.nk}": ("j", "i"), "slicez_k5": ("j", "i")}
    assert not os.path.exists(os.path.join(out, "slicex_i1000_px0_py0_pz0.nc"))
    for stem, dims in files.items():
        with netcdf_file(os.path.join(out, stem + "_px0_py0_pz0.nc"), "r", mmap=False) as f:
            assert list(f.dimensions) == ["time", *dims] and f.dimensions["time"] is None
            t = f.variables["time"][:].copy()
            assert len(t) == p.nt_total
            assert np.allclose(t, np.arange(p.nt_total, dtype=np.float32) * np.float32(p.dt))
            idx = int(stem.split("_")[1][1:]) - 1
            for c, cn in enumerate(CMPS):
                got = f.variables[cn][:].copy()
                for it in (5, p.nt_total - 1):
                    w = states[it][c, 3:-3, 3:-3, 3:-3]
                    want = w[:, :, idx] if stem.startswith("slicex") else (
                        w[:, idx, :] if stem.startswith("slicey") else w[idx])
                    assert np.linalg.norm(got[it] - want) <= 1e-4 * max(np.linalg.norm(want), 1e-30), (stem, cn, it)
