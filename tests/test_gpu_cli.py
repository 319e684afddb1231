"""The drop-in CLI end to end on the GPU: reference-format inputs -> SAC files, compared with
the oracle run on the same inputs (per-station relative L2 <= 1e-4)."""
import os
import subprocess

import numpy as np
import pytest

from cgfd_b200 import formats
from oracle.oracle import Oracle
from helpers import small_problem, per_station_rel_l2

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpu-cgfd3d-elastic_b200", "_build", "cgfd3d_b200")
CMPS = ["Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Tyz", "Txz", "Txy"]


@pytest.mark.parametrize("medium,metric", [("iso", "calculate"), ("vti", "import")])
def test_cli_sac_output_matches_oracle(tmp_path, medium, metric):
    nsteps = 60
    p = small_problem(medium, nsteps=nsteps)
    par = formats.write_case(str(tmp_path), p, nsteps, metric=metric)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    if metric == "calculate":
        from cgfd_b200 import synth
        p.metric = synth.metrics(p.coord)  # the CLI's FP64 metric
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(CMPS):
            hdr, data = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))
            assert hdr["npts"] == p.nt_total and hdr["delta"] == pytest.approx(p.dt)
            assert hdr["nvhdr"] == 6 and hdr["iftype"] == 1 and hdr["leven"] == 1 and hdr["b"] == 0.0
            assert hdr["stdp"] == pytest.approx(p.dt)  # the reference passes dt as stdp
            got[n, c] = data
    assert per_station_rel_l2(got, ref) <= 1e-4
    if medium == "iso":
        hdr, exx = formats.read_sac(os.path.join(out, f"{p.sta.names[0]}.Exx.sac"))
        assert exx.shape[0] == p.nt_total and np.isfinite(exx).all()
    # peak ground motion file (PG_slice_output): 15 variables (j, i) with ghosts, vs the oracle
    from scipy.io import netcdf_file
    with netcdf_file(os.path.join(out, "PG_V_A_D_px0_py0_pz0.nc"), "r", mmap=False) as f:
        names = ["PGV", "PGVh", "PGVx", "PGVy", "PGVz", "PGA", "PGAh", "PGAx", "PGAy", "PGAz",
                 "PGD", "PGDh", "PGDx", "PGDy", "PGDz"]
        pg = np.stack([f.variables[n][:].copy() for n in names])
        assert list(f.dimensions) == ["j", "i"] and pg.shape == (15, p.nj + 6, p.ni + 6)
        assert list(f.count_index_of_physical_points) == [p.ni, p.nj]
    opg = orc.peak_motion()
    for q in range(15):
        assert np.linalg.norm(pg[q] - opg[q]) <= 1e-4 * np.linalg.norm(opg[q]), q
