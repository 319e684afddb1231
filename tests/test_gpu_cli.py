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


def test_cli_snapshots_match_oracle(tmp_path):
    """"snapshot" entries (io_snap_nc_create/put): a free-surface slice every 5 steps with
    velocity, stress and strain, and a strided volume at the last step, as NetCDF record
    variables, against the oracle's wavefield at the same steps."""
    nsteps = 30
    p = small_problem("iso", nsteps=nsteps)
    snaps = [{"name": "surf", "grid_index_start": [1, 1, p.nk], "grid_index_count": [p.ni, p.nj, 1],
              "grid_index_incre": [1, 1, 1], "time_index_start": 0, "time_index_incre": 5,
              "save_velocity": 1, "save_stress": 1, "save_strain": 1},
             {"name": "vol", "grid_index_start": [2, 1, 1], "grid_index_count": [p.ni, p.nj, p.nk],
              "grid_index_incre": [2, 3, 2], "time_index_start": p.nt_total - 1, "time_index_incre": 1,
              "save_velocity": 1, "save_stress": 0, "save_strain": 0}]
    par = formats.write_case(str(tmp_path), p, nsteps, snapshots=snaps)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    from cgfd_b200 import synth
    from scipy.io import netcdf_file
    p.metric = synth.metrics(p.coord)
    orc = Oracle(p)
    states = {}
    for it in range(p.nt_total):
        states[it] = orc.wavefield()  # w_pre at the start of step it
        orc.run(1)
    out = os.path.join(str(tmp_path), "output")
    lam, mu = p.medium[1], p.medium[2]
    with netcdf_file(os.path.join(out, "surf_px0_py0_pz0.nc"), "r", mmap=False) as f:
        assert list(f.dimensions) == ["time", "k", "j", "i"] and f.dimensions["time"] is None
        t = f.variables["time"][:].copy()
        steps = list(range(0, p.nt_total, 5))
        assert len(t) == len(steps) and np.allclose(t, np.array(steps, np.float32) * np.float32(p.dt))
        names = ["Vx", "Vy", "Vz", "Txx", "Tyy", "Tzz", "Txz", "Tyz", "Txy"]
        comp = [0, 1, 2, 3, 4, 5, 7, 6, 8]
        for n, it in enumerate(steps):
            w = states[it][:, p.nk + 2:p.nk + 3, 3:-3, 3:-3]
            for name, c in zip(names, comp):
                got = f.variables[name][n]
                assert np.linalg.norm(got - w[c]) <= 1e-4 * max(np.linalg.norm(w[c]), 1e-30), (name, it)
            # isotropic strain from stress (io_snap_stress_to_strain_eliso)
            l, m = lam[p.nk + 2:p.nk + 3, 3:-3, 3:-3], mu[p.nk + 2:p.nk + 3, 3:-3, 3:-3]
            e1 = (l + m) / (m * (3 * l + 2 * m))
            e2 = -l / (2 * m * (3 * l + 2 * m))
            exx = e2 * (w[3] + w[4] + w[5]) - (e2 - e1) * w[3]
            got = f.variables["Exx"][n]
            assert np.linalg.norm(got - exx) <= 1e-4 * max(np.linalg.norm(exx), 1e-30)
            got = f.variables["Exz"][n]
            assert np.linalg.norm(got - 0.5 / m * w[7]) <= 1e-4 * max(np.linalg.norm(w[7] / m), 1e-30)
        assert list(f.first_index_in_this_thread_with_ghosts) == [3, 3, p.nk + 2]
    with netcdf_file(os.path.join(out, "vol_px0_py0_pz0.nc"), "r", mmap=False) as f:
        vx = f.variables["Vx"][:].copy()
        assert vx.shape == (1, (p.nk + 1) // 2, (p.nj + 2) // 3, p.ni // 2)
        w = states[p.nt_total - 1][0, 3:-3:2, 3:-3:3, 4:-3:2]
        assert np.linalg.norm(vx[0] - w) <= 1e-4 * np.linalg.norm(w)
        assert list(f.index_stride_in_this_thread) == [2, 3, 2]


def test_cli_layered_medium_matches_oracle(tmp_path):
    """medium input_way "infile_layer" with the har equivalent medium: the CLI discretises the
    layered model on the GPU; its seismograms equal the oracle's run on the medium the
    reference's own media code builds from the same file (per-station rel L2 <= 1e-4)."""
    import media_ref
    if not media_ref.available():
        pytest.skip("oracle/_ref/libref_media.so not built")
    from cgfd_b200 import synth
    nsteps = 60
    p = small_problem("iso", nsteps=nsteps)
    model = synth.layer_model(p.coord, seed=4, depths=(-1200.0, -2200.0))
    lay = os.path.join(str(tmp_path), "model.lay")
    formats.write_layer_file(lay, model)
    extra = {"medium": {"type": "elastic_iso", "input_way": "infile_layer", "infile_layer": lay,
                        "equivalent_medium_method": "har"}}
    par = formats.write_case(str(tmp_path), p, nsteps, extra=extra)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p.metric = synth.metrics(p.coord)
    p.medium = media_ref.layer2model_el_iso(p.coord, model, 1)
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(CMPS):
            got[n, c] = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))[1]
    assert np.abs(ref).max() > 0
    assert per_station_rel_l2(got, ref) <= 1e-4


@pytest.mark.parametrize("mtype,ftype,method", [("elastic_vti", 23, "ari"), ("elastic_aniso", 26, "loc"),
                                               ("acoustic_iso", 10, "har")])
def test_cli_layered_anisotropic_medium_matches_oracle(tmp_path, mtype, ftype, method):
    """infile_layer for the anisotropic and acoustic media: a Thomsen VTI layer file into a VTI
    medium (ari equivalent medium), a Bond-rotated TI file into a 21-Cij medium, an
    acoustic_isotropic file into an acoustic medium (har). The CLI discretises the file on the
    GPU; its seismograms equal the oracle's run on the medium the reference's own media code
    builds from the same file (per-station rel L2 <= 1e-4; acoustic: per group Vx Vy Vz / P)."""
    import media_ref
    if not media_ref.available():
        pytest.skip("oracle/_ref/libref_media.so not built")
    from cgfd_b200 import synth
    nsteps = 60
    med = {"elastic_vti": "vti", "elastic_aniso": "aniso", "acoustic_iso": "ac"}[mtype]
    p = small_problem(med, nsteps=nsteps)
    model = synth.layer_media(p.coord, ftype, seed=4, depths=(-1200.0, -2200.0))
    lay = os.path.join(str(tmp_path), "model.lay")
    formats.write_layer_media_file(lay, model)
    extra = {"medium": {"type": mtype, "input_way": "infile_layer", "infile_layer": lay,
                        "equivalent_medium_method": method}}
    par = formats.write_case(str(tmp_path), p, nsteps, extra=extra)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p.metric = synth.metrics(p.coord)
    p.medium = media_ref.layer2model(p.coord, model, {"elastic_vti": 3, "elastic_aniso": 4, "acoustic_iso": 1}[mtype],
                                     {"loc": 0, "har": 1, "ari": 2}[method])
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    cmps = ["Vx", "Vy", "Vz", "P"] if med == "ac" else CMPS
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(cmps):
            got[n, c] = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))[1]
    assert np.abs(ref).max() > 0
    if med == "ac":
        assert per_station_rel_l2(got[:, :3], ref[:, :3]) <= 1e-4
        assert per_station_rel_l2(got[:, 3:4], ref[:, 3:4]) <= 1e-4
    else:
        assert per_station_rel_l2(got, ref) <= 1e-4


def test_cli_acoustic_medium_matches_oracle(tmp_path):
    """An acoustic_iso par file (media_*.nc with rho and kappa): SAC files of Vx Vy Vz P per
    station (wav_ac_init's components) against the oracle, a z slice with the 4 components and
    a snapshot whose stress group is the pressure "Tii" (io_snap_nc_create_ac)."""
    nsteps = 60
    p = small_problem("ac", nsteps=nsteps, nsrc=2)
    snaps = [{"name": "below", "grid_index_start": [1, 1, p.nk - 1], "grid_index_count": [p.ni, p.nj, 1],
              "grid_index_incre": [1, 1, 1], "time_index_start": 0, "time_index_incre": 20,
              "save_velocity": 1, "save_stress": 1, "save_strain": 0}]
    par = formats.write_case(str(tmp_path), p, nsteps, metric="import", snapshots=snaps,
                             extra={"slice": {"z_index": [p.nk - 5]}})
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(["Vx", "Vy", "Vz", "P"]):
            hdr, data = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))
            assert hdr["npts"] == p.nt_total
            got[n, c] = data
        assert not os.path.exists(os.path.join(out, f"{name}.Txx.sac"))
    assert per_station_rel_l2(got[:, :3], ref[:, :3]) <= 1e-4
    assert per_station_rel_l2(got[:, 3:4], ref[:, 3:4]) <= 1e-4
    from scipy.io import netcdf_file
    with netcdf_file(os.path.join(out, f"slicez_k{p.nk - 5}_px0_py0_pz0.nc"), "r", mmap=False) as f:
        assert [v for v in f.variables if v != "time"] == ["Vx", "Vy", "Vz", "P"]
        assert f.variables["P"][:].shape[1:] == (p.nj, p.ni)
    with netcdf_file(os.path.join(out, "below_px0_py0_pz0.nc"), "r", mmap=False) as f:
        assert sorted(v for v in f.variables if v != "time") == ["Tii", "Vx", "Vy", "Vz"]
        # the state at the start of step 40 = the oracle's after 40 steps
        o40 = Oracle(p)
        o40.run(40)
        w = o40.wavefield()
        tii = f.variables["Tii"][2]
        assert np.linalg.norm(tii[0] - w[3, -5, 3:-3, 3:-3]) <= 1e-4 * np.linalg.norm(w[3, -5, 3:-3, 3:-3])


def test_cli_binary_medium_matches_oracle(tmp_path):
    """medium input_way "binfile" (elastic_iso): three raw float32 volumes, file dimensions z, x,
    y. The CLI discretises them on the GPU; its seismograms equal the oracle's run on the medium
    the reference's own media_bin2model_el_iso builds from the same files (per-station rel L2
    <= 1e-4)."""
    import media_ref
    if not media_ref.available():
        pytest.skip("oracle/_ref/libref_media.so not built")
    from cgfd_b200 import synth
    nsteps = 60
    p = small_problem("iso", nsteps=nsteps)
    model = synth.bin_model(p.coord, seed=4)
    medium = formats.write_bin_model(os.path.join(str(tmp_path), "bin"), model)
    par = formats.write_case(str(tmp_path), p, nsteps, extra={"medium": medium})
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p.metric = synth.metrics(p.coord)
    p.medium = media_ref.bin2model_el_iso(p.coord, model)
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(CMPS):
            got[n, c] = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))[1]
    assert np.abs(ref).max() > 0
    assert per_station_rel_l2(got, ref) <= 1e-4


@pytest.mark.parametrize("med,ftype", [("iso", 21), ("vti", 23)])
def test_cli_grid_medium_matches_oracle(tmp_path, med, ftype):
    """medium input_way "infile_grid" (har): an elastic_isotropic grid file into an iso medium and
    a Thomsen VTI grid file into a VTI medium. The CLI discretises the file on the GPU; its
    seismograms equal the oracle's run on the medium the reference's own media_grid2model_el_iso /
    _el_vti builds from the same file (per-station rel L2 <= 1e-4)."""
    import media_ref
    if not media_ref.available():
        pytest.skip("oracle/_ref/libref_media.so not built")
    from cgfd_b200 import synth
    nsteps = 60
    p = small_problem(med, nsteps=nsteps)
    model = synth.grid_media(p.coord, seed=4, type=ftype)
    path = os.path.join(str(tmp_path), "model.grd")
    formats.write_grid_media_file(path, model)
    medium = {"type": "elastic_" + med, "input_way": "infile_grid", "infile_grid": path,
              "equivalent_medium_method": "har"}
    par = formats.write_case(str(tmp_path), p, nsteps, extra={"medium": medium})
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    p.metric = synth.metrics(p.coord)
    p.medium = media_ref.grid2model(p.coord, model, {"iso": 2, "vti": 3}[med], 1)
    orc = Oracle(p)
    orc.run()
    ref = orc.seismograms()
    out = os.path.join(str(tmp_path), "output")
    got = np.zeros_like(ref)
    for n, name in enumerate(p.sta.names):
        for c, cn in enumerate(CMPS):
            got[n, c] = formats.read_sac(os.path.join(out, f"{name}.{cn}.sac"))[1]
    assert np.abs(ref).max() > 0
    assert per_station_rel_l2(got, ref) <= 1e-4
