"""The drop-in CLI on CPU: reads par.json, NetCDF grid/media (written by scipy, an independent
NetCDF implementation), .src and station list, checks dt in FP64 - then stops at device
creation because there is no GPU here."""
import os
import re
import subprocess

import numpy as np
import pytest

from cgfd_b200 import formats, synth
from helpers import small_problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpu-cgfd3d-elastic_b200", "_build", "cgfd3d_b200")


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(gpu_available(), reason="checks the CPU-side stages only")
@pytest.mark.parametrize("medium", ["iso", "vti", "aniso"])
def test_cli_reads_reference_formats(tmp_path, medium):
    p = small_problem(medium, nsteps=4)
    par = formats.write_case(str(tmp_path), p, 4)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1
    m = re.search(r"maximum allowed time step = ([0-9.eE+-]+)", r.stdout)
    assert m, r.stdout + r.stderr
    assert float(m.group(1)) == pytest.approx(synth.dt_estimate(p), rel=1e-5)
    assert "metrics on the GPU:" in r.stderr  # reached the device stage (GPU metric calculation)


def test_cli_rejects_off_path_options(tmp_path):
    p = small_problem("iso", nsteps=2)
    par = formats.write_case(str(tmp_path), p, 2)
    import json
    cfg = json.load(open(par))
    cfg["medium"]["input_way"] = "code"  # the reference's built-in test media
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "not on this path" in r.stderr
    cfg["medium"]["input_way"] = "import"
    cfg["boundary_x_left"] = {"ablexp": {"number_of_layers": 10}}
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "ablexp" in r.stderr
    # visco-elastic media: GMB only, and Q volumes through the media import only
    cfg = json.load(open(par))
    cfg.pop("boundary_x_left", None)
    cfg["medium"]["type"] = "viscoelastic_iso"
    cfg["medium"]["input_way"] = "infile_layer"
    cfg["visco_config"] = {"visco_type": "gmb", "number_of_maxwell": 3, "min_freq": 0.2, "max_freq": 20.0,
                           "refer_freq": 2.0}
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "one-component" in r.stderr, r.stderr
    cfg["visco_config"]["visco_type"] = "graves_Qs"
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "gmb" in r.stderr, r.stderr


def test_cli_dt_check_rejects_unstable_step(tmp_path):
    p = small_problem("iso", nsteps=2)
    p.dt = 1.0
    par = formats.write_case(str(tmp_path), p, 2)
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "> dtmax" in r.stderr


def test_cli_reads_grid_and_binary_media_files(tmp_path):
    """The media file readers run before the device: a grid file whose layer boundary surfaces
    differ is refused as read_grid_file's checkGridData does, and a binary model file shorter than
    its size is refused ("Insufficient data", read_bin_file)."""
    import json
    from cgfd_b200 import synth
    p = small_problem("iso", nsteps=2)
    par = formats.write_case(str(tmp_path), p, 2)
    cfg = json.load(open(par))
    model = synth.grid_media(p.coord, seed=4)
    model.elevation[model.ngz[0]] += 1.0  # the second layer's first surface leaves the first's last
    grd = os.path.join(str(tmp_path), "model.grd")
    formats.write_grid_media_file(grd, model)
    cfg["medium"] = {"type": "elastic_iso", "input_way": "infile_grid", "infile_grid": grd,
                     "equivalent_medium_method": "loc"}
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "must equal the first elevations" in r.stderr, r.stderr
    medium = formats.write_bin_model(os.path.join(str(tmp_path), "bin"), synth.bin_model(p.coord, seed=4))
    with open(medium["binfile"]["Vs"], "r+b") as f:
        f.truncate(100)
    cfg["medium"] = medium
    json.dump(cfg, open(par, "w"))
    r = subprocess.run([CLI, par, "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Insufficient data" in r.stderr, r.stderr
