"""I/O with the reference harness (oracle/_ref/ref_harness): writes a Problem in the
reference's input formats and reads back the reference's outputs. Test infrastructure."""
import os
import subprocess

import numpy as np

from cgfd_b200 import formats

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def write_inputs(p, d, nsteps):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.txt"), "w") as f:
        f.write(f"{p.ni} {p.nj} {p.nk} {p.medium_type} {p.nt_total} {nsteps} {int(p.free_top)} {p.dt:.9g} {p.t0:.9g}\n")
        for a in range(3):
            for s in range(2):
                fc = p.pml[a][s]
                if fc:
                    f.write(f"1 {fc['num_layers']} {fc['alpha_max']:.9g} {fc['beta_max']:.9g} {fc['ref_vel']:.9g}\n")
                else:
                    f.write("0 0 0 0 0\n")
        if p.medium_type == 5:  # visco-elastic: "nmaxwell fr fmin fmax"
            v = p.visco
            f.write(f"{int(v['nmaxwell'])} {v['fr']:.9g} {v['fmin']:.9g} {v['fmax']:.9g}\n")
    np.ascontiguousarray(p.coord, np.float32).tofile(os.path.join(d, "coord.bin"))
    np.ascontiguousarray(p.medium, np.float32).tofile(os.path.join(d, "medium.bin"))
    formats.write_src(os.path.join(d, "src.src"), p.src)
    formats.write_station_list(os.path.join(d, "station.list"), p.sta)


def run(p, d, nsteps, timeout=600):
    write_inputs(p, d, nsteps)
    r = subprocess.run([HARNESS, d], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
    shp = (p.nk + 6, p.nj + 6, p.ni + 6)
    info = dict(ln.split() for ln in open(os.path.join(d, "ref_info.txt")))
    nrecv = int(info["nrecv"])
    seis = np.fromfile(os.path.join(d, "ref_seismo.bin"), np.float32).reshape(nrecv, 9, p.nt_total)
    wave = np.fromfile(os.path.join(d, "ref_wave.bin"), np.float32).reshape((9,) + shp)
    metric = np.fromfile(os.path.join(d, "ref_metric.bin"), np.float32).reshape((10,) + shp)
    pg_path = os.path.join(d, "ref_pg.bin")
    pg = np.fromfile(pg_path, np.float32).reshape((15,) + shp[1:]) if os.path.exists(pg_path) else None
    gmb = None
    gmb_path = os.path.join(d, "ref_gmb.bin")
    if os.path.exists(gmb_path):  # visco-elastic: lambda, mu, Ylam[n], Ymu[n] (unrelaxed), then wl[n]
        nm = int(p.visco["nmaxwell"])
        raw = np.fromfile(gmb_path, np.float32)
        n3 = shp[0] * shp[1] * shp[2]
        gmb = {"fields": raw[:(2 + 2 * nm) * n3].reshape((2 + 2 * nm,) + shp), "wl": raw[(2 + 2 * nm) * n3:]}
    return {"gmb": gmb, "seismo": seis, "wave": wave, "metric": metric, "pg": pg, "loop_ms": float(info["loop_ms"]),
            "cell_stages": int(info["cell_stages"]), "nsrc": int(info["nsrc"])}
