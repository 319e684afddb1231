"""Readers and writers of the reference's text input formats.

.src (src_t.cu:143-790; writer example/prep_source/src_export.m):
    evtnm / N / stf_given [len | dt nt] / cmp_type mech_type / loc_coord_type loc_3dim /
    N location lines / per source: (t_start name c0..c9 + component line) or
    (t_start + nt component lines). Lines starting with '#' are comments (io_funcs.cu:2130).
station list (io_funcs.cu:52-80): N / `name flag_coord flag_depth x y z` per station.
"""
import numpy as np

from .abi import Sources, Stations, WAVELETS

_NAMES = {v: k for k, v in WAVELETS.items()}
_NCMP = {1: 3, 2: 6, 3: 9}


def _lines(text):
    for ln in text.splitlines():
        if not ln or ln[0] == "#" or ln == "\n":
            continue
        yield ln


def _cmp_slice(cmp_type):
    return {1: slice(0, 3), 2: slice(3, 9), 3: slice(0, 9)}[cmp_type]


def write_src(path, src: Sources, evtnm="event"):
    out = [evtnm, str(src.num)]
    if src.stf_given == 0:
        out.append(f"0 {src.stf_length:.9g}")
    else:
        out.append(f"1 {src.stf_dt:.9g} {src.stf_nt}")
    out.append(f"{src.cmp_type} {src.mechanism_type}")
    out.append(f"{src.loc_coord_type} {src.loc_3dim}")
    for s in range(src.num):
        out.append(" ".join(f"{v:.9g}" for v in src.loc[s]))
    sl = _cmp_slice(src.cmp_type)
    for s in range(src.num):
        if src.stf_given == 0:
            coefs = " ".join(f"{v:.9g}" for v in src.wavelet_coefs[s])
            out.append(f"{src.t_start[s]:.9g} {_NAMES[int(src.wavelet[s])]} {coefs}")
            out.append(" ".join(f"{v:.9g}" for v in src.cmp[s][sl]))
        else:
            out.append(f"{src.t_start[s]:.9g}")
            for t in range(src.stf_nt):
                out.append(" ".join(f"{v:.9g}" for v in src.cmp_values[s, t][sl]))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_src(path) -> Sources:
    with open(path) as f:
        it = _lines(f.read())
    next(it)  # event name
    n = int(next(it).split()[0])
    w = next(it).split()
    stf_given = int(w[0])
    stf_length = float(w[1]) if stf_given == 0 else 0.0
    stf_dt = float(w[1]) if stf_given == 1 else 0.0
    stf_nt = int(w[2]) if stf_given == 1 else 0
    cmp_type, mech = [int(x) for x in next(it).split()[:2]]
    loc_coord, loc_3dim = [int(x) for x in next(it).split()[:2]]
    loc = np.array([[float(x) for x in next(it).split()[:3]] for _ in range(n)], np.float32)
    sl = _cmp_slice(cmp_type)
    t_start = np.zeros(n, np.float32)
    if stf_given == 0:
        wav = np.zeros(n, np.int32)
        coefs = np.zeros((n, 10), np.float32)
        cmp = np.zeros((n, 9), np.float32)
        # sscanf semantics of src_t.cu:491-507: values missing on a line keep what the previous
        # source left in the same variables (0 before the first source)
        prev_c = np.zeros(10, np.float32)
        prev = np.zeros(9, np.float32)
        for s in range(n):
            w = next(it).split()
            t_start[s] = float(w[0])
            wav[s] = WAVELETS[w[1]]
            c = [float(x) for x in w[2:12]]
            prev_c[:len(c)] = c
            coefs[s] = prev_c
            v = [float(x) for x in next(it).split()][: sl.stop - sl.start]
            prev[sl.start:sl.start + len(v)] = v
            cmp[s] = prev
        return Sources(loc=loc, t_start=t_start, wavelet=wav, wavelet_coefs=coefs, cmp=cmp, stf_given=0,
                       stf_length=stf_length, cmp_type=cmp_type, mechanism_type=mech, loc_coord_type=loc_coord,
                       loc_3dim=loc_3dim)
    vals = np.zeros((n, stf_nt, 9), np.float32)
    for s in range(n):
        t_start[s] = float(next(it).split()[0])
        for t in range(stf_nt):
            v = [float(x) for x in next(it).split()]
            vals[s, t, sl] = v[: sl.stop - sl.start]
    return Sources(loc=loc, t_start=t_start, cmp_values=vals, stf_given=1, stf_dt=stf_dt, stf_nt=stf_nt,
                   cmp_type=cmp_type, mechanism_type=mech, loc_coord_type=loc_coord, loc_3dim=loc_3dim)


def write_station_list(path, sta: Stations):
    names = sta.names or [f"sta{n:04d}" for n in range(sta.num)]
    fc = sta.flag_coord if sta.flag_coord is not None else np.zeros(sta.num, np.int32)
    out = [str(sta.num)]
    for n in range(sta.num):
        x, y, z = sta.loc[n]
        out.append(f"{names[n]} {int(fc[n])} {int(sta.flag_depth[n])} {x:.9g} {y:.9g} {z:.9g}")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_station_list(path) -> Stations:
    with open(path) as f:
        it = _lines(f.read())
    n = int(next(it).split()[0])
    names, fc, fd, loc = [], [], [], []
    for _ in range(n):
        w = next(it).split()
        names.append(w[0])
        fc.append(int(w[1]))
        fd.append(int(w[2]))
        loc.append([float(x) for x in w[3:6]])
    return Stations(loc=np.array(loc, np.float32), flag_depth=np.array(fd, np.int32),
                    flag_coord=np.array(fc, np.int32), names=names)


# ---------------------------------------------------------------------------------------
# Reference-format input sets and SAC files
# ---------------------------------------------------------------------------------------
def _write_nc(path, names, fields, ni, nj, nk, version=2):
    """Physical points of reference-layout fields as float variables (k, j, i), with the
    global attributes of gd_curv_coord_export (gd_t.cu:636-726). Uses scipy's NetCDF classic
    writer, an implementation independent of the library's reader."""
    from scipy.io import netcdf_file
    f = netcdf_file(path, "w", version=version)
    f.createDimension("i", ni)
    f.createDimension("j", nj)
    f.createDimension("k", nk)
    for n, fld in zip(names, fields):
        v = f.createVariable(n, "f4", ("k", "j", "i"))
        v[:] = np.ascontiguousarray(fld[3:-3, 3:-3, 3:-3], np.float32)
    setattr(f, "global_index_of_first_physical_points", np.array([0, 0, 0], np.int32))
    setattr(f, "count_of_physical_points", np.array([ni, nj, nk], np.int32))
    f.close()


MEDIUM_NAMES = {
    1: ["rho", "kappa"],
    2: ["rho", "lambda", "mu"],
    3: ["rho", "c11", "c13", "c33", "c55", "c66"],
    4: ["rho"] + [f"c{a}{b}" for a in range(1, 7) for b in range(a, 7)],
}
MEDIUM_TYPES = {1: "acoustic_iso", 2: "elastic_iso", 3: "elastic_vti", 4: "elastic_aniso"}


def write_case(d, p, nsteps, metric="calculate", check_stability=1, snapshots=None, extra=None):
    """Writes a full reference-format input set for problem `p` into directory `d`:
    par.json, grid/coord_px0_py0_pz0.nc, media/media_px0_py0_pz0.nc, src.src, station.list
    (and grid/metric_px0_py0_pz0.nc when metric == "import"); `extra` adds par-file entries
    (e.g. "receiver_line", "slice"). Returns the par.json path."""
    import json
    import os
    os.makedirs(os.path.join(d, "grid"), exist_ok=True)
    os.makedirs(os.path.join(d, "media"), exist_ok=True)
    _write_nc(os.path.join(d, "grid", "coord_px0_py0_pz0.nc"), ["x", "y", "z"], p.coord, p.ni, p.nj, p.nk)
    if metric == "import":
        _write_nc(os.path.join(d, "grid", "metric_px0_py0_pz0.nc"),
                  ["jac", "xi_x", "xi_y", "xi_z", "eta_x", "eta_y", "eta_z", "zeta_x", "zeta_y", "zeta_z"],
                  p.metric, p.ni, p.nj, p.nk)
    _write_nc(os.path.join(d, "media", "media_px0_py0_pz0.nc"), MEDIUM_NAMES[p.medium_type], p.medium,
              p.ni, p.nj, p.nk)
    write_src(os.path.join(d, "src.src"), p.src)
    write_station_list(os.path.join(d, "station.list"), p.sta)
    names = [["boundary_x_left", "boundary_x_right"], ["boundary_y_front", "boundary_y_back"],
             ["boundary_z_bottom", "boundary_z_top"]]
    par = {
        "number_of_total_grid_points_x": p.ni, "number_of_total_grid_points_y": p.nj,
        "number_of_total_grid_points_z": p.nk, "number_of_mpiprocs_x": 1, "number_of_mpiprocs_y": 1,
        "size_of_time_step": float(p.dt), "number_of_time_steps": int(nsteps), "check_stability": check_stability,
        "grid_generation_method": {"import": os.path.join(d, "grid")},
        "metric_calculation_method": ({"import": os.path.join(d, "grid")} if metric == "import" else {"calculate": 1}),
        "medium": {"type": MEDIUM_TYPES[p.medium_type], "input_way": "import",
                   "import": os.path.join(d, "media"), "#code": "func_name_here"},
        "in_source_file": os.path.join(d, "src.src"),
        "in_station_file": os.path.join(d, "station.list"),
        "output_dir": os.path.join(d, "output"),
        "check_nan_every_nummber_of_steps": 0, "output_all": 0,
    }
    for a in range(3):
        for s in range(2):
            f = p.pml[a][s]
            if f:
                par[names[a][s]] = {"cfspml": {"number_of_layers": f["num_layers"], "alpha_max": f["alpha_max"],
                                               "beta_max": f["beta_max"], "ref_vel": f["ref_vel"]}}
    if p.free_top:
        par["boundary_z_top"] = {"free": "timg"}
    if snapshots:
        par["snapshot"] = list(snapshots)  # entries in the par-file form (1-based grid_index_start)
    if extra:
        par.update(extra)
    path = os.path.join(d, "par.json")
    with open(path, "w") as f:
        json.dump(par, f, indent=2)
    return path


def read_sac(path):
    """(header dict, data) of a SAC file written little-endian (the reference's native order)."""
    raw = open(path, "rb").read()
    fh = np.frombuffer(raw[:280], "<f4")
    ih = np.frombuffer(raw[280:440], "<i4")
    ch = raw[440:632]
    hdr = {"delta": float(fh[0]), "b": float(fh[5]), "e": float(fh[6]), "stla": float(fh[31]),
           "stlo": float(fh[32]), "stel": float(fh[33]), "stdp": float(fh[34]), "evla": float(fh[35]),
           "nvhdr": int(ih[6]), "npts": int(ih[9]), "iftype": int(ih[15]), "leven": int(ih[35]),
           "kstnm": ch[0:8], "kcmpnm": ch[160:168], "depmin": float(fh[1])}
    data = np.frombuffer(raw[632:632 + 4 * hdr["npts"]], "<f4").copy()
    return hdr, data


class LayerModel:
    """A layered elastic-isotropic model, the contents of the reference's "elastic_isotropic"
    interface file (read_interface_file, src/media/media_read_file.cpp:22-210): interfaces top
    first on a uniform nx x ny mesh; per interface the elevation and the value / gradient /
    power of rho, vp, vs of the layer below it, each [num_interfaces, ny, nx]."""

    FIELDS = ("elevation", "rho", "rho_grad", "rho_pow", "vp", "vp_grad", "vp_pow", "vs", "vs_grad", "vs_pow")

    def __init__(self, x0, y0, dx, dy, **fields):
        self.x0, self.y0, self.dx, self.dy = float(x0), float(y0), float(dx), float(dy)
        for n in self.FIELDS:
            setattr(self, n, np.ascontiguousarray(fields[n], np.float32))
        self.ny, self.nx = self.elevation.shape[1:]


def write_layer_file(path, m: LayerModel):
    """The interface file in the reference's format: media type, number of interfaces, the mesh
    "NX NY MINX MINY DX DY", then one line per interface and mesh point (x fastest) with the
    elevation and value, gradient, power of rho, vp, vs (values written so that they read back
    exactly as float)."""
    ni = m.elevation.shape[0]
    with open(path, "w") as f:
        f.write("# layered elastic-isotropic model\nelastic_isotropic\n")
        f.write(f"{ni}\n{m.nx} {m.ny} {m.x0:.9g} {m.y0:.9g} {m.dx:.9g} {m.dy:.9g}\n")
        cols = np.stack([getattr(m, n) for n in LayerModel.FIELDS], axis=-1).reshape(-1, len(LayerModel.FIELDS))
        for row in cols:
            f.write(" ".join(f"{v:.9g}" for v in row) + "\n")


# Layer file types (the reference's media type numbers) and their parameters in file order
LAYER_TYPES = {
    10: ("acoustic_isotropic", ("rho", "vp")),
    21: ("elastic_isotropic", ("rho", "vp", "vs")),
    22: ("elastic_vti_prem", ("rho", "vph", "vpv", "vsh", "vsv", "eta")),
    23: ("elastic_vti_thomsen", ("rho", "vp0", "vs0", "epsilon", "delta", "gamma")),
    24: ("elastic_vti_cij", ("rho", "c11", "c33", "c55", "c66", "c13")),
    25: ("elastic_tti_thomsen", ("rho", "vp0", "vs0", "epsilon", "delta", "gamma", "azimuth", "dip")),
    26: ("elastic_tti_bond", ("rho", "c11", "c33", "c55", "c66", "c13", "azimuth", "dip")),
    27: ("elastic_aniso_cij", ("rho", "c11", "c12", "c13", "c14", "c15", "c16", "c22", "c23", "c24", "c25", "c26",
                               "c33", "c34", "c35", "c36", "c44", "c45", "c46", "c55", "c56", "c66")),
}


class LayerMedia:
    """A layer file of the acoustic or any elastic type (read_interface_file,
    src/media/media_read_file.cpp:22-700):
    interfaces top first on a uniform nx x ny mesh; `elevation` [num_interfaces, ny, nx] and
    `param` [npar, 3, num_interfaces, ny, nx]: value, gradient and power of each parameter of
    LAYER_TYPES[type], in the file's order, for the layer below each interface."""

    def __init__(self, type, x0, y0, dx, dy, elevation, param):
        self.type = int(type)
        self.x0, self.y0, self.dx, self.dy = float(x0), float(y0), float(dx), float(dy)
        self.elevation = np.ascontiguousarray(elevation, np.float32)
        self.param = np.ascontiguousarray(param, np.float32)
        self.ny, self.nx = self.elevation.shape[1:]
        assert self.param.shape == (len(LAYER_TYPES[self.type][1]), 3) + self.elevation.shape


def write_layer_media_file(path, m: LayerMedia):
    """The interface file of m in the reference's format: the type name, number of interfaces,
    "NX NY MINX MINY DX DY", then per interface and mesh point (x fastest) the elevation and
    value, gradient, power of every parameter (values written so that they read back exactly)."""
    ni = m.elevation.shape[0]
    name = LAYER_TYPES[m.type][0]
    with open(path, "w") as f:
        f.write(f"# layered {name} model\n{name}\n")
        f.write(f"{ni}\n{m.nx} {m.ny} {m.x0:.9g} {m.y0:.9g} {m.dx:.9g} {m.dy:.9g}\n")
        cols = [m.elevation.reshape(-1)]
        for q in range(m.param.shape[0]):
            for c in range(3):
                cols.append(m.param[q, c].reshape(-1))
        for row in np.stack(cols, axis=-1):
            f.write(" ".join(f"{v:.9g}" for v in row) + "\n")


class BinModel:
    """A 3-D binary model (the par file's medium input_way "binfile"): volumes rho, vp, vs with
    size[0] x size[1] x size[2] samples, file dimension 0 fastest (numpy shape (size[2], size[1],
    size[0])); order[d] is the grid axis (0 x, 1 y, 2 z) of file dimension d."""

    def __init__(self, order, size, spacing, origin, rho, vp, vs):
        self.order, self.size = [int(v) for v in order], [int(v) for v in size]
        self.spacing, self.origin = [float(v) for v in spacing], [float(v) for v in origin]
        shape = (self.size[2], self.size[1], self.size[0])
        self.rho, self.vp, self.vs = (np.ascontiguousarray(v, np.float32).reshape(shape) for v in (rho, vp, vs))


def write_bin_model(d, m: BinModel):
    """The three raw float32 files (rho.bin, vp.bin, vs.bin) into directory d and the par-file
    "medium" entry that reads them; returns that entry (medium type elastic_iso)."""
    import os
    os.makedirs(d, exist_ok=True)
    files = {}
    for name, v in (("rho", m.rho), ("Vp", m.vp), ("Vs", m.vs)):
        path = os.path.join(d, name.lower() + ".bin")
        np.ascontiguousarray(v, "<f4").tofile(path)
        files[name] = path
    axes = "xyz"
    entry = {"size": list(m.size), "spacing": list(m.spacing), "origin": list(m.origin),
             "dim1": axes[m.order[0]], "dim2": axes[m.order[1]], "dim3": axes[m.order[2]]}
    entry.update(files)
    return {"type": "elastic_iso", "input_way": "binfile", "binfile": entry}


class GridMedia:
    """A grid model (read_grid_file, src/media/media_read_file.cpp:670-1266): `ngz[l]` surfaces per
    layer, top first, on a uniform nx x ny mesh; `elevation` [NI, ny, nx] and `param` [npar, NI,
    ny, nx], the parameters of LAYER_TYPES[type] in file order (values only)."""

    def __init__(self, ngz, x0, y0, dx, dy, elevation, param, type=21):
        self.type = int(type)
        self.ngz = [int(v) for v in ngz]
        self.x0, self.y0, self.dx, self.dy = float(x0), float(y0), float(dx), float(dy)
        self.elevation = np.ascontiguousarray(elevation, np.float32)
        self.param = np.ascontiguousarray(param, np.float32)
        self.ny, self.nx = self.elevation.shape[1:]
        npar = len(LAYER_TYPES[self.type][1])
        assert self.elevation.shape[0] == sum(self.ngz) and self.param.shape == (npar,) + self.elevation.shape


def write_grid_media_file(path, m: GridMedia):
    """The grid media file of m in the reference's format: the type name, the number of layers,
    the surfaces of each layer, "NX NY MINX MINY DX DY", then per surface and mesh point (x
    fastest) the elevation and the type's parameters (values written so that they read back
    exactly)."""
    with open(path, "w") as f:
        f.write(LAYER_TYPES[m.type][0] + "\n")
        f.write(f"{len(m.ngz)}\n" + " ".join(str(v) for v in m.ngz) + "\n")
        f.write(f"{m.nx} {m.ny} {m.x0:.9g} {m.y0:.9g} {m.dx:.9g} {m.dy:.9g}\n")
        cols = [m.elevation.reshape(-1)] + [m.param[q].reshape(-1) for q in range(m.param.shape[0])]
        for row in np.stack(cols, axis=-1):
            f.write(" ".join(f"{v:.9g}" for v in row) + "\n")
