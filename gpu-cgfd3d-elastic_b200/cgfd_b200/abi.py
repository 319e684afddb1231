"""ctypes mirror of include/cgfd_b200.h.

`Problem` carries the inputs of drv_rk_curv_col_allstep (reference
src/forward/drv_rk_curv_col.cu:28-50) as numpy arrays in the reference host layout
[cmp][k][j][i] with 3 ghost points per side; `Simulation` owns the device state.
"""
import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

CGFD_MEDIUM_ACOUSTIC_ISO = 1
CGFD_MEDIUM_ELASTIC_ISO = 2
CGFD_MEDIUM_ELASTIC_VTI = 3
CGFD_MEDIUM_ELASTIC_ANISO = 4
CGFD_MEDIUM_VISCO_ISO = 5
CGFD_ERR_BUSY = -7
CGFD_ERR_NOMEM = -3
CGFD_PREC_FP32 = 0
CGFD_PREC_BF16_COEF = 1
CGFD_PREC_FP16_COEF = 2
CGFD_PREC_U16_COEF = 3
CGFD_PREC_FP16_WAVE = 4
CGFD_PREC_FP64 = 5
# wavelet names of src_t.cu:873-903 -> ids
WAVELETS = {"ricker": 0, "gaussian": 1, "ricker_deriv": 2, "gaussian_deriv": 3, "klauder": 4}

_HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(os.path.dirname(_HERE), "_build", "libcgfd_b200.so")


class CgfdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cgfd error {code}: {msg}")
        self.code = code


class PmlFace(C.Structure):
    _fields_ = [("enable", C.c_int), ("num_layers", C.c_int), ("alpha_max", C.c_float),
                ("beta_max", C.c_float), ("ref_vel", C.c_float)]


class SourceDesc(C.Structure):
    _fields_ = [("num", C.c_int), ("stf_given", C.c_int), ("stf_length", C.c_float),
                ("stf_dt", C.c_float), ("stf_nt", C.c_int), ("cmp_type", C.c_int),
                ("mechanism_type", C.c_int), ("loc_coord_type", C.c_int), ("loc_3dim", C.c_int),
                ("loc", C.c_void_p), ("t_start", C.c_void_p), ("wavelet", C.c_void_p),
                ("wavelet_coefs", C.c_void_p), ("cmp", C.c_void_p), ("cmp_values", C.c_void_p)]


class StationDesc(C.Structure):
    _fields_ = [("num", C.c_int), ("flag_coord", C.c_void_p), ("flag_depth", C.c_void_p),
                ("loc", C.c_void_p)]


class ViscoDesc(C.Structure):
    """cgfd_visco_desc: GMB parameters of a visco-elastic medium (par_t.cu:728-770)."""
    _fields_ = [("nmaxwell", C.c_int), ("fr", C.c_float), ("fmin", C.c_float), ("fmax", C.c_float)]


class ProblemDesc(C.Structure):
    _fields_ = [("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("medium_type", C.c_int),
                ("coord", C.c_void_p), ("metric", C.c_void_p), ("medium", C.c_void_p),
                ("pml", (PmlFace * 2) * 3), ("free_top", C.c_int), ("dt", C.c_float),
                ("t0", C.c_float), ("nt_total", C.c_int), ("src", SourceDesc),
                ("sta", StationDesc), ("precision", C.c_int), ("device", C.c_int),
                ("visco", C.POINTER(ViscoDesc))]


def medium_ncmp(medium_type):
    return {CGFD_MEDIUM_ACOUSTIC_ISO: 2, CGFD_MEDIUM_ELASTIC_ISO: 3, CGFD_MEDIUM_ELASTIC_VTI: 6,
            CGFD_MEDIUM_ELASTIC_ANISO: 22, CGFD_MEDIUM_VISCO_ISO: 5}[medium_type]


def ref_shape(ni, nj, nk):
    """(nz, ny, nx) of one field in the reference layout."""
    return (nk + 6, nj + 6, ni + 6)


def _ptr(a):
    return None if a is None else a.ctypes.data


@dataclass
class Sources:
    """In-memory .src content (src_t.cu:205-611)."""
    loc: np.ndarray                      # [n,3] float32, 0-based grid index
    t_start: np.ndarray                  # [n]
    wavelet: Optional[np.ndarray] = None  # [n] int32 ids
    wavelet_coefs: Optional[np.ndarray] = None  # [n,10]
    cmp: Optional[np.ndarray] = None     # [n,9] fx fy fz mxx myy mzz myz mxz mxy
    cmp_values: Optional[np.ndarray] = None  # [n,nt,9]
    stf_given: int = 0
    stf_length: float = 0.0
    stf_dt: float = 0.0
    stf_nt: int = 0
    cmp_type: int = 2
    mechanism_type: int = 0
    loc_coord_type: int = 0
    loc_3dim: int = 0

    @property
    def num(self):
        return int(self.loc.shape[0])


@dataclass
class Stations:
    """In-memory station list (io_funcs.cu:52-80): 1-based x,y index; z per flag_depth."""
    loc: np.ndarray                      # [n,3]
    flag_depth: np.ndarray               # [n] int32
    flag_coord: Optional[np.ndarray] = None
    names: Optional[list] = None

    @property
    def num(self):
        return int(self.loc.shape[0])


@dataclass
class Problem:
    ni: int
    nj: int
    nk: int
    medium_type: int
    coord: Optional[np.ndarray]          # [3,nz,ny,nx] float32
    metric: np.ndarray                   # [10,nz,ny,nx]
    medium: np.ndarray                   # [ncmp,nz,ny,nx] (rho = density)
    dt: float
    nt_total: int
    t0: float = 0.0
    pml: list = field(default_factory=lambda: [[None, None], [None, None], [None, None]])
    free_top: int = 1
    src: Optional[Sources] = None
    sta: Optional[Stations] = None
    precision: int = CGFD_PREC_FP32
    device: int = 0
    # visco-elastic media (medium rho lambda mu Qp Qs): {"nmaxwell", "fr", "fmin", "fmax"}
    visco: Optional[dict] = None

    def desc(self):
        """Build the C description; the returned object keeps every array alive."""
        keep = []

        def arr(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a

        d = self._desc_no_src(arr)
        if self.src is not None and self.src.num > 0:
            _fill_src(d.src, self.src, arr)
        d._keep = keep
        return d

    def _desc_no_src(self, arr):
        d = ProblemDesc()
        d.ni, d.nj, d.nk = self.ni, self.nj, self.nk
        d.medium_type = self.medium_type
        d.coord = _ptr(arr(self.coord, np.float32))
        d.metric = _ptr(arr(self.metric, np.float32))
        d.medium = _ptr(arr(self.medium, np.float32))
        for a in range(3):
            for s in range(2):
                f = self.pml[a][s]
                if f:
                    d.pml[a][s] = PmlFace(1, int(f["num_layers"]), float(f["alpha_max"]),
                                          float(f["beta_max"]), float(f["ref_vel"]))
        d.free_top = int(self.free_top)
        d.dt, d.t0, d.nt_total = float(self.dt), float(self.t0), int(self.nt_total)
        if self.sta is not None and self.sta.num > 0:
            t = self.sta
            d.sta.num = t.num
            fc = t.flag_coord if t.flag_coord is not None else np.zeros(t.num, np.int32)
            d.sta.flag_coord = _ptr(arr(fc, np.int32))
            d.sta.flag_depth = _ptr(arr(t.flag_depth, np.int32))
            d.sta.loc = _ptr(arr(t.loc, np.float32))
        d.precision = int(self.precision)
        d.device = int(self.device)
        if self.visco is not None:
            v = self.visco
            vd = ViscoDesc(int(v["nmaxwell"]), float(v["fr"]), float(v["fmin"]), float(v["fmax"]))
            d._visco = vd
            d.visco = C.pointer(vd)
        return d


class LayerModelDesc(C.Structure):
    """cgfd_layer_model: a layered elastic-isotropic model (the reference's interface file)."""
    _fields_ = [("num_interfaces", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("x0", C.c_float), ("y0", C.c_float), ("dx", C.c_float), ("dy", C.c_float)] + \
        [(n, C.c_void_p) for n in ("elevation", "rho", "rho_grad", "rho_pow", "vp", "vp_grad", "vp_pow",
                                   "vs", "vs_grad", "vs_pow")]


CGFD_MEDIA_LOC, CGFD_MEDIA_HAR, CGFD_MEDIA_ARI = 0, 1, 2


def media_layer_gpu(coord, model, method=CGFD_MEDIA_LOC, device=0):
    """cgfd_media_layer_el_iso_gpu: medium [3, nz, ny, nx] (rho, lambda, mu) of the layered
    model (formats.LayerModel) on the grid coord [3, nz, ny, nx]."""
    _, nz, ny, nx = coord.shape
    keep = []

    def arr(a):
        a = np.ascontiguousarray(a, np.float32)
        keep.append(a)
        return a.ctypes.data
    d = LayerModelDesc(int(model.elevation.shape[0]), int(model.nx), int(model.ny), float(model.x0), float(model.y0),
                       float(model.dx), float(model.dy), *[arr(getattr(model, n)) for n in model.FIELDS])
    c = np.ascontiguousarray(coord, np.float32)
    out = np.zeros((3, nz, ny, nx), np.float32)
    check(lib().cgfd_media_layer_el_iso_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, C.byref(d), int(method),
                                            out.ctypes.data))
    return out


class LayerMediaDesc(C.Structure):
    """cgfd_layer_media: a layer file of any elastic type."""
    _fields_ = [("type", C.c_int), ("num_interfaces", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
                ("x0", C.c_float), ("y0", C.c_float), ("dx", C.c_float), ("dy", C.c_float),
                ("elevation", C.c_void_p), ("param", C.c_void_p)]


def media_layer_any_gpu(coord, model, medium_type, method=CGFD_MEDIA_LOC, device=0):
    """cgfd_media_layer_gpu: the medium of medium_type (CGFD_MEDIUM_ACOUSTIC_ISO / _ELASTIC_*:
    [2 | 3 | 6 | 22, nz, ny, nx] in the problem description's order) from the layer file model
    (formats.LayerMedia) on the grid coord [3, nz, ny, nx]."""
    _, nz, ny, nx = coord.shape
    el = np.ascontiguousarray(model.elevation, np.float32)
    pa = np.ascontiguousarray(model.param, np.float32)
    d = LayerMediaDesc(int(model.type), int(el.shape[0]), int(model.nx), int(model.ny), float(model.x0),
                       float(model.y0), float(model.dx), float(model.dy), el.ctypes.data, pa.ctypes.data)
    c = np.ascontiguousarray(coord, np.float32)
    nf = {1: 2, 2: 3, 3: 6, 4: 22}[int(medium_type)]
    out = np.zeros((nf, nz, ny, nx), np.float32)
    check(lib().cgfd_media_layer_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, C.byref(d), int(medium_type),
                                     int(method), out.ctypes.data))
    return out


class BinModelDesc(C.Structure):
    """cgfd_bin_model: the three volumes of a binary model, file order."""
    _fields_ = [("order", C.c_int * 3), ("size", C.c_int * 3), ("spacing", C.c_float * 3), ("origin", C.c_float * 3),
                ("rho", C.c_void_p), ("vp", C.c_void_p), ("vs", C.c_void_p)]


def media_bin_gpu(coord, model, device=0):
    """cgfd_media_bin_el_iso_gpu: medium [3, nz, ny, nx] (rho, lambda, mu) of the binary model
    (formats.BinModel) on the grid coord [3, nz, ny, nx]."""
    _, nz, ny, nx = coord.shape
    vols = [np.ascontiguousarray(v, np.float32) for v in (model.rho, model.vp, model.vs)]
    d = BinModelDesc((C.c_int * 3)(*model.order), (C.c_int * 3)(*model.size), (C.c_float * 3)(*model.spacing),
                     (C.c_float * 3)(*model.origin), vols[0].ctypes.data, vols[1].ctypes.data, vols[2].ctypes.data)
    c = np.ascontiguousarray(coord, np.float32)
    out = np.zeros((3, nz, ny, nx), np.float32)
    check(lib().cgfd_media_bin_el_iso_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, C.byref(d),
                                          out.ctypes.data))
    return out


class GridMediaDesc(C.Structure):
    """cgfd_grid_media: a grid model of elastic_isotropic type."""
    _fields_ = [("type", C.c_int), ("num_layers", C.c_int), ("ngz", C.c_void_p), ("nx", C.c_int), ("ny", C.c_int),
                ("x0", C.c_float), ("y0", C.c_float), ("dx", C.c_float), ("dy", C.c_float),
                ("elevation", C.c_void_p), ("param", C.c_void_p)]


def media_grid_gpu(coord, model, method=CGFD_MEDIA_LOC, device=0, medium_type=None):
    """cgfd_media_grid_el_iso_gpu: medium [3, nz, ny, nx] (rho, lambda, mu) of the grid model
    (formats.GridMedia) on the grid coord [3, nz, ny, nx]; with medium_type (CGFD_MEDIUM_ELASTIC_*)
    cgfd_media_grid_gpu: that medium in the problem description's order."""
    _, nz, ny, nx = coord.shape
    ngz = np.ascontiguousarray(model.ngz, np.int32)
    el = np.ascontiguousarray(model.elevation, np.float32)
    pa = np.ascontiguousarray(model.param, np.float32)
    d = GridMediaDesc(int(model.type), len(model.ngz), ngz.ctypes.data, int(model.nx), int(model.ny), float(model.x0),
                      float(model.y0), float(model.dx), float(model.dy), el.ctypes.data, pa.ctypes.data)
    c = np.ascontiguousarray(coord, np.float32)
    out = np.zeros((3, nz, ny, nx), np.float32)
    if medium_type is None:
        check(lib().cgfd_media_grid_el_iso_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, C.byref(d),
                                               int(method), out.ctypes.data))
        return out
    out = np.zeros(({2: 3, 3: 6, 4: 22}[int(medium_type)], nz, ny, nx), np.float32)
    check(lib().cgfd_media_grid_gpu(int(device), nx - 6, ny - 6, nz - 6, c.ctypes.data, C.byref(d), int(medium_type),
                                    int(method), out.ctypes.data))
    return out


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget", C.c_size_t), ("max_active", C.c_int), ("max_batch", C.c_int),
                ("steps_per_slice", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("pending", C.c_longlong), ("active", C.c_longlong), ("batches", C.c_longlong),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("cell_stages_per_s", C.c_double), ("source_steps_per_s", C.c_double),
                ("hbm_budget", C.c_size_t), ("hbm_in_use", C.c_size_t), ("hbm_peak", C.c_size_t)]


def problem_bytes(problem, shots=None):
    """(resident, peak) device bytes a Simulation(problem, shots) will hold (no device call)."""
    d = problem.desc()
    keep = []

    def arr(a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a
    sd = None
    n = 1
    if shots is not None:
        sd = (SourceDesc * len(shots))()
        for k, s in enumerate(shots):
            _fill_src(sd[k], s, arr)
        n = len(shots)
    r, pk = C.c_size_t(), C.c_size_t()
    check(lib().cgfd_problem_bytes(C.byref(d), n, C.addressof(sd) if sd is not None else None, C.byref(r),
                                   C.byref(pk)))
    return int(r.value), int(pk.value)


def _fill_src(ds, s, arr):
    ds.num = s.num
    ds.stf_given, ds.stf_length = s.stf_given, s.stf_length
    ds.stf_dt, ds.stf_nt = s.stf_dt, s.stf_nt
    ds.cmp_type, ds.mechanism_type = s.cmp_type, s.mechanism_type
    ds.loc_coord_type, ds.loc_3dim = s.loc_coord_type, s.loc_3dim
    ds.loc = _ptr(arr(s.loc, np.float32))
    ds.t_start = _ptr(arr(s.t_start, np.float32))
    ds.wavelet = _ptr(arr(s.wavelet, np.int32))
    ds.wavelet_coefs = _ptr(arr(s.wavelet_coefs, np.float32))
    ds.cmp = _ptr(arr(s.cmp, np.float32))
    ds.cmp_values = _ptr(arr(s.cmp_values, np.float32))


_lib = None


def lib():
    """Load libcgfd_b200.so from the package build folder; there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(lib_path):
        raise RuntimeError(f"{lib_path} is missing: build it with `make -C gpu-cgfd3d-elastic_b200` "
                           "(or __graft_entry__.build())")
    L = C.CDLL(lib_path)
    P = C.c_void_p
    sig = {
        "cgfd_version": (C.c_int, []),
        "cgfd_last_error": (C.c_char_p, []),
        "cgfd_problem_create": (C.c_int, [C.POINTER(ProblemDesc), C.POINTER(P)]),
        "cgfd_batch_create": (C.c_int, [C.POINTER(ProblemDesc), C.c_int, P, C.POINTER(P)]),
        "cgfd_num_shots": (C.c_int, [P]),
        "cgfd_get_wavefield_shot": (C.c_int, [P, C.c_int, P]),
        "cgfd_set_wavefield_shot": (C.c_int, [P, C.c_int, P]),
        "cgfd_problem_destroy": (C.c_int, [P]),
        "cgfd_run": (C.c_int, [P, C.c_int]),
        "cgfd_enqueue_steps": (C.c_int, [P, C.c_int]),
        "cgfd_synchronize": (C.c_int, [P]),
        "cgfd_check_wait_bound": (C.c_int, [P]),
        "cgfd_current_step": (C.c_int, [P]),
        "cgfd_set_step": (C.c_int, [P, C.c_int]),
        "cgfd_get_seismograms": (C.c_int, [P, P]),
        "cgfd_num_stations": (C.c_int, [P]),
        "cgfd_station_info": (C.c_int, [P, P, P]),
        "cgfd_get_wavefield": (C.c_int, [P, P]),
        "cgfd_get_peak_motion": (C.c_int, [P, C.c_int, P]),
        "cgfd_set_line_receivers": (C.c_int, [P, C.c_int, P]),
        "cgfd_set_tile_shape": (C.c_int, [P, C.c_int]),
        "cgfd_get_tile_shape": (C.c_int, [P]),
        "cgfd_set_shot_group": (C.c_int, [P, C.c_int]),
        "cgfd_get_shot_group": (C.c_int, [P]),
        "cgfd_get_line_seismograms": (C.c_int, [P, P]),
        "cgfd_set_slices": (C.c_int, [P, C.c_int, P, C.c_int, P, C.c_int, P, C.c_int]),
        "cgfd_get_slices": (C.c_int, [P, C.c_int, C.c_int, P]),
        "cgfd_get_wavefield_box": (C.c_int, [P, C.c_int, P, P, P, P]),
        "cgfd_set_wavefield": (C.c_int, [P, P]),
        "cgfd_device_bytes": (C.c_size_t, [P]),
        "cgfd_stream": (P, [P]),
        "cgfd_set_graph_mode": (C.c_int, [P, C.c_int]),
        "cgfd_set_zchunk": (C.c_int, [P, C.c_int]),
        "cgfd_get_zchunk": (C.c_int, [P]),
        "cgfd_autotune": (C.c_int, [P, C.c_int, C.POINTER(C.c_int)]),
        "cgfd_set_timing": (C.c_int, [P, C.c_int]),
        "cgfd_set_bulk_variant": (C.c_int, [P, C.c_int]),
        "cgfd_get_timing": (C.c_int, [P, P, P, P, C.c_int]),
        "cgfd_fill_ghosts": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P]),
        "cgfd_visco_gmb": (C.c_int, [P, C.c_longlong, P, P, P, P, P, P, P, P, P]),
        "cgfd_metric_calc": (C.c_int, [C.c_int, C.c_int, C.c_int, P, P]),
        "cgfd_metric_calc_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P]),
        "cgfd_media_layer_el_iso_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P, C.c_int, P]),
        "cgfd_media_layer_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P, C.c_int, C.c_int, P]),
        "cgfd_media_bin_el_iso_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P, P]),
        "cgfd_media_grid_el_iso_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P, C.c_int, P]),
        "cgfd_media_grid_gpu": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, P, P, C.c_int, C.c_int, P]),
        "cgfd_dt_estimate": (C.c_int, [C.POINTER(ProblemDesc), C.c_double, C.POINTER(C.c_double)]),
        "cgfd_keep_three_digits": (C.c_double, [C.c_double]),
        "cgfd_problem_bytes": (C.c_int, [C.POINTER(ProblemDesc), C.c_int, P, C.POINTER(C.c_size_t),
                                         C.POINTER(C.c_size_t)]),
        "cgfd_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(P)]),
        "cgfd_server_submit": (C.c_int, [P, C.POINTER(ProblemDesc), C.POINTER(C.c_longlong)]),
        "cgfd_server_poll": (C.c_int, [P, C.c_longlong, P, C.POINTER(C.c_int)]),
        "cgfd_server_wait": (C.c_int, [P, C.c_longlong, C.c_double]),
        "cgfd_server_get_stats": (C.c_int, [P, C.POINTER(ServerStats)]),
        "cgfd_server_destroy": (C.c_int, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise CgfdError(rc, lib().cgfd_last_error().decode())
    return rc


class Simulation:
    """Device state of one forward simulation (cgfd_problem_create ... destroy), or of a batch
    of shots sharing one grid (cgfd_batch_create) when `shots` (list of Sources) is given."""

    def __init__(self, problem: Problem, shots=None):
        self.problem = problem
        self._desc = problem.desc()
        h = C.c_void_p()
        self.nshot = 1
        if shots is None:
            check(lib().cgfd_problem_create(C.byref(self._desc), C.byref(h)))
        else:
            keep = []

            def arr(a, dt):
                if a is None:
                    return None
                a = np.ascontiguousarray(a, dtype=dt)
                keep.append(a)
                return a
            sd = (SourceDesc * len(shots))()
            for n, s in enumerate(shots):
                _fill_src(sd[n], s, arr)
            self._shots = (sd, keep)
            self.nshot = len(shots)
            check(lib().cgfd_batch_create(C.byref(self._desc), self.nshot, C.addressof(sd), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().cgfd_problem_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps=-1):
        check(lib().cgfd_run(self.h, int(nsteps)))

    def enqueue(self, nsteps):
        check(lib().cgfd_enqueue_steps(self.h, int(nsteps)))

    def synchronize(self):
        check(lib().cgfd_synchronize(self.h))

    def autotune(self, steps=4):
        """cgfd_autotune: fastest z-chunk length of this problem (state reset to step 0)."""
        c = C.c_int()
        check(lib().cgfd_autotune(self.h, int(steps), C.byref(c)))
        return c.value

    def check_wait_bound(self):
        """cgfd_check_wait_bound: (status, message) of one device pipeline wait that nothing
        completes; a working bound gives CGFD_ERR_CUDA and leaves the problem usable."""
        rc = lib().cgfd_check_wait_bound(self.h)
        return rc, lib().cgfd_last_error().decode()

    @property
    def step(self):
        return lib().cgfd_current_step(self.h)

    def set_step(self, it):
        check(lib().cgfd_set_step(self.h, int(it)))

    @property
    def num_stations(self):
        return lib().cgfd_num_stations(self.h)

    def seismograms(self):
        """[nsta, 9, nt_total], or [nshot, nsta, 9, nt_total] for a batch."""
        n = self.num_stations
        out = np.zeros((self.nshot, max(n, 0), 9, self.problem.nt_total), np.float32)
        check(lib().cgfd_get_seismograms(self.h, out.ctypes.data))
        return out[0] if self.nshot == 1 else out

    def wavefield_box(self, start, count, stride=(1, 1, 1), shot=0):
        """[9, count_z, count_y, count_x] strided sub-box of w_pre (0-based physical indices)."""
        a = [np.ascontiguousarray(v, np.int32) for v in (start, count, stride)]
        out = np.zeros((9, int(count[2]), int(count[1]), int(count[0])), np.float32)
        check(lib().cgfd_get_wavefield_box(self.h, int(shot), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data,
                                           out.ctypes.data))
        return out

    def set_line_receivers(self, ijk):
        """cgfd_set_line_receivers: grid points [n, 3] (physical 0-based i, j, k)."""
        a = np.ascontiguousarray(np.asarray(ijk, np.int32).reshape(-1, 3))
        self._line_n = a.shape[0]
        check(lib().cgfd_set_line_receivers(self.h, int(a.shape[0]), a.ctypes.data))

    def line_seismograms(self):
        """[npts, 9, nt_total], or [nshot, npts, 9, nt_total] for a batch."""
        n = getattr(self, "_line_n", 0)
        out = np.zeros((self.nshot, n, 9, self.problem.nt_total), np.float32)
        check(lib().cgfd_get_line_seismograms(self.h, out.ctypes.data))
        return out[0] if self.nshot == 1 else out

    def set_slices(self, ix=(), iy=(), iz=(), ring_steps=16):
        """cgfd_set_slices: x / y / z plane indices (physical 0-based), device ring of steps."""
        a = [np.ascontiguousarray(np.asarray(v, np.int32)) for v in (ix, iy, iz)]
        self._slices = tuple(len(v) for v in a)
        check(lib().cgfd_set_slices(self.h, len(a[0]), a[0].ctypes.data, len(a[1]), a[1].ctypes.data,
                                    len(a[2]), a[2].ctypes.data, int(ring_steps)))

    def slices(self, it, shot=0):
        """(x [nx, 9, nk, nj], y [ny, 9, nk, ni], z [nz, 9, nj, ni]) planes of step `it`."""
        p = self.problem
        nx, ny, nz = self._slices
        sizes = [nx * 9 * p.nk * p.nj, ny * 9 * p.nk * p.ni, nz * 9 * p.nj * p.ni]
        out = np.zeros(sum(sizes), np.float32)
        check(lib().cgfd_get_slices(self.h, int(shot), int(it), out.ctypes.data))
        a, b = sizes[0], sizes[0] + sizes[1]
        return (out[:a].reshape(nx, 9, p.nk, p.nj), out[a:b].reshape(ny, 9, p.nk, p.ni),
                out[b:].reshape(nz, 9, p.nj, p.ni))

    def peak_motion(self, shot=0):
        """[15, ny, nx] free-surface peak ground motion (PGV, PGVh, PGVx..z, PGA.., PGD..)."""
        p = self.problem
        out = np.zeros((15, p.nj + 6, p.ni + 6), np.float32)
        check(lib().cgfd_get_peak_motion(self.h, int(shot), out.ctypes.data))
        return out

    def wavefield(self, shot=0):
        p = self.problem
        out = np.zeros((9,) + ref_shape(p.ni, p.nj, p.nk), np.float32)
        check(lib().cgfd_get_wavefield_shot(self.h, int(shot), out.ctypes.data))
        return out

    def set_wavefield(self, w, shot=0):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().cgfd_set_wavefield_shot(self.h, int(shot), w.ctypes.data))

    def device_bytes(self):
        return int(lib().cgfd_device_bytes(self.h))

    def set_graph_mode(self, on):
        check(lib().cgfd_set_graph_mode(self.h, int(on)))

    def set_zchunk(self, nzc):
        check(lib().cgfd_set_zchunk(self.h, int(nzc)))

    @property
    def zchunk(self):
        return lib().cgfd_get_zchunk(self.h)

    def set_tile_shape(self, shape):
        check(lib().cgfd_set_tile_shape(self.h, int(shape)))

    @property
    def tile_shape(self):
        return lib().cgfd_get_tile_shape(self.h)

    def set_shot_group(self, group):
        check(lib().cgfd_set_shot_group(self.h, int(group)))

    @property
    def shot_group(self):
        return lib().cgfd_get_shot_group(self.h)

    def set_bulk_variant(self, tma):
        check(lib().cgfd_set_bulk_variant(self.h, int(tma)))

    def set_timing(self, on):
        check(lib().cgfd_set_timing(self.h, int(on)))

    def timing(self, reset=False):
        """{kind: (total_ms, launches)} per kernel kind plus "bulk" (all stages) and the
        total number of library kernel launches."""
        ms = np.zeros(8, np.float64)
        cnt = np.zeros(8, np.int64)
        tot = C.c_longlong()
        check(lib().cgfd_get_timing(self.h, ms.ctypes.data, cnt.ctypes.data, C.addressof(tot), int(reset)))
        kinds = ("bulk_s0", "bulk_s1", "bulk_s2", "bulk_s3", "surface", "source", "recv", "wave_scale")
        out = {k: (float(ms[n]), int(cnt[n])) for n, k in enumerate(kinds)}
        out["bulk"] = (float(ms[:4].sum()), int(cnt[:4].sum()))
        out["launches"] = int(tot.value)
        return out

    @property
    def stream(self):
        return lib().cgfd_stream(self.h)


class Server:
    """Serving loop on one GPU (cgfd_server_*): submit problems, poll/wait for seismograms.
    The model arrays of a submitted problem must stay alive until its request completes;
    Server keeps a reference to each submitted description until its result is taken."""

    def __init__(self, device=0, hbm_budget=0, max_active=4, max_batch=8, steps_per_slice=50):
        o = ServerOpts(int(device), int(hbm_budget), int(max_active), int(max_batch), int(steps_per_slice))
        h = C.c_void_p()
        check(lib().cgfd_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self._live = {}

    def submit(self, problem):
        d = problem.desc()
        rid = C.c_longlong()
        check(lib().cgfd_server_submit(self.h, C.byref(d), C.byref(rid)))
        self._live[rid.value] = (d, problem)
        return rid.value

    def poll(self, rid):
        """None while queued/running; the [nsta, 9, nt_total] seismograms once done."""
        nsta = C.c_int()
        rc = lib().cgfd_server_poll(self.h, rid, None, C.byref(nsta))
        if rc == CGFD_ERR_BUSY:
            return None
        check(rc)
        p = self._live[rid][1]
        out = np.zeros((nsta.value, 9, p.nt_total), np.float32)
        check(lib().cgfd_server_poll(self.h, rid, out.ctypes.data, C.byref(nsta)))
        del self._live[rid]
        return out

    def wait(self, rid, timeout=-1.0):
        rc = lib().cgfd_server_wait(self.h, rid, float(timeout))
        if rc == CGFD_ERR_BUSY:
            return None
        check(rc)
        return self.poll(rid)

    def stats(self):
        st = ServerStats()
        check(lib().cgfd_server_get_stats(self.h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().cgfd_server_destroy(self.h)
            self.h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def visco_gmb(visco, lam, mu, qp, qs):
    """cgfd_visco_gmb: the GMB fit of n points. Returns (lam_u, mu_u, Ylam [nmax, n], Ymu [nmax, n],
    wl [nmax])."""
    lam, mu, qp, qs = (np.ascontiguousarray(np.ravel(a), np.float32) for a in (lam, mu, qp, qs))
    n, nm = lam.size, int(visco["nmaxwell"])
    vd = ViscoDesc(nm, float(visco["fr"]), float(visco["fmin"]), float(visco["fmax"]))
    lu, mu_u = np.zeros(n, np.float32), np.zeros(n, np.float32)
    yl, ym = np.zeros((max(nm, 1), n), np.float32), np.zeros((max(nm, 1), n), np.float32)
    wl = np.zeros(max(nm, 1), np.float32)
    check(lib().cgfd_visco_gmb(C.addressof(vd), n, lam.ctypes.data, mu.ctypes.data, qp.ctypes.data, qs.ctypes.data,
                               lu.ctypes.data, mu_u.ctypes.data, yl.ctypes.data, ym.ctypes.data, wl.ctypes.data))
    return lu, mu_u, yl, ym, wl
