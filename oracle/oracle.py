"""ctypes wrapper of the CPU oracle (oracle/_build/libcgfd_oracle.so).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
--impl reference legs use it, always as the checker or the timed CPU reference, never as
part of the product path.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libcgfd_oracle.so")
_lib = None


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        for name, res, args in [
            ("orc_error", C.c_char_p, []),
            ("orc_create", P, [P, C.c_int]),
            ("orc_destroy", None, [P]),
            ("orc_run", C.c_int, [P, C.c_int]),
            ("orc_set_step", C.c_int, [P, C.c_int]),
            ("orc_num_stations", C.c_int, [P]),
            ("orc_get_seismograms", C.c_int, [P, P]),
            ("orc_get_wavefield", C.c_int, [P, P]),
            ("orc_get_peak_motion", C.c_int, [P, P]),
            ("orc_locate_points", C.c_int, [C.c_int, C.c_int, C.c_int, P, C.c_int, P, P, P, P]),
            ("orc_set_wavefield", C.c_int, [P, P]),
            ("orc_pml_coefs", C.c_int, [P, C.c_int, C.c_int, P, P, P]),
            ("orc_free_mats", C.c_int, [P, P, P]),
            ("orc_src_info", C.c_int, [P, P, P, P, P, P, P, P]),
            ("orc_coord_ghosts", C.c_int, [C.c_int, C.c_int, C.c_int, P]),
            ("orc_metric_calc", C.c_int, [C.c_int, C.c_int, C.c_int, P, P]),
            ("orc_metric_calc_f64", C.c_int, [C.c_int, C.c_int, C.c_int, P, P]),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def metric_fp32(coord):
    """gd_curv_metric_cal restated in FP32 (the reference's precision)."""
    _, nz, ny, nx = coord.shape
    out = np.zeros((10, nz, ny, nx), np.float32)
    c = np.ascontiguousarray(coord, np.float32)
    lib().orc_metric_calc(nx - 6, ny - 6, nz - 6, c.ctypes.data, out.ctypes.data)
    return out


def locate_points(coord, xyz, depth_flag=None):
    """(idx [n,3] global physical index or -1000, inc [n,3] shift) of points given by physical
    coordinates, located like the reference (nearest point, cell test, 101^3 sampling)."""
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    q = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    n = q.shape[0]
    flags = np.ascontiguousarray(depth_flag if depth_flag is not None else np.zeros(n), np.int32)
    idx = np.zeros((n, 3), np.int32)
    inc = np.zeros((n, 3), np.float32)
    if lib().orc_locate_points(nx - 6, ny - 6, nz - 6, c.ctypes.data, n, q.ctypes.data, flags.ctypes.data,
                               idx.ctypes.data, inc.ctypes.data) != 0:
        raise RuntimeError("oracle: " + lib().orc_error().decode())
    return idx, inc


def fill_ghosts(coord):
    _, nz, ny, nx = coord.shape
    lib().orc_coord_ghosts(nx - 6, ny - 6, nz - 6, coord.ctypes.data)


class Oracle:
    """One oracle simulation over a cgfd_b200 Problem (same description struct)."""

    def __init__(self, problem, fp64=False):
        self.problem = problem
        self._desc = problem.desc()
        h = lib().orc_create(C.addressof(self._desc), 1 if fp64 else 0)
        if not h:
            raise RuntimeError("oracle: " + lib().orc_error().decode())
        self.h = h

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, nsteps=-1):
        rc = lib().orc_run(self.h, int(nsteps))
        if rc:
            raise RuntimeError("oracle: " + lib().orc_error().decode())

    def set_step(self, it):
        lib().orc_set_step(self.h, int(it))

    @property
    def num_stations(self):
        return lib().orc_num_stations(self.h)

    def seismograms(self):
        out = np.zeros((self.num_stations, 9, self.problem.nt_total), np.float32)
        lib().orc_get_seismograms(self.h, out.ctypes.data)
        return out

    def peak_motion(self):
        """[15, ny, nx] free-surface peak ground motion (PGV, PGVh, PGVx..z, PGA.., PGD..)."""
        p = self.problem
        out = np.zeros((15, p.nj + 6, p.ni + 6), np.float32)
        lib().orc_get_peak_motion(self.h, out.ctypes.data)
        return out

    def wavefield(self):
        p = self.problem
        out = np.zeros((9, p.nk + 6, p.nj + 6, p.ni + 6), np.float32)
        lib().orc_get_wavefield(self.h, out.ctypes.data)
        return out

    def set_wavefield(self, w):
        w = np.ascontiguousarray(w, np.float32)
        lib().orc_set_wavefield(self.h, w.ctypes.data)
