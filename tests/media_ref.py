"""ctypes access to the reference's own media discretisation (oracle/_ref/libref_media.so, built
from the reference's src/media sources by oracle/Makefile.ref). Test infrastructure."""
import ctypes as C
import os
import tempfile

import numpy as np

from cgfd_b200 import formats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_media.so")
METHODS = {0: b"loc", 1: b"har", 2: b"ari"}


def available():
    return os.path.exists(LIB)


def layer2model_el_iso(coord, model, method=0):
    """medium [3, nz, ny, nx] = rho, lambda, mu by media_layer2model_el_iso on the grid coord."""
    L = C.CDLL(LIB)
    fn = L.ref_media_layer2model_el_iso
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 6 + [C.c_size_t] * 3 + [C.c_char_p, C.c_char_p]
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    lam, mu, rho = (np.zeros((nz, ny, nx), np.float32) for _ in range(3))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.lay")
        formats.write_layer_file(path, model)
        rc = fn(lam.ctypes.data, mu.ctypes.data, rho.ctypes.data, c[0].ctypes.data, c[1].ctypes.data,
                c[2].ctypes.data, nx, ny, nz, path.encode(), METHODS[method])
    assert rc == 0
    return np.stack([rho, lam, mu])


def layer2model(coord, model, medium_type, method=0):
    """The medium of medium_type (1 acoustic [rho kappa], 2 iso [rho lambda mu], 3 VTI [rho c11 c13
    c33 c55 c66], 4 21-Cij [rho c11 ... c66]) from the layer file model (formats.LayerMedia) by the
    reference's media_layer2model_ac_iso / _el_iso / _el_vti / _el_aniso on the grid coord."""
    L = C.CDLL(LIB)
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.lay")
        formats.write_layer_media_file(path, model)
        if medium_type == 1:
            fn = L.ref_media_layer2model_ac_iso
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p] * 5 + [C.c_size_t] * 3 + [C.c_char_p, C.c_char_p]
            rho, kappa = (np.zeros((nz, ny, nx), np.float32) for _ in range(2))
            rc = fn(rho.ctypes.data, kappa.ctypes.data, c[0].ctypes.data, c[1].ctypes.data, c[2].ctypes.data,
                    nx, ny, nz, path.encode(), METHODS[method])
            out = np.stack([rho, kappa])
        elif medium_type == 2:
            fn = L.ref_media_layer2model_el_iso
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p] * 6 + [C.c_size_t] * 3 + [C.c_char_p, C.c_char_p]
            lam, mu, rho = (np.zeros((nz, ny, nx), np.float32) for _ in range(3))
            rc = fn(lam.ctypes.data, mu.ctypes.data, rho.ctypes.data, c[0].ctypes.data, c[1].ctypes.data,
                    c[2].ctypes.data, nx, ny, nz, path.encode(), METHODS[method])
            out = np.stack([rho, lam, mu])
        elif medium_type == 3:
            fn = L.ref_media_layer2model_el_vti
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p] * 9 + [C.c_size_t] * 3 + [C.c_char_p, C.c_char_p]
            f = [np.zeros((nz, ny, nx), np.float32) for _ in range(6)]  # rho c11 c33 c55 c66 c13
            rc = fn(*[a.ctypes.data for a in f], c[0].ctypes.data, c[1].ctypes.data, c[2].ctypes.data, nx, ny, nz,
                    path.encode(), METHODS[method])
            out = np.stack([f[0], f[1], f[5], f[2], f[3], f[4]])
        else:
            fn = L.ref_media_layer2model_el_aniso
            fn.restype = C.c_int
            fn.argtypes = [C.c_void_p] * 4 + [C.c_size_t] * 3 + [C.c_char_p, C.c_char_p]
            f = [np.zeros((nz, ny, nx), np.float32) for _ in range(22)]
            ptrs = (C.c_void_p * 22)(*[a.ctypes.data for a in f])
            rc = fn(ptrs, c[0].ctypes.data, c[1].ctypes.data, c[2].ctypes.data, nx, ny, nz, path.encode(),
                    METHODS[method])
            out = np.stack(f)
    assert rc == 0
    return out


def bin2model_el_iso(coord, model):
    """medium [3, nz, ny, nx] = rho, lambda, mu by the reference's media_bin2model_el_iso from the
    binary model (formats.BinModel) on the grid coord, with the grid's x / y range as
    gd_curv_set_minmax computes it (every point, ghosts included)."""
    L = C.CDLL(LIB)
    fn = L.ref_media_bin2model_el_iso
    fn.restype = C.c_int
    fn.argtypes = ([C.c_void_p] * 6 + [C.c_size_t] * 3 + [C.c_float] * 4 + [C.c_void_p] * 4 +
                   [C.c_char_p] * 3)
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    rho, lam, mu = (np.zeros((nz, ny, nx), np.float32) for _ in range(3))
    order = (C.c_int * 3)(*model.order)
    size = (C.c_int * 3)(*model.size)
    spacing = (C.c_float * 3)(*model.spacing)
    origin = (C.c_float * 3)(*model.origin)
    with tempfile.TemporaryDirectory() as d:
        paths = []
        for name, v in (("rho", model.rho), ("vp", model.vp), ("vs", model.vs)):
            path = os.path.join(d, name + ".bin")
            np.ascontiguousarray(v, np.float32).tofile(path)
            paths.append(path.encode())
        rc = fn(rho.ctypes.data, lam.ctypes.data, mu.ctypes.data, c[0].ctypes.data, c[1].ctypes.data,
                c[2].ctypes.data, nx, ny, nz, float(c[0].min()), float(c[0].max()), float(c[1].min()),
                float(c[1].max()), order, size, spacing, origin, *paths)
    assert rc == 0
    return np.stack([rho, lam, mu])


def grid2model_el_iso(coord, model, method=0):
    """medium [3, nz, ny, nx] = rho, lambda, mu by the reference's media_grid2model_el_iso from the
    grid model (formats.GridMedia) on the grid coord, with the grid's x / y range as
    gd_curv_set_minmax computes it."""
    L = C.CDLL(LIB)
    fn = L.ref_media_grid2model_el_iso
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 6 + [C.c_int] * 3 + [C.c_float] * 4 + [C.c_char_p, C.c_char_p]
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    rho, lam, mu = (np.zeros((nz, ny, nx), np.float32) for _ in range(3))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.grd")
        formats.write_grid_media_file(path, model)
        rc = fn(rho.ctypes.data, lam.ctypes.data, mu.ctypes.data, c[0].ctypes.data, c[1].ctypes.data,
                c[2].ctypes.data, nx, ny, nz, float(c[0].min()), float(c[0].max()), float(c[1].min()),
                float(c[1].max()), path.encode(), METHODS[method])
    assert rc == 0
    return np.stack([rho, lam, mu])


def grid2model(coord, model, medium_type, method=0):
    """The medium of medium_type (2 iso, 3 VTI [rho c11 c13 c33 c55 c66], 4 21-Cij [rho c11 ... c66])
    from the grid model (formats.GridMedia) by the reference's media_grid2model_el_iso / _el_vti /
    _el_aniso on the grid coord."""
    if medium_type == 2:
        return grid2model_el_iso(coord, model, method)
    L = C.CDLL(LIB)
    fn = L.ref_media_grid2model_el_vti if medium_type == 3 else L.ref_media_grid2model_el_aniso
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 4 + [C.c_int] * 3 + [C.c_float] * 4 + [C.c_char_p, C.c_char_p]
    _, nz, ny, nx = coord.shape
    c = np.ascontiguousarray(coord, np.float32)
    nf = 6 if medium_type == 3 else 22
    f = [np.zeros((nz, ny, nx), np.float32) for _ in range(nf)]
    ptrs = (C.c_void_p * nf)(*[a.ctypes.data for a in f])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "model.grd")
        formats.write_grid_media_file(path, model)
        rc = fn(ptrs, c[0].ctypes.data, c[1].ctypes.data, c[2].ctypes.data, nx, ny, nz, float(c[0].min()),
                float(c[0].max()), float(c[1].min()), float(c[1].max()), path.encode(), METHODS[method])
    assert rc == 0
    if medium_type == 3:  # rho c11 c33 c55 c66 c13 -> the description's rho c11 c13 c33 c55 c66
        return np.stack([f[0], f[1], f[5], f[2], f[3], f[4]])
    return np.stack(f)
