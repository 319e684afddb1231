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
