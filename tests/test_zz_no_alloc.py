"""cgfd_get_wavefield_shot_noalloc (static device scratch, no allocation) against the existing
cgfd_get_wavefield_shot, through the C ABI.

Tolerance: exact. Both copy the same device values into the reference layout, so the two
outputs must be identical. Two calls in a row share the one scratch array.
"""
import ctypes as C

import numpy as np
import pytest

from cgfd_b200 import Simulation, lib, synth
from helpers import small_problem

pytestmark = pytest.mark.gpu

SCRATCH_FLOATS = 1 << 20


def _noalloc():
    fn = lib().cgfd_get_wavefield_shot_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    return fn


def test_noalloc_matches_existing_entry_point_twice():
    p = small_problem("vti", ni=44, nj=40, nk=34, nsteps=30, nsrc=0, seed=9)
    rng = np.random.default_rng(4)
    shots = [synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(600.0, 1200.0), fc_range=(3.0, 4.0),
                              stf_length=p.nt_total * p.dt) for _ in range(2)]
    sim = Simulation(p, shots=shots)
    sim.run(25)
    fn = _noalloc()
    for shot in (0, 1):  # two calls in a row through the shared scratch
        ref = sim.wavefield(shot)
        out = np.full_like(ref, np.nan)
        assert fn(sim.h, shot, out.ctypes.data) == 0
        assert np.abs(ref).max() > 0
        assert np.array_equal(out, ref)


def test_noalloc_chunks_over_many_planes():
    """A grid whose reference volume is several times the scratch: the copy goes chunk by
    chunk and still equals the existing entry point."""
    p = small_problem("iso", ni=200, nj=180, nk=60, nsteps=6, npml=4, sta_grid=None, seed=2)
    assert (p.ni + 6) * (p.nj + 6) * (p.nk + 6) > 2 * SCRATCH_FLOATS
    sim = Simulation(p)
    sim.run(5)
    ref = sim.wavefield()
    out = np.zeros_like(ref)
    assert _noalloc()(sim.h, 0, out.ctypes.data) == 0
    assert np.array_equal(out, ref)


def _device_memory(device=0):
    """(pool reserved bytes, pool used bytes, free device bytes) of `device` through the CUDA
    driver API: the default memory pool the library allocates from, and cuMemGetInfo of the
    primary context the library made current on this thread."""
    cu = C.CDLL("libcuda.so.1")
    dev = C.c_int()
    assert cu.cuDeviceGet(C.byref(dev), device) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    reserved, used = C.c_uint64(), C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, 5, C.byref(reserved)) == 0  # CU_MEMPOOL_ATTR_RESERVED_MEM_CURRENT
    assert cu.cuMemPoolGetAttribute(pool, 7, C.byref(used)) == 0      # CU_MEMPOOL_ATTR_USED_MEM_CURRENT
    free, total = C.c_size_t(), C.c_size_t()
    assert cu.cuMemGetInfo_v2(C.byref(free), C.byref(total)) == 0
    return reserved.value, used.value, free.value


def test_noalloc_takes_no_device_memory():
    """The property the entry point exists for: with a problem resident, further calls change
    neither the memory pool's reserved / used bytes nor the device's free memory (the plain
    cgfd_get_wavefield_shot takes a wavefield component from the pool for its duration)."""
    p = small_problem("iso", ni=120, nj=100, nk=50, nsteps=6, npml=4, sta_grid=None, seed=5)
    sim = Simulation(p)
    sim.run(4)
    ref = sim.wavefield()
    out = np.zeros_like(ref)
    fn = _noalloc()
    assert fn(sim.h, 0, out.ctypes.data) == 0  # first call after create
    for _ in range(2):
        before = _device_memory(p.device)
        assert fn(sim.h, 0, out.ctypes.data) == 0
        after = _device_memory(p.device)
        assert after == before, (before, after)
        assert np.array_equal(out, ref)


def test_noalloc_rejects_bad_arguments():
    p = small_problem("iso", nsteps=4, nsrc=0, sta_grid=None)
    sim = Simulation(p)
    out = np.zeros((9, p.nk + 6, p.nj + 6, p.ni + 6), np.float32)
    fn = _noalloc()
    assert fn(sim.h, 1, out.ctypes.data) == -1  # one shot only
    assert fn(None, 0, out.ctypes.data) == -1


def test_noalloc_rejects_planes_beyond_the_scratch():
    """(ni+6)*(nj+6) above 2^20 floats: refused with CGFD_ERR_INVALID and a message."""
    p = small_problem("iso", ni=1030, nj=1020, nk=10, nsteps=2, npml=2, nsrc=0, sta_grid=None)
    assert (p.ni + 6) * (p.nj + 6) > SCRATCH_FLOATS
    sim = Simulation(p)
    out = np.zeros((9, p.nk + 6, p.nj + 6, p.ni + 6), np.float32)
    assert _noalloc()(sim.h, 0, out.ctypes.data) == -1
    assert b"exceeds the no-allocation scratch" in lib().cgfd_last_error()
