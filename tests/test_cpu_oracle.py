"""CPU checks of the oracle and the host setup (no GPU): math known-answer tests."""
import numpy as np
import pytest

from cgfd_b200 import synth, Problem, CGFD_MEDIUM_ELASTIC_ISO
from oracle.oracle import Oracle, metric_fp32, fill_ghosts
from helpers import small_problem, rel_l2


def _cart_coord(ni, nj, nk, dx, dy, dz):
    c = np.zeros((3, nk + 6, nj + 6, ni + 6), np.float32)
    c[0, 3:-3, 3:-3, 3:-3] = (np.arange(ni) * dx)[None, None, :]
    c[1, 3:-3, 3:-3, 3:-3] = (np.arange(nj) * dy)[None, :, None]
    c[2, 3:-3, 3:-3, 3:-3] = (np.arange(nk) * dz)[:, None, None]
    fill_ghosts(c)
    return c


def test_cartesian_metric_kat():
    """Flat Cartesian grid: metrics = diag(1/dx,1/dy,1/dz), jac = dx*dy*dz (oracle FP32, product FP64)."""
    dx, dy, dz = 100.0, 80.0, 50.0
    c = _cart_coord(12, 11, 10, dx, dy, dz)
    for m in (metric_fp32(c), synth.metrics(c)):
        sl = (slice(None),) * 1 + (slice(3, -3),) * 3
        jac = m[0][sl[1:]]
        # the centered 7-point op of fd_t.cu:162 returns 1.00004 * slope on linear fields
        s = 2 * (0.7709 - 2 * 0.1667 + 3 * 0.02084)
        assert np.allclose(jac, dx * dy * dz * s ** 3, rtol=1e-5)
        assert np.allclose(m[1][sl[1:]], 1 / (dx * s), rtol=1e-5)
        assert np.allclose(m[5][sl[1:]], 1 / (dy * s), rtol=1e-5)
        assert np.allclose(m[9][sl[1:]], 1 / (dz * s), rtol=1e-5)
        for off in (2, 3, 4, 6, 7, 8):
            assert np.abs(m[off][sl[1:]]).max() < 1e-6 / dx  # FP32 rounding of the coordinates


def test_metric_fp32_vs_fp64_curvilinear():
    c = synth.curvilinear_grid(30, 28, 20, 100.0, seed=4)
    a, b = metric_fp32(c), synth.metrics(c)
    assert rel_l2(a[:, 3:-3, 3:-3, 3:-3], b[:, 3:-3, 3:-3, 3:-3]) < 1e-5


def test_fp32_oracle_close_to_fp64_oracle():
    p = small_problem("iso", nsteps=40)
    a, b = Oracle(p), Oracle(p, fp64=True)
    a.run()
    b.run()
    assert rel_l2(a.seismograms(), b.seismograms()) < 1e-4


def test_linear_field_zero_rhs_interior():
    """DRP operators are exact on constant fields: a uniform stress state in a homogeneous
    Cartesian box without boundaries stays (numerically) unchanged away from the edges."""
    ni = nj = nk = 24
    c = _cart_coord(ni, nj, nk, 100.0, 100.0, 100.0)
    m = metric_fp32(c)
    med = np.zeros((3,) + c.shape[1:], np.float32)
    med[0], med[1], med[2] = 2500.0, 2500.0 * (4000 ** 2 - 2 * 2300 ** 2), 2500.0 * 2300 ** 2
    p = Problem(ni=ni, nj=nj, nk=nk, medium_type=CGFD_MEDIUM_ELASTIC_ISO, coord=c, metric=m, medium=med,
                dt=0.005, nt_total=3, free_top=0)
    w = np.zeros((9,) + c.shape[1:], np.float32)
    w[3, 3:-3, 3:-3, 3:-3] = 1e6
    o = Oracle(p)
    o.set_wavefield(w)
    o.run(1)
    out = o.wavefield()
    inner = (slice(10, -10),) * 3
    assert np.allclose(out[3][inner], 1e6, rtol=1e-6)
    assert np.abs(out[:3][(slice(None),) + inner]).max() < 1e-6


def test_rk4_linear_ode_through_pml_aux():
    """The RK combine reproduces classic RK4: a pointwise decay aux' = -A aux in a PML
    face with zero wavefield keeps the aux at zero, and the wavefield at zero."""
    p = small_problem("iso", nsrc=0, sta_grid=None, nsteps=3)
    o = Oracle(p)
    o.run(3)
    assert np.abs(o.wavefield()).max() == 0.0


def test_gaussian_source_weights_sum_to_one():
    import ctypes as C
    from oracle.oracle import lib as olib
    p = small_problem("iso", nsteps=5)
    o = Oracle(p)
    n, mx = C.c_int(), C.c_int()
    ext_num = np.zeros(4, np.int32)
    coef = np.zeros(4 * 343, np.float32)
    olib().orc_src_info(o.h, C.addressof(n), C.addressof(mx), None, ext_num.ctypes.data, None,
                        coef.ctypes.data, None)
    assert n.value == 1
    assert ext_num[0] == 343  # source well inside: all 7^3 points kept
    assert abs(float(coef[:343].sum()) - 1.0) < 1e-5


def test_pml_coefficients_kat():
    """Inner edge: D = 0, B = 1, A = alpha_max * (0) ... outer edge: A = D + 0, B = 1/beta_max."""
    p = small_problem("iso", nsteps=2, npml=6)
    o = Oracle(p)
    from oracle.oracle import lib as olib
    A, B, D = (np.zeros(7, np.float32) for _ in range(3))
    n = olib().orc_pml_coefs(o.h, 0, 0, A.ctypes.data, B.ctypes.data, D.ctypes.data)
    assert n == 7
    # side 0: index N (= 6) is the inner edge
    assert D[6] == 0.0 and B[6] == 1.0 and abs(A[6] - 3.0) < 1e-6
    assert abs(B[0] - 1 / 2.5) < 1e-6 and abs(A[0] - D[0]) < 1e-3 * D[0]
    assert np.all(np.diff(D[::-1]) >= 0)


def test_flat_free_surface_matrix_kat():
    """Flat free surface: dzVz = -lam/(lam+2mu) (dxVx + dyVy), dzVx = -dxVz, dzVy = -dyVz."""
    ni, nj, nk = 12, 12, 12
    c = _cart_coord(ni, nj, nk, 100.0, 100.0, 100.0)
    m = metric_fp32(c)
    lam, mu = 2.0e10, 1.3e10
    med = np.zeros((3,) + c.shape[1:], np.float32)
    med[0], med[1], med[2] = 2500.0, lam, mu
    p = Problem(ni=ni, nj=nj, nk=nk, medium_type=CGFD_MEDIUM_ELASTIC_ISO, coord=c, metric=m, medium=med,
                dt=0.005, nt_total=2, free_top=1)
    o = Oracle(p)
    from oracle.oracle import lib as olib
    nx, ny = ni + 6, nj + 6
    mx = np.zeros(nx * ny * 9, np.float32)
    my = np.zeros(nx * ny * 9, np.float32)
    assert olib().orc_free_mats(o.h, mx.ctypes.data, my.ctypes.data) == 0
    A = mx.reshape(ny, nx, 3, 3)[6, 6]
    Bm = my.reshape(ny, nx, 3, 3)[6, 6]
    r = lam / (lam + 2 * mu)
    # rows: dzVx, dzVy, dzVz; columns: dxVx, dxVy, dxVz (metric ratios are 1 on a cube grid)
    assert np.allclose(A, [[0, 0, -1], [0, 0, 0], [-r, 0, 0]], atol=1e-6)
    assert np.allclose(Bm, [[0, 0, 0], [0, 0, -1], [0, -r, 0]], atol=1e-6)


def test_coordinate_location_recovers_cell_positions():
    """The oracle's restatement of the reference's location (nearest point, containing cell,
    101^3 sampling) returns the index + shift of points built by trilinear interpolation,
    to the sampling step 0.01; a depth of 0 lands on the free surface."""
    from oracle.oracle import locate_points
    p = small_problem("iso", nsteps=4)
    c = p.coord

    def tri(i0, j0, k0, f):
        out = np.zeros(3)
        for kk in (0, 1):
            for jj in (0, 1):
                for ii in (0, 1):
                    w = (f[0] if ii else 1 - f[0]) * (f[1] if jj else 1 - f[1]) * (f[2] if kk else 1 - f[2])
                    out += w * c[:, k0 + 3 + kk, j0 + 3 + jj, i0 + 3 + ii]
        return out
    cases = [((10, 12, 8), (0.37, 0.61, 0.25)), ((20, 5, 15), (0.9, 0.1, 0.5)), ((3, 30, 2), (0.5, 0.5, 0.5))]
    pts = np.array([tri(*a, f) for a, f in cases], np.float32)
    idx, inc = locate_points(c, pts)
    for (a, f), ix, fr in zip(cases, idx, inc):
        assert np.allclose(ix + fr, np.array(a) + np.array(f), atol=0.0101)
    top = c[:, p.nk + 2, 9 + 3, 7 + 3]
    idx, inc = locate_points(c, np.array([[top[0], top[1], 0.0]], np.float32), [1])
    assert tuple(idx[0]) == (7, 9, p.nk - 1) and np.allclose(inc[0], 0.0, atol=0.0101)
    out, _ = locate_points(c, np.array([[1e9, 0.0, 0.0]], np.float32))
    assert (out == -1000).all()
