"""C ABI checks that need no GPU: the library loads, exports every function declared in
include/cgfd_b200.h, host-side helpers work and invalid descriptions are rejected."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cgfd_b200
from cgfd_b200 import synth, formats, Problem, CGFD_MEDIUM_ELASTIC_ISO
from cgfd_b200.abi import ProblemDesc
from oracle.oracle import metric_fp32
from helpers import small_problem, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(cgfd_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = cgfd_b200.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.cgfd_version() >= 100


def test_metric_calc_fp64_matches_fp32_restatement():
    c = synth.curvilinear_grid(24, 22, 18, 100.0, seed=7)
    a = synth.metrics(c)
    b = metric_fp32(c)
    assert rel_l2(a[:, 3:-3, 3:-3, 3:-3], b[:, 3:-3, 3:-3, 3:-3]) < 1e-5


def test_dt_estimate_and_three_digits():
    p = small_problem("iso", nsteps=2)
    dtmax = synth.dt_estimate(p)
    assert 0.005 < dtmax < 0.05
    # blk_keep_three_digi zeroes characters 3..8 of "%9.7e": two significant digits survive
    assert synth.keep_three_digits(0.0123456) == pytest.approx(0.012, rel=1e-6)
    assert synth.keep_three_digits(4.56789e-3) == pytest.approx(4.5e-3, rel=1e-6)


def test_src_and_station_roundtrip(tmp_path):
    p = small_problem("iso", nsteps=3, nsrc=3)
    formats.write_src(str(tmp_path / "a.src"), p.src)
    s = formats.read_src(str(tmp_path / "a.src"))
    assert np.allclose(s.loc, p.src.loc) and np.allclose(s.cmp[:, 3:], p.src.cmp[:, 3:])
    assert s.mechanism_type == 1 and s.cmp_type == 2 and s.loc_3dim == 1
    formats.write_station_list(str(tmp_path / "st.list"), p.sta)
    t = formats.read_station_list(str(tmp_path / "st.list"))
    assert np.allclose(t.loc, p.sta.loc) and list(t.flag_depth) == list(p.sta.flag_depth)


def test_reference_example_files_parse():
    """The reference's own example inputs (test_source.src, station.list) in its grammar."""
    src_text = "event_3force_ricker\n1\n0 6\n2 0\n0 0 \n150.0 100.0 100.0\n" \
               "0.0 ricker_deriv 2 1.0 0 0 0 0 0 0 0 0\n1.0e16 1.0e16 1.0e16\n"
    import tempfile
    with tempfile.NamedTemporaryFile("w", suffix=".src", delete=False) as f:
        f.write(src_text)
    s = formats.read_src(f.name)
    os.unlink(f.name)
    assert s.num == 1 and s.stf_length == 6.0 and s.cmp_type == 2
    assert np.allclose(s.cmp[0, 3:6], 1e16) and np.allclose(s.cmp[0, 6:], 0)
    assert s.wavelet_coefs[0, 0] == 2 and s.wavelet_coefs[0, 1] == 1.0


def _create(desc):
    h = C.c_void_p()
    rc = cgfd_b200.lib().cgfd_problem_create(C.byref(desc), C.byref(h))
    if rc == 0:
        cgfd_b200.lib().cgfd_problem_destroy(h)
    return rc, cgfd_b200.lib().cgfd_last_error().decode()


def test_invalid_descriptions_are_rejected():
    p = small_problem("iso", nsteps=2)
    d = p.desc()
    d.ni = 3
    rc, msg = _create(d)
    assert rc == -1 and "at least 8" in msg
    d = p.desc()
    d.medium_type = 6  # no such medium
    rc, msg = _create(d)
    assert rc == -5
    d = p.desc()
    d.medium_type = 5  # visco-elastic iso without its GMB parameters
    rc, msg = _create(d)
    assert rc == -1 and "visco" in msg
    pv = small_problem("vis", nsteps=2)
    pv.precision = cgfd_b200.CGFD_PREC_FP64  # visco-elastic: FP32 only
    rc, msg = _create(pv.desc())
    assert rc == -5 and "visco" in msg
    d = p.desc()
    d.medium_type = 1  # acoustic: FP32 and FP64 only
    d.precision = cgfd_b200.CGFD_PREC_U16_COEF
    rc, msg = _create(d)
    assert rc == -5 and "acoustic" in msg
    d = p.desc()
    d.dt = 0.0
    rc, msg = _create(d)
    assert rc == -1
    d = p.desc()
    d.src.loc_coord_type = 2
    rc, msg = _create(d)
    assert rc == -1 and "loc_coord_type" in msg
    d = p.desc()
    d.pml[2][1].enable = 1
    d.pml[2][1].num_layers = 3
    rc, msg = _create(d)
    assert rc == -1 and "free and PML" in msg


def test_null_arguments():
    L = cgfd_b200.lib()
    assert L.cgfd_problem_create(None, None) == -1
    assert L.cgfd_run(None, 1) == -1
    assert L.cgfd_problem_destroy(None) == 0


def test_problem_bytes_on_host():
    """cgfd_problem_bytes needs no device: it grows with the batch and shrinks with 16-bit
    storage."""
    import dataclasses
    from cgfd_b200 import problem_bytes, synth, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE
    p = small_problem("iso", nsrc=0)
    rng = np.random.default_rng(0)
    shots = [synth.dc_sources(p.coord, p.ni, p.nj, 1, rng, depth_range=(600.0, 1200.0), stf_length=p.nt_total * p.dt)
             for _ in range(3)]
    one, _ = problem_bytes(dataclasses.replace(p, src=shots[0]))
    three, _ = problem_bytes(p, shots)
    assert three > one
    u16, _ = problem_bytes(dataclasses.replace(p, src=shots[0], precision=CGFD_PREC_U16_COEF))
    w16, _ = problem_bytes(dataclasses.replace(p, src=shots[0], precision=CGFD_PREC_FP16_WAVE))
    assert w16 < u16 < one


def test_server_without_gpu_fails_cleanly():
    from conftest import gpu_available
    from cgfd_b200 import Server, CgfdError
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(CgfdError) as e:
        Server()
    assert e.value.code == -2


def test_visco_gmb_fit_properties():
    """cgfd_visco_gmb (md_vis_GMB_cal_Y): log-uniform relaxation frequencies, weights of order 1/Q,
    moduli unchanged at Q -> infinity, rejection of Q < 1."""
    v = {"nmaxwell": 3, "fr": 2.0, "fmin": 0.2, "fmax": 20.0}
    lam = np.full(4, 8e9, np.float32)
    mu = np.full(4, 6e9, np.float32)
    qs = np.array([20, 50, 100, 1e7], np.float32)
    lu, mu_u, yl, ym, wl = cgfd_b200.visco_gmb(v, lam, mu, 2 * qs, qs)
    assert np.allclose(wl, 2 * np.pi * np.array([0.2, 2.0, 20.0]), rtol=1e-6)
    assert np.all(mu_u[:3] > mu[:3]) and abs(mu_u[3] / mu[3] - 1) < 1e-5
    assert np.all(np.abs(ym[:, :3] * qs[:3]) < 3.0) and np.all(np.abs(ym[:, 3]) < 1e-5)
    # the fitted Q^-1(w) = sum Y_n (wl_n w + wl_n^2 Q^-1) / (wl_n^2 + w^2) matches 1/Qs inside the band
    w = 2 * np.pi * np.geomspace(0.3, 15.0, 9)
    for t in range(3):
        fit = sum(ym[n, t] * (wl[n] * w + wl[n] ** 2 / qs[t]) / (wl[n] ** 2 + w ** 2) for n in range(3))
        assert np.all(np.abs(fit * qs[t] - 1.0) < 0.1), t
    with pytest.raises(cgfd_b200.CgfdError):
        cgfd_b200.visco_gmb(v, lam, mu, 2 * qs, np.zeros(4, np.float32))
