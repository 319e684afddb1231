"""The GMB fit of visco-elastic media (cgfd_visco_gmb, FP64) against the CPU restatement of the
reference's float algorithm (oracle/visco_gmb.py, md_vis_GMB_cal_Y), on the Q values and moduli of
the visco-elastic test medium and of a spread of Q."""
import numpy as np

import cgfd_b200
from oracle.visco_gmb import gmb_fit
from helpers import small_problem

VIS = {"nmaxwell": 3, "fr": 2.0, "fmin": 0.2, "fmax": 20.0}


def _compare(v, lam, mu, qp, qs):
    a = cgfd_b200.visco_gmb(v, lam, mu, qp, qs)
    b = gmb_fit(v, lam, mu, qp, qs)
    assert np.allclose(a[4], b[4], rtol=1e-6)  # relaxation frequencies
    for x, y in zip(a[:2], b[:2]):  # unrelaxed moduli
        assert np.abs(x - y).max() <= 1e-5 * np.abs(y).max()
    for x, y in zip(a[2:4], b[2:4]):  # weights
        assert np.abs(x - y).max() <= 3e-5 * np.abs(y).max()


def test_gmb_fit_matches_restatement_on_test_medium():
    p = small_problem("vis", nsteps=2)
    m = p.medium[:, 3:-3, 3:-3, 3:-3].reshape(5, -1)
    pick = np.unique(m[3:].T, axis=0, return_index=True)[1]  # one point per distinct (Qp, Qs)
    _compare(p.visco, m[1, pick], m[2, pick], m[3, pick], m[4, pick])


def test_gmb_fit_matches_restatement_over_q():
    qs = np.array([5, 10, 20, 40, 80, 150, 300, 1000], np.float32)
    lam = np.full(qs.size, 9.0e9, np.float32)
    mu = np.full(qs.size, 6.5e9, np.float32)
    for nm in (1, 2, 3, 5):
        _compare(dict(VIS, nmaxwell=nm), lam, mu, 2 * qs, qs)


def test_problem_bytes_counts_memory_variables():
    """cgfd_problem_bytes of a visco-elastic problem adds at least the 4 levels of 6 nmax memory
    variables and the anelastic weights to the elastic problem's bytes."""
    pi = small_problem("iso", nsteps=2)
    pv = small_problem("vis", nsteps=2)
    ri, _ = cgfd_b200.problem_bytes(pi)
    rv, _ = cgfd_b200.problem_bytes(pv)
    cells = (pv.ni + 6) * (pv.nj + 6) * (pv.nk + 6)
    assert rv - ri >= (4 * 6 + 2) * 3 * cells * 4
