"""Seeded problem definitions shared by the golden-fixture generator and the tests."""
from oracle.oracle import metric_fp32
from cgfd_b200 import synth

GOLDEN_CASES = {
    # name: (medium, ni, nj, nk, nsteps, npml, seed)
    "iso_small": ("iso", 28, 26, 22, 120, 5, 1),
    "vti_small": ("vti", 28, 26, 22, 120, 5, 2),
    "aniso_small": ("aniso", 28, 26, 22, 120, 5, 3),
    "ac_small": ("ac", 28, 26, 22, 120, 5, 4),
}


def golden_problem(name):
    medium, ni, nj, nk, nsteps, npml, seed = GOLDEN_CASES[name]
    p = synth.make_problem(ni, nj, nk, 100.0, nsteps, dt=0.006, medium=medium, npml=npml, nsrc=2,
                           sta_grid=(3, 3), seed=seed, metric_fn=metric_fp32, src_depth=(600.0, 900.0),
                           center_src=False, fc=(3.0, 4.0))
    return p, nsteps
