"""The CPU oracle against golden vectors produced by the reference's own solver code
(tests/golden/ref_*.npz, generated on a B200 by tests/golden/make_ref_golden.py through
oracle/_ref/ref_harness). No GPU needed: this pins the oracle to the reference.

Tolerance: per-station relative L2 <= 2e-5 (denominator floored at 1e-3 of the strongest
station), final-wavefield relative L2 <= 2e-5. Both sides are FP32; the reference runs
on the GPU with fused multiply-adds, the oracle on the CPU without.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, metric_fp32
from golden.cases import GOLDEN_CASES, golden_problem
from helpers import per_station_rel_l2, rel_l2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference_golden(name):
    path = os.path.join(HERE, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated")
    z = np.load(path)
    p, nsteps = golden_problem(name)
    assert int(z["nsteps"]) == nsteps
    # the oracle's FP32 metric restatement reproduces the reference's gd_curv_metric_cal
    m = metric_fp32(p.coord)
    assert rel_l2(m[:, 3:-3, 3:-3, 3:-3], z["metric"][:, 3:-3, 3:-3, 3:-3]) < 1e-6
    p.metric = z["metric"]
    o = Oracle(p)
    o.run(nsteps)
    ref = z["seismo"][:, :, :nsteps]
    assert ref.shape[0] == 9 and np.abs(ref).max() > 0
    assert per_station_rel_l2(o.seismograms()[:, :, :nsteps], ref) <= 2e-5
    w = o.wavefield()[:, 3:-3, 3:-3, 3:-3]
    assert rel_l2(w, z["wave"]) <= 2e-5
    # free-surface peak ground motion computed by the reference's PG_calcu_gpu
    assert "pg" in z.files, "fixture lacks the peak ground motion (regenerate with make_ref_golden.py)"
    pg = o.peak_motion()
    for q in range(15):
        assert np.abs(z["pg"][q]).max() > 0
        assert rel_l2(pg[q], z["pg"][q]) <= 2e-5, q


@pytest.mark.parametrize("medium", ["vti", "aniso"])
def test_long_run_fixture_matches_study_configuration(medium):
    """The committed FP64 seismograms belong to the study's problem (same dt, stations, steps)."""
    import precision_study
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", f"fp64_long_{medium}.npz"))
    ni, nj, nk = [int(v) for v in z["shape"]]
    p = precision_study.problem(medium, ni, nj, nk, int(z["steps"]))
    assert abs(p.dt - float(z["dt"])) < 1e-9
    assert z["seis"].shape == (p.sta.num, 9, p.nt_total)
    assert np.isfinite(z["seis"]).all() and np.abs(z["seis"]).max() > 0
