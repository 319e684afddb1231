"""Long-run storage-precision bars against committed FP64 oracle seismograms
(tests/golden/fp64_long_{vti,aniso}.npz, made by `python tests/precision_study.py oracle
--cache tests/golden`): 128x128x64, 50 m, CFS-PML 10, free surface, one double-couple source,
16 surface stations, 2000 steps.

Bars (gather rel L2 / worst per-station rel L2 / peak amplitude error):
  FP32                 <= 1e-5 each    (measured ~2e-6: FP32 rounding only)
  U16_COEF             <= 1e-4 each    (measured <= 5e-5)
  FP16_WAVE (mixed)    <= 1e-3 each    (the seismogram bar of the mixed mode)
"""
import os

import numpy as np
import pytest

from cgfd_b200 import Simulation, CGFD_PREC_FP32, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE
from helpers import rel_l2, per_station_rel_l2
import precision_study

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BARS = {CGFD_PREC_FP32: 1e-5, CGFD_PREC_U16_COEF: 1e-4, CGFD_PREC_FP16_WAVE: 1e-3}


@pytest.mark.parametrize("medium", precision_study.MEDIA)
@pytest.mark.parametrize("precision", list(BARS))
def test_long_run_precision(medium, precision):
    z = np.load(os.path.join(GOLDEN, f"fp64_long_{medium}.npz"))
    steps, (ni, nj, nk) = int(z["steps"]), [int(v) for v in z["shape"]]
    ref = z["seis"]
    p = precision_study.problem(medium, ni, nj, nk, steps)
    assert abs(p.dt - float(z["dt"])) < 1e-9
    p.precision = precision
    sim = Simulation(p)
    sim.run()
    s = sim.seismograms()
    sim.close()
    peak = float(np.abs(ref).max())
    errs = (rel_l2(s, ref), per_station_rel_l2(s, ref), abs(float(np.abs(s).max()) - peak) / peak)
    print(f"\n{medium} precision {precision}: gather {errs[0]:.2e} station {errs[1]:.2e} peak {errs[2]:.2e}")
    assert all(e <= BARS[precision] for e in errs), errs
