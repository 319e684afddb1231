"""Failure detection without a GPU fault: a device-side pipeline wait that nothing completes
runs out its bound, the kernel records the timeout and returns, the host reports
CGFD_ERR_CUDA with the pipeline-timeout message, and the context and problem stay usable
(the run continues and equals an uninterrupted run bitwise)."""
import numpy as np
import pytest

from cgfd_b200 import Simulation
from helpers import small_problem

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_and_context_survives():
    p = small_problem("iso", nsteps=12)
    ref = Simulation(p)
    ref.run(10)
    a = Simulation(p)
    a.run(5)
    rc, msg = a.check_wait_bound()
    assert rc == -2 and "pipeline wait timed out" in msg
    a.run(5)  # the error word was cleared: the run goes on
    assert np.array_equal(a.seismograms(), ref.seismograms())
    assert np.array_equal(a.wavefield(), ref.wavefield())
    rc2, _ = a.check_wait_bound()  # repeatable
    assert rc2 == -2


@pytest.mark.parametrize("medium", ["iso", "aniso"])
@pytest.mark.parametrize("where", ["pml_corner", "interior", "surface_slab"])
def test_nonfinite_wavefield_sentinel(medium, where):
    """A NaN planted on the host (cgfd_set_wavefield) at a cell that no station samples within
    the step: the RK combine of the step's last stage finds it, and the host gets
    CGFD_ERR_NONFINITE with the wavefield message (no GPU fault; the station check alone would
    miss it). A clean run of the same problem reports nothing."""
    from cgfd_b200 import CgfdError
    p = small_problem(medium, nsteps=12)
    clean = Simulation(p)
    clean.run(2)
    ijk = {"pml_corner": (2, 2, 2), "interior": (20, 18, 10), "surface_slab": (1, 1, p.nk - 2)}[where]
    w = np.zeros((9, p.nk + 6, p.nj + 6, p.ni + 6), np.float32)
    w[4, ijk[2] + 3, ijk[1] + 3, ijk[0] + 3] = np.nan
    sim = Simulation(p)
    sim.set_wavefield(w)
    with pytest.raises(CgfdError) as e:
        sim.run(1)
    assert e.value.code == -4 and "wavefield" in str(e.value)
