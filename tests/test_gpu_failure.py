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
