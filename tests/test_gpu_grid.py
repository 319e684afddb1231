"""FP64 grid metrics on the GPU (cgfd_metric_calc_gpu) against the host FP64 calculation
(cgfd_metric_calc): bitwise equal, ghosts included (both round products and sums of the
7-point operator in the same order without fused multiply-add, and extrapolate the ghosts
axis by axis). The host version is itself checked against the reference's FP32 metric
(tests/test_cpu_golden.py), so the GPU version carries that pin."""
import numpy as np
import pytest

from cgfd_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(40, 36, 30), (97, 64, 51)])
def test_gpu_metric_equals_host_fp64(shape):
    ni, nj, nk = shape
    coord = synth.curvilinear_grid(ni, nj, nk, 100.0, seed=5)
    host = synth.metrics(coord)
    dev = synth.metrics_gpu(coord)
    assert np.abs(host[0]).min() > 0
    assert np.array_equal(dev, host)


def test_gpu_metric_rejects_bad_sizes():
    from cgfd_b200 import lib
    out = np.zeros(10, np.float32)
    assert lib().cgfd_metric_calc_gpu(0, 2, 2, 2, out.ctypes.data, out.ctypes.data) == -1


@pytest.mark.parametrize("medium,precision", [("iso", 0), ("vti", 3), ("aniso", 5)])
def test_problem_without_metric_equals_host_metric(medium, precision):
    """A description without a metric (desc.metric NULL): the problem computes it on the device
    from the coordinates. Its run equals the run given the host FP64 metric (cgfd_metric_calc)
    bitwise, seismograms and final wavefield: the metric itself is bitwise equal, and so are the
    host-side setups that read it (source weights from the Jacobian, free-surface matrices from
    the top plane). FP32, 16-bit fixed-point coefficients and the FP64 build."""
    import dataclasses
    from cgfd_b200 import Simulation
    p = synth.make_problem(52, 44, 36, 100.0, 40, dt=None, medium=medium, npml=6, nsrc=1, sta_grid=(3, 3),
                           seed=5, src_depth=(800.0, 800.0), center_src=True)
    p.precision = precision
    q = dataclasses.replace(p, metric=None)
    a = Simulation(p)
    a.run()
    b = Simulation(q)
    b.run()
    assert np.abs(a.seismograms()).max() > 0
    assert np.array_equal(a.seismograms(), b.seismograms())
    assert np.array_equal(a.wavefield(), b.wavefield())
    assert a.device_bytes() == b.device_bytes()
    a.close()
    b.close()
