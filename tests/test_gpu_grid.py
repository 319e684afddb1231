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
