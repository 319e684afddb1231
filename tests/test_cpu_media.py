"""The reference's own media discretisation (oracle/_ref/libref_media.so) on CPU: the layered
model written by formats.write_layer_file and read back by the reference gives, away from the
interfaces, each layer's rho, lambda = rho vp^2 - 2 mu, mu = rho vs^2 within 5e-6 relative (the
reference's float bilinear interpolation of a constant layer rounds by an ulp or two, which the
difference in lambda amplifies about threefold). This
pins the file writer and the checker the GPU media test compares against."""
import numpy as np
import pytest

from cgfd_b200 import synth
import media_ref

pytestmark = pytest.mark.skipif(not media_ref.available(), reason="oracle/_ref/libref_media.so not built")


def test_reference_media_reads_our_layer_file():
    coord = synth.curvilinear_grid(30, 28, 46, 100.0, seed=3)  # 4.5 km deep: all three layers
    m = synth.layer_model(coord, relief=0.0, grad=False)
    med = media_ref.layer2model_el_iso(coord, m, 0)
    z = coord[2]
    for n, (vp, vs, rho) in enumerate(synth.LAYERS_3):
        top = 1e30 if n == 0 else -1500.0 if n == 1 else -3500.0
        bot = -1500.0 if n == 0 else -3500.0 if n == 1 else -1e30
        sel = (z < top - 2.0) & (z > bot + 2.0)
        assert sel.sum() > 100
        mu = np.float32(np.float32(vs) * np.float32(vs) * np.float32(rho))
        lam = np.float32(float(np.float32(np.float32(vp) * np.float32(vp) * np.float32(rho))) - 2.0 * float(mu))
        for got, want in ((med[0][sel], np.float32(rho)), (med[2][sel], mu), (med[1][sel], lam)):
            assert np.abs(got.astype(np.float64) / float(want) - 1.0).max() <= 5e-6
