"""Media discretisation on the GPU (cgfd_media_layer_el_iso_gpu) against the reference's own
host code (media_layer2model_el_iso from the reference's src/media, oracle/_ref/libref_media.so)
on the same curvilinear grid and layered model with undulating interfaces and depth gradients,
for the three methods (loc, har, ari). Bar: every value equal to the reference's within 1e-6
relative (both evaluate the same float / double expressions in the same order; the one
library difference is the double pow of the gradient term), and at least 99.9% bitwise equal."""
import numpy as np
import pytest

from cgfd_b200 import synth, media_layer_gpu, CgfdError
import media_ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not media_ref.available(), reason="libref_media.so not built")]


@pytest.mark.parametrize("method", [0, 1, 2])
def test_gpu_media_matches_reference(method):
    coord = synth.curvilinear_grid(48, 44, 40, 100.0, seed=7)
    model = synth.layer_model(coord, seed=9)
    ref = media_ref.layer2model_el_iso(coord, model, method)
    got = media_layer_gpu(coord, model, method)
    assert np.isfinite(ref).all() and (ref[0] > 0).all()
    rel = np.abs(got.astype(np.float64) - ref) / np.abs(ref).astype(np.float64)
    assert rel.max() <= 1e-6, rel.max()
    assert (got == ref).mean() >= 0.999
    if method:
        loc = media_ref.layer2model_el_iso(coord, model, 0)
        assert (ref != loc).any()  # the averaging changed the points at the interfaces


def test_gpu_media_rejects_points_outside_the_mesh():
    coord = synth.curvilinear_grid(24, 24, 20, 100.0, seed=7)
    model = synth.layer_model(coord, seed=9)
    model.x0 += 500.0  # the mesh no longer covers the grid's first columns
    with pytest.raises(CgfdError) as e:
        media_layer_gpu(coord, model, 0)
    assert e.value.code == -1
