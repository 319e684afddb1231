"""Media discretisation on the GPU (cgfd_media_layer_el_iso_gpu, cgfd_media_layer_gpu,
cgfd_media_bin_el_iso_gpu, cgfd_media_grid_el_iso_gpu) against the reference's own host code
(media_layer2model_ac_iso / _el_iso / _el_vti / _el_aniso, media_bin2model_el_iso and
media_grid2model_el_iso from the reference's src/media,
oracle/_ref/libref_media.so)
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


# (layer file type, target medium type): acoustic files into acoustic media, VTI files into VTI
# media, every elastic file type into 21-Cij
CASES = [(10, 1), (22, 3), (23, 3), (24, 3), (21, 4), (23, 4), (25, 4), (26, 4), (27, 4)]


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("ftype,medium", CASES)
def test_gpu_layer_media_matches_reference(ftype, medium, method):
    """cgfd_media_layer_gpu against the reference's media_layer2model_el_vti / _el_aniso on the
    same grid and layer file: every field within 1e-6 of its largest magnitude, and at least 99%
    of the values bitwise equal, for the files without a rotation. The Bond-rotated TTI files
    take their sines and cosines from another math library (last-ulp differences): 2e-5, and
    under the harmonic average the c_ij whose values change sign from layer to layer (c14, c36,
    c45 of this model) are left out: their harmonic mean divides by sums near zero, where the
    reference's own value is arbitrary in the last digits (it reaches 100-4000 times the c_ij's
    largest layer value)."""
    from cgfd_b200 import media_layer_any_gpu
    coord = synth.curvilinear_grid(40, 36, 32, 100.0, seed=7)
    model = synth.layer_media(coord, ftype, seed=9)
    ref = media_ref.layer2model(coord, model, medium, method)
    got = media_layer_any_gpu(coord, model, medium, method)
    assert got.shape == ref.shape and np.isfinite(ref).all() and (ref[0] > 0).all()
    rotated = ftype in (25, 26)
    tol = 2e-5 if rotated else 1e-6
    loc = media_ref.layer2model(coord, model, medium, 0) if method else ref
    for f in range(ref.shape[0]):
        if rotated and method == 1 and (loc[f] > 0).any() and (loc[f] < 0).any():
            assert np.isfinite(got[f]).all()
            continue
        scale = float(np.abs(ref[f]).max())
        if scale == 0.0:
            assert not got[f].any(), f
            continue
        err = float(np.abs(got[f].astype(np.float64) - ref[f]).max())
        assert err <= tol * scale, (f, err, scale)
    if not rotated:
        assert (got == ref).mean() >= 0.99
    if method:
        assert (ref != loc).any()


def test_gpu_layer_media_rejects_wrong_file_type():
    from cgfd_b200 import media_layer_any_gpu
    coord = synth.curvilinear_grid(24, 24, 20, 100.0, seed=7)
    with pytest.raises(CgfdError) as e:
        media_layer_any_gpu(coord, synth.layer_media(coord, 25, seed=9), 3, 0)  # a TTI file into a VTI medium
    assert e.value.code == -1
    for ftype, medium in ((10, 2), (21, 1)):  # acoustic files only into acoustic media, and back
        with pytest.raises(CgfdError) as e:
            media_layer_any_gpu(coord, synth.layer_media(coord, ftype, seed=9), medium, 0)
        assert e.value.code == -1


def test_gpu_bin_media_matches_reference():
    """cgfd_media_bin_el_iso_gpu against the reference's media_bin2model_el_iso on the same grid and
    binary model (file dimensions z, x, y; z stored downwards): the same float operations in the
    same order, so at least 99.9% of the values bitwise equal and all within 1e-6 relative."""
    from cgfd_b200 import media_bin_gpu
    coord = synth.curvilinear_grid(40, 36, 32, 100.0, seed=7)
    model = synth.bin_model(coord, seed=3)
    ref = media_ref.bin2model_el_iso(coord, model)
    got = media_bin_gpu(coord, model)
    assert np.isfinite(ref).all() and (ref[0] > 0).all()
    rel = np.abs(got.astype(np.float64) - ref) / np.abs(ref).astype(np.float64)
    assert rel.max() <= 1e-6, rel.max()
    assert (got == ref).mean() >= 0.999


def test_gpu_bin_media_rejects_a_model_beside_the_grid():
    from cgfd_b200 import media_bin_gpu
    coord = synth.curvilinear_grid(24, 24, 20, 100.0, seed=7)
    model = synth.bin_model(coord, seed=3)
    model.origin[1] += 1e6  # file dimension 1 runs along x: the model lies beyond the grid
    with pytest.raises(CgfdError) as e:
        media_bin_gpu(coord, model)
    assert e.value.code == -1
    model = synth.bin_model(coord, seed=3)
    model.order = [0, 0, 1]
    with pytest.raises(CgfdError) as e:
        media_bin_gpu(coord, model)
    assert e.value.code == -1


@pytest.mark.parametrize("method", [0, 1, 2])
def test_gpu_grid_media_matches_reference(method):
    """cgfd_media_grid_el_iso_gpu against the reference's media_grid2model_el_iso on the same grid
    and grid model (3 layers of 3, 4, 3 surfaces with undulating layer tops): at least 99.9% of the
    values bitwise equal and all within 1e-6 relative, for loc, har and ari."""
    from cgfd_b200 import media_grid_gpu
    coord = synth.curvilinear_grid(40, 36, 32, 100.0, seed=7)
    model = synth.grid_media(coord, seed=3)
    ref = media_ref.grid2model_el_iso(coord, model, method)
    got = media_grid_gpu(coord, model, method)
    assert np.isfinite(ref).all() and (ref[0] > 0).all()
    rel = np.abs(got.astype(np.float64) - ref) / np.abs(ref).astype(np.float64)
    assert rel.max() <= 1e-6, rel.max()
    assert (got == ref).mean() >= 0.999
    if method:
        assert (ref != media_ref.grid2model_el_iso(coord, model, 0)).any()


def test_gpu_grid_media_rejects_a_mesh_smaller_than_the_grid():
    from cgfd_b200 import media_grid_gpu
    coord = synth.curvilinear_grid(24, 24, 20, 100.0, seed=7)
    model = synth.grid_media(coord, seed=3, margin=0.0)
    model.x0 += 500.0  # the mesh no longer covers the grid's first columns
    with pytest.raises(CgfdError) as e:
        media_grid_gpu(coord, model, 0)
    assert e.value.code == -1


# (grid file type, target medium type): VTI files into VTI media, the other types into 21-Cij
GRID_CASES = [(22, 3), (23, 3), (24, 3), (21, 4), (23, 4), (25, 4), (27, 4)]


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("ftype,medium", GRID_CASES)
def test_gpu_grid_media_any_type_matches_reference(ftype, medium, method):
    """cgfd_media_grid_gpu against the reference's media_grid2model_el_vti / _el_aniso on the same
    grid and grid file: every field within 1e-6 of its largest magnitude (the TTI file: 2e-5, its
    sines and cosines from another math library), at least 99% bitwise equal without a rotation.
    As for the layer files, under the harmonic average the c_ij of the TTI file whose values
    change sign across the grid are left out (their harmonic mean divides by sums near zero)."""
    from cgfd_b200 import media_grid_gpu
    coord = synth.curvilinear_grid(40, 36, 32, 100.0, seed=7)
    model = synth.grid_media(coord, seed=3, type=ftype)
    ref = media_ref.grid2model(coord, model, medium, method)
    got = media_grid_gpu(coord, model, method, medium_type=medium)
    assert got.shape == ref.shape and np.isfinite(ref).all() and (ref[0] > 0).all()
    tol = 2e-5 if ftype == 25 else 1e-6
    loc = media_ref.grid2model(coord, model, medium, 0) if method == 1 and ftype == 25 else None
    for f in range(ref.shape[0]):
        if loc is not None and (loc[f] > 0).any() and (loc[f] < 0).any():
            assert np.isfinite(got[f]).all()
            continue
        scale = float(np.abs(ref[f]).max())
        if scale == 0.0:
            assert not got[f].any(), f
            continue
        assert float(np.abs(got[f].astype(np.float64) - ref[f]).max()) <= tol * scale, f
    if ftype != 25:
        assert (got == ref).mean() >= 0.99
