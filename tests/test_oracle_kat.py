"""The oracle's compositing arithmetic against the reference's own testRender()
(SparseVolumeRadianceField/VolumeFieldRender.cu:111-183), printed to 6 decimals."""
import json

import numpy as np

from conftest import GOLDEN


def test_composite_kat_matches_reference_printout():
    import orc

    kat = json.loads((GOLDEN / "kat_test_render.json").read_text())
    rr, w, og, cg = orc.composite_kat(kat["opacity"], kat["colour"], kat["gt"])
    tol = kat["print_resolution"] + 1e-12
    np.testing.assert_allclose(rr, kat["render_res"], atol=tol, rtol=0)
    np.testing.assert_allclose(w, kat["weights"], atol=tol, rtol=0)
    np.testing.assert_allclose(og, kat["opacity_grad"], atol=tol, rtol=0)
    np.testing.assert_allclose(cg, np.array(kat["colour_grad"]), atol=tol, rtol=0)


def test_kat_weights_sum_to_one_minus_transmittance():
    import orc

    kat = json.loads((GOLDEN / "kat_test_render.json").read_text())
    _, w, _, _ = orc.composite_kat(kat["opacity"], kat["colour"], kat["gt"])
    assert abs(w.sum() - (1 - np.exp(-np.sum(kat["opacity"])))) < 1e-12
