"""The jitter generator (SolidStrategy 0) against the reference's own: objectScene::
setSelfSampleOffset (SceneUtils.cu:792-798) -> randGPU (Utils.cu:1002-1044), cuRAND's
scrambled Sobol64 with the reference's quirks.  Offsets bit-exact with the reference's
kernels for the same host rand() seeds, within 1e-12 of the oracle's restatement, and a
jittered march bit-exact with the reference's march on its own offsets."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref_available():
    import refharness

    return refharness.available()


@pytest.mark.parametrize("n", [64, 256])
def test_offsets_bit_exact_against_reference(cuda, n):
    import cpx
    import orc
    import refharness as R

    params = np.zeros((28, n ** 3), np.float32)
    if not _ref_available():
        pytest.skip("reference build missing")
    ref = R.RefScene(n, n, n, 9, 2, 0.5, params)
    scene = cpx.ObjectScene(n, n, n, 9)
    try:
        for seed in (0, 7):
            want = ref.sample_offsets(seed)
            seeds = R.rand_values(seed, 3)
            scene.fill_sample_offsets(0.25, seeds)
            got = scene.sample_offsets(len(want[0]))
            for a in range(3):
                assert np.array_equal(got[a].view(np.uint64), want[a].view(np.uint64)), a
                o = orc.sobol_offsets(len(want[a]), int(seeds[a]), 0.25)
                assert np.abs(o - got[a]).max() <= 1e-12 * 0.25
    finally:
        ref.close()
        scene.close()


@pytest.mark.skipif("not _ref_available()")
def test_jittered_march_bit_exact_against_reference(cuda):
    import cpx
    import cpx_scenes as S
    import refharness as R

    cfg = S.small_config(seed=13, n=64, n_cams=6, img=96, n_rays=1024)
    n = cfg["W"]
    ref = R.RefScene(n, n, n, 9, 2, 0.5, cfg["params"])
    ref.rays_init(cfg["cams"], 96, 96, cfg["images"], cfg["pix"], True)
    scene = cpx.ObjectScene(n, n, n, 9)
    scene.upload_params(cfg["params"])
    rays = cpx.Rays(ref.n_rays)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"], 96, 96)
    try:
        ref.sample_offsets(11)
        ref.render_forward(0, ref.n_rays)
        want = ref.rays_download()
        scene.fill_sample_offsets(0.25, R.rand_values(11, 3))
        cpx.RenderUtils.renderRays(rays, scene)
        scene.check()
        got = rays.download(fields=cpx.RAY_OUTPUTS)
        assert np.array_equal(got["acc_density"].view(np.uint32), want["acc_density"].view(np.uint32))
        assert np.array_equal(got["acc_weights"].view(np.uint32), want["acc_weights"].view(np.uint32))
        for c in "rgb":
            assert np.abs(got[f"acc_{c}"] - want[f"acc_{c}"]).max() <= 1e-5
        # the offsets moved the samples: the unjittered march differs
        scene.set_sample_offsets(None, None, None)
        cpx.RenderUtils.renderRays(rays, scene)
        plain = rays.download(fields=("acc_density",))
        assert not np.array_equal(plain["acc_density"], got["acc_density"])
    finally:
        ref.close()
        scene.close()
        rays.close()
