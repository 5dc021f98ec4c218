"""The oracle against the reference's own kernels (fixtures from tests/golden/make_ref_golden.py,
generated by running SparseVolumeRadianceField built for sm_100a on a B200).

Bit-exact: ray origins/directions/near/far and ground-truth bytes, occupancy bytes,
in-cage flags, index offsets.  Float results through exp/log/pow (host libm vs CUDA)
within the stated tolerances."""
import numpy as np
import pytest

from conftest import GOLDEN

import make_ref_golden as G  # noqa: E402  (tests/golden is on sys.path via this file's conftest)
import orc
from tolerances import GRAD_REL, RGB_ABS, assert_grads_close, normwise  # noqa: F401


def oracle_rays(case, bbox):
    nr = sum(len(p) for p in case["pix"])
    rays = orc.RaySet(nr, True)
    off = 0
    for cam, img, pix in zip(case["cams"], case["images"], case["pix"]):
        orc.rays_from_camera(cam, bbox, case["img"], *img, True, pix, rays, off)
        off += len(pix)
    return rays


@pytest.fixture(scope="module")
def dense():
    ref = np.load(GOLDEN / "ref_dense.npz")
    case = G.dense_case()
    n = case["n"]
    rays = oracle_rays(case, (0, n - 1, 0, n - 1, 0, n - 1))
    return ref, case, rays


def test_rays_bit_exact(dense):
    ref, case, rays = dense
    for k, ok in (("ox", "ox"), ("oy", "oy"), ("oz", "oz"), ("dx", "dx"), ("dy", "dy"), ("dz", "dz"),
                  ("near", "near_t"), ("far", "far_t"), ("mask", "mask"), ("r", "r"), ("g", "g"), ("b", "b")):
        assert np.array_equal(ref[f"ray_{k}"].view(np.uint8), rays[ok].view(np.uint8)), k


def test_forward_matches_reference(dense):
    ref, case, rays = dense
    n = case["n"]
    sc = orc.Scene(n, n, n, 9, case["params"], step=0.5)
    orc.render_forward(sc, rays)
    assert np.abs(rays["acc_den"] - ref["fwd_acc_density"]).max() <= 1e-5 * max(1.0, np.abs(ref["fwd_acc_density"]).max())
    assert np.abs(rays["acc_w"] - ref["fwd_acc_weights"]).max() <= 1e-5
    for c in "rgb":
        assert np.abs(rays[f"acc_{c}"] - ref[f"fwd_acc_{c}"]).max() <= RGB_ABS


def test_backward_matches_reference(dense):
    ref, case, rays = dense
    n = case["n"]
    sc = orc.Scene(n, n, n, 9, case["params"], step=0.5)
    for k in ("acc_density", "acc_weights", "acc_r", "acc_g", "acc_b"):  # the reference's forward outputs
        rays.a[{"acc_density": "acc_den", "acc_weights": "acc_w"}.get(k, k)][:] = ref[f"fwd_{k}"]
    losses, grad, _ = orc.render_backward(sc, rays, G.MASK_COEF, G.HUBER)
    assert np.abs(losses - ref["losses"]).max() <= 255 * RGB_ABS
    assert_grads_close(grad, ref["grad_bwd"])


def test_tv_and_adam_match_reference(dense):
    ref, case, _ = dense
    n = case["n"]
    sc = orc.Scene(n, n, n, 9, case["params"], step=0.5, adaptive_lr=case["adaptive"])
    g = ref["grad_bwd"].copy()
    orc.tv_grad(sc, g, 1e-3, 1e-3, 0, 6)
    assert normwise(g - ref["grad_bwd"], ref["grad_tv"] - ref["grad_bwd"]) <= 1e-5
    g = ref["grad_tv"].copy()
    m = np.zeros_like(g)
    v = np.zeros_like(g)
    orc.adam(sc, g, m, v, 0.1, 0.01, 1)
    assert np.abs(sc.params - ref["params_adam"]).max() <= 4 * np.spacing(np.abs(ref["params_adam"]).max())
    assert normwise(m, ref["m_adam"]) <= 1e-6 and normwise(v, ref["v_adam"]) <= 1e-6
    assert not g.any() and not ref["grad_after_adam"].any()


@pytest.mark.parametrize("key,nb", [("t0n3", 3), ("t0n6", 6), ("t0n26", 26)])
def test_tv_type0_variants_match_reference(key, nb):
    ref = np.load(GOLDEN / "ref_tv.npz")
    case = G.tv_case()
    n = case["n"]
    sc = orc.Scene(n, n, n, 9, case["params"], step=0.5)
    g = case["grad"].copy()
    orc.tv_grad(sc, g, 2e-3, 1e-3, 0, nb)
    assert normwise(g - case["grad"], ref[key] - case["grad"]) <= 1e-5


def type1_cell_terms(params, n, lam_d, lam_sh, with_sh):
    """Per-vertex contributions of each of its (up to 8) cells to the type-1 term
    (RenderUtils.cu:2469-2547): terms[a, v, k] from the cell whose corner k is v."""
    p = params.reshape(params.shape[0], n, n, n).astype(np.float32)
    m = n - 1
    terms = np.zeros((params.shape[0], n, n, n, 8), np.float64)
    corners = [(dz, dy, dx) for dz in (0, 1) for dy in (0, 1) for dx in (0, 1)]
    vals = [p[:, dz:dz + m, dy:dy + m, dx:dx + m] for dz, dy, dx in corners]
    mean_d = sum(v[0] for v in vals) / np.float32(8)                          # density: sum, then /8
    mean_s = sum(v[1:] / np.float32(8) for v in vals)                         # SH: sum of a/8
    for k, (dz, dy, dx) in enumerate(corners):
        t = np.zeros((params.shape[0], m, m, m), np.float64)
        t[0] = lam_d * (vals[k][0] - mean_d)
        if with_sh:
            t[1:] = lam_sh * (vals[k][1:] - mean_s)
        terms[:, dz:dz + m, dy:dy + m, dx:dx + m, k] = t
    return terms.reshape(params.shape[0], -1, 8)


@pytest.mark.parametrize("key,ostep", [("t1s0", 0), ("t1s2", 2)])
def test_tv_type1_matches_reference_up_to_its_race(key, ostep):
    """The reference applies the type-1 term with an unsynchronised += from neighbouring
    threads, so some updates are lost.  The oracle applies every update once; each
    reference element must equal the oracle's value minus a subset of that vertex's
    per-cell contributions."""
    ref = np.load(GOLDEN / "ref_tv.npz")
    case = G.tv_case()
    n = case["n"]
    sc = orc.Scene(n, n, n, 9, case["params"], step=0.5, optimize_step=ostep)
    g = case["grad"].copy()
    orc.tv_grad(sc, g, 2e-3, 1e-3, 1, 6)
    diff = (ref[key].astype(np.float64) - g).reshape(g.shape[0], -1)
    terms = type1_cell_terms(case["params"], n, 2e-3, 1e-3, ostep <= 1)
    tol = 1e-9 + 1e-6 * np.abs(terms).max()
    bad = np.abs(diff) > tol
    assert bad.mean() < 0.25  # most updates land
    subsets = np.array([[(s >> k) & 1 for k in range(8)] for s in range(256)], np.float64)
    t = terms[bad]                                       # [n_bad, 8]
    sums = t @ subsets.T                                 # [n_bad, 256]
    best = np.abs(sums + diff[bad][:, None]).min(1)
    assert np.all(best <= tol), best.max()


def test_sparse_tables_and_march_match_reference():
    ref = np.load(GOLDEN / "ref_sparse.npz")
    case = G.sparse_case()
    n = case["n"]
    occ, cage, idx, cnt, _ = orc.occupancy(case["params"][0], n, n, n, case["threshold"])
    assert np.array_equal(occ, ref["occupancy"])
    assert np.array_equal(cage, ref["in_cage"])
    assert np.array_equal(idx, ref["index_offsets"])
    assert cnt == int(ref["in_cage_count"][0])
    comp = orc.compact(case["params"], cage, cnt)
    rays = oracle_rays(case, (0, n - 1, 0, n - 1, 0, n - 1))
    sc = orc.Scene(n, n, n, 9, comp, step=0.5, sparse=True, occ=occ, index_offsets=idx, in_cage=cage)
    orc.render_forward(sc, rays)
    for c in "rgb":
        assert np.abs(rays[f"acc_{c}"] - ref[f"fwd_acc_{c}"]).max() <= RGB_ABS
    assert np.abs(rays["acc_w"] - ref["fwd_acc_weights"]).max() <= 1e-5
    for k in ("acc_density", "acc_weights", "acc_r", "acc_g", "acc_b"):
        rays.a[{"acc_density": "acc_den", "acc_weights": "acc_w"}.get(k, k)][:] = ref[f"fwd_{k}"]
    losses, grad, _ = orc.render_backward(sc, rays, G.MASK_COEF, G.HUBER)
    assert np.abs(losses - ref["losses"]).max() <= 255 * RGB_ABS
    assert_grads_close(grad, ref["grad_bwd"])
    g = ref["grad_bwd"].copy()
    orc.tv_grad(sc, g, 1e-3, 1e-3, 0, 6)
    assert normwise(g - ref["grad_bwd"], ref["grad_tv"] - ref["grad_bwd"]) <= 1e-5
