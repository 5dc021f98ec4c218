"""Generate tests/golden/ref_*.npz from the reference's own CUDA kernels.

Runs on a GPU box: oracle/_ref/libcpxref.so is the reference's unmodified
sources (SparseVolumeRadianceField/*.cu, built for sm_100a by oracle/Makefile)
plus the ref_harness.cu shim.  Inputs are regenerated from the seeds in
clear-plenoxels_b200/cpx_scenes.py, so the fixtures hold outputs only:

  ref_dense.npz   rays from _rays::initialSelf (all 12 input fields), renderRays
                  outputs, renderRays_withGradients_RGB losses and gradients,
                  addVarianceLoss (type 0/6) gradients, updateRGBScene params
                  and moments, on a 16^3 SH-band-2 grid.
  ref_tv.npz      addVarianceLoss for type 0 with 3/6/26 neighbours and type 1
                  (optimizeStep 0 and 2) from a seeded gradient, on a 12^3 grid.
  ref_sparse.npz  pruneSelf + getCagedNums tables and the sparse march outputs
                  and gradients on a 24^3 blob grid.

Usage:  python tests/golden/make_ref_golden.py OUT_DIR
"""
import pathlib
import sys

import numpy as np

REPO = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(REPO / "clear-plenoxels_b200"))
sys.path.insert(0, str(REPO / "oracle"))

import cpx_scenes as S  # noqa: E402
import refharness as R  # noqa: E402

MASK_COEF = 1.0
HUBER = 0.1


def dense_case(seed=1, n=16, n_cams=6, img=48, n_rays=768):
    """Blob scene small enough for a full dump of every output."""
    rng = np.random.default_rng(seed)
    centres, sigmas, peaks = S.random_blobs(rng, 4)
    dens = S.blob_density(n, n, n, centres, sigmas, peaks)
    params = S.make_params(dens, 9, rng, 0.3)
    cams = [S.look_at_camera(p, n, img, img) for p in S.fibonacci_sphere(n_cams, 4.0)]
    images = [tuple(rng.integers(0, 256, size=img * img, dtype=np.uint8) for _ in range(3)) +
              (rng.integers(0, 256, size=img * img, dtype=np.uint8),) for _ in range(n_cams)]
    pix = S.sample_pixels(rng, n_cams, img, img, n_rays)
    adaptive = (rng.random(n ** 3) > 0.2).astype(np.float32)
    return dict(n=n, params=params, cams=cams, images=images, pix=pix, img=img, adaptive=adaptive, rng=rng)


def tv_case(seed=2, n=12):
    rng = np.random.default_rng(seed)
    params = S.make_params(rng.normal(5.0, 4.0, size=n ** 3).astype(np.float32), 9, rng, 0.5)
    grad = rng.normal(0.0, 1e-3, size=params.shape).astype(np.float32)
    return dict(n=n, params=params, grad=grad)


def sparse_case(seed=3, n=24, n_cams=6, img=48, n_rays=768, threshold=8.0):
    rng = np.random.default_rng(seed)
    centres, sigmas, peaks = S.random_blobs(rng, 5, centre_range=0.8)
    dens = S.blob_density(n, n, n, centres, sigmas, peaks)
    params = S.make_params(dens, 9, rng, 0.3)
    cams = [S.look_at_camera(p, n, img, img) for p in S.fibonacci_sphere(n_cams, 4.0)]
    images = [tuple(rng.integers(0, 256, size=img * img, dtype=np.uint8) for _ in range(4))
              for _ in range(n_cams)]
    pix = S.sample_pixels(rng, n_cams, img, img, n_rays)
    return dict(n=n, params=params, cams=cams, images=images, pix=pix, img=img, threshold=threshold)


def run_dense(out_dir):
    c = dense_case()
    n = c["n"]
    sc = R.RefScene(n, n, n, 9, 2, 0.5, c["params"], adaptive_lr=c["adaptive"])
    sc.optimizer_init()
    sc.rays_init(c["cams"], c["img"], c["img"], c["images"], c["pix"], True)
    rays_in = sc.rays_download()
    nr = sc.n_rays
    sc.render_forward(0, nr)
    fwd = sc.rays_download()
    losses = sc.render_backward(0, nr, MASK_COEF, HUBER)
    g_bwd = sc.grads()
    sc.tv(1e-3, 1e-3, 0, 6)
    g_tv = sc.grads()
    sc.adam(0.1, 0.01, 1)
    p1 = sc.params()
    m1, v1 = sc.moments()
    g_after = sc.grads()
    sc.close()
    np.savez_compressed(
        out_dir / "ref_dense.npz",
        **{f"ray_{k}": rays_in[k] for k in ("ox", "oy", "oz", "dx", "dy", "dz", "near", "far", "mask", "r", "g", "b")},
        **{f"fwd_{k}": fwd[k] for k in ("acc_density", "acc_weights", "acc_r", "acc_g", "acc_b")},
        losses=losses, grad_bwd=g_bwd, grad_tv=g_tv, params_adam=p1, m_adam=m1, v_adam=v1,
        grad_after_adam=g_after,
        meta=np.array([n, nr, 9, 2], np.int64),
    )
    print("dense:", nr, "rays; max |grad|", float(np.abs(g_bwd).max()))


def run_tv(out_dir):
    c = tv_case()
    n = c["n"]
    res = {}
    for key, (typ, nb, ostep) in {
        "t0n3": (0, 3, 0), "t0n6": (0, 6, 0), "t0n26": (0, 26, 0), "t1s0": (1, 6, 0), "t1s2": (1, 6, 2),
    }.items():
        sc = R.RefScene(n, n, n, 9, 2, 0.5, c["params"])
        sc.optimizer_init()
        sc.set_grads(c["grad"])
        sc.tv(2e-3, 1e-3, typ, nb, ostep)
        res[key] = sc.grads()
        sc.close()
    np.savez_compressed(out_dir / "ref_tv.npz", **res)
    print("tv:", list(res))


def run_sparse(out_dir):
    c = sparse_case()
    n = c["n"]
    sc = R.RefScene(n, n, n, 9, 2, 0.5, c["params"], sparse_threshold=c["threshold"])
    occ, cage, idx = sc.occupancy()
    sc.optimizer_init()
    sc.rays_init(c["cams"], c["img"], c["img"], c["images"], c["pix"], True)
    nr = sc.n_rays
    sc.render_forward(0, nr)
    fwd = sc.rays_download()
    losses = sc.render_backward(0, nr, MASK_COEF, HUBER)
    g = sc.grads()
    sc.tv(1e-3, 1e-3, 0, 6)
    g_tv = sc.grads()
    sc.adam(0.1, 0.01, 1)
    p1 = sc.params()
    sc.close()
    np.savez_compressed(
        out_dir / "ref_sparse.npz", occupancy=occ, in_cage=cage, index_offsets=idx,
        in_cage_count=np.array([sc.in_cage_count], np.int64),
        **{f"fwd_{k}": fwd[k] for k in ("acc_density", "acc_weights", "acc_r", "acc_g", "acc_b")},
        losses=losses, grad_bwd=g, grad_tv=g_tv, params_adam=p1,
    )
    print("sparse:", sc.in_cage_count, "in cage;", nr, "rays")


def main():
    out_dir = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else REPO / "tests" / "golden")
    out_dir.mkdir(parents=True, exist_ok=True)
    run_dense(out_dir)
    run_tv(out_dir)
    run_sparse(out_dir)


if __name__ == "__main__":
    main()
