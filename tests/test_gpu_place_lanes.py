"""Sample placement marches a few rays per 32-thread warp (CPX_PLACE_LANES sets the fewest; the
library picks as few as keep the batch in one wave).  How many rays share a warp changes only
which lanes run together, never a ray's own arithmetic: the sample counts, accumulated density
and weight, colours and per-ray losses of a forward + backward must be the same bits for every
setting, in the reference-exact FP64 placement and in the FP32 march of the mixed forms.

The setting is read once per process, so each one runs in a child process of its own."""
import json
import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = pathlib.Path(__file__).resolve().parents[1]

CHILD = r"""
import json, sys
import numpy as np
import torch
sys.path[:0] = [sys.argv[1] + "/clear-plenoxels_b200", sys.argv[1] + "/tests"]
import cpx
import cpx_scenes as S

out = {}
cfg = S.small_config(seed=23, n=40, n_cams=6, img=48, n_rays=1024)
n = cfg["W"]
for prec in ("fp32", "bf16"):
    scene = cpx.ObjectScene(n, n, n, 9, step_size=cfg["step"], precision=prec)
    scene.upload_params(cfg["params"])
    nr = sum(len(p) for p in cfg["pix"])
    rays = cpx.Rays(nr, white_bg=True)
    rays.initial_self(scene, [cpx.Camera.make(**c) for c in cfg["cams"]], cfg["images"], cfg["pix"],
                      cfg["img_w"], cfg["img_h"])
    losses = torch.zeros(nr, dtype=torch.float64, device="cuda:0")
    cpx.RenderUtils.renderRays_forwardBackward(scene, rays, losses, None, 0, nr, 1.0, 0.1)
    scene.check()
    o = rays.download(fields=cpx.RAY_OUTPUTS)
    out[prec] = {"counts": scene.last_sample_counts(nr).tolist(),
                 "losses": losses.cpu().numpy().tolist(),
                 **{k: np.asarray(v).tolist() for k, v in o.items()}}
    scene.close()
    rays.close()
print(json.dumps(out))
"""


def _run(lanes):
    env = dict(os.environ, CPX_PLACE_LANES=str(lanes))
    r = subprocess.run([sys.executable, "-c", CHILD, str(REPO)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_placement_bits_do_not_depend_on_rays_per_warp(cuda):
    base = _run(32)
    assert sum(base["fp32"]["counts"]) > 0
    for lanes in (8, 2, 1):
        got = _run(lanes)
        for prec in ("fp32", "bf16"):
            for k, v in base[prec].items():
                assert np.array_equal(np.asarray(got[prec][k]), np.asarray(v)), (lanes, prec, k)
