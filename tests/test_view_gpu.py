"""The perspective camera view (Viewer::makeCameraView, BT/Viewer.h:109-133)
and the look-around offsets of pixInterpolation (BT/MakeImageKernel.cu
:464-465, driven by the arrow keys at :1081-1102; here frame parameters).

The view is exact against the reference's own Viewer (golden fixture from
tests/golden/make_golden.py): its angles are evaluated with the reference's
expressions on the host.  Frames through a perspective view are compared
with the reference's map kernels with the tolerances of test_map_gpu.py."""
import math
import os

import numpy as np
import pytest

from parity import map_grid_from_dense, synthetic_stars, value_noise_bgr

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_camera_view_matches_reference_viewer(bt, cuda):
    f = np.load(os.path.join(GOLD, "ref_views.npz"))
    k = 0
    while f"view{k}" in f:
        ang, up, right, W, H = f[f"args{k}"]
        v = bt.Viewer(ang, up, right, int(W), int(H), False)
        got = v.viewMatrix.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), f[f"view{k}"].view(np.uint32)), k
        k += 1
    assert k == 3


def test_camera_view_offset_bound(bt, cuda):
    W, H, ang = 64, 32, math.pi / 2
    up_max = (math.pi - H * ang / W) / 2
    bt.Viewer(ang, up_max * 0.999, 0, W, H, False)
    with pytest.raises(bt.BtError):
        bt.Viewer(ang, up_max * 1.001, 0, W, H, False)


def compare_img(a, b, label, exact_frac=0.95, close_frac=0.999):
    d = np.abs(a.astype(np.int32) - b.astype(np.int32)).max(-1)
    ex, cl = float((d == 0).mean()), float((d <= 1).mean())
    print(f"{label}: exact {ex:.4f} within1 {cl:.5f} max {d.max()}")
    assert ex >= exact_frac and cl >= close_frac, (label, ex, cl, int(d.max()))


@pytest.mark.parametrize("view_args,hor,ver", [
    ((math.pi / 2, 0.0, 0.0), 0.0, 0.0),
    ((1.2, 0.2, 0.5), 0.0, 0.0),
    ((math.pi / 2, 0.0, 0.0), 0.35, -0.12),  # look-around offsets
])
def test_perspective_frame_vs_reference(bt, cuda, oracle_mod, view_args, hor, ver):
    if not oracle_mod.have_ref_map():
        pytest.skip("reference map harness not built")
    g = np.load(os.path.join(GOLD, "g_c2_l7s4.npz"))
    cam = bt.Camera.from_array(g["cam"], float(g["a"]))
    grid = bt.Grid(int(g["maxlevel"]), int(g["startlevel"]), bool(g["angle"]), cam)
    ref_grid, rows, GM = map_grid_from_dense(g["theta"], g["phi"], g["exists"], True)
    W, H = 160, 96
    viewer = bt.Viewer(view_args[0], view_args[1], view_args[2], W, H, False)
    view = viewer.viewMatrix.cpu().numpy()
    bgr = value_noise_bgr(256, 512, seed=11)
    stars = synthetic_stars(4000, seed=12, tmax=15000.0)
    tl = 7
    sp = bt.StarProcessor(*stars, treeLevel=tl)
    pos, mg, tree = oracle_mod.ref_star_tree(*stars, tl)
    cam7 = cam.getParamArray()
    ref = oracle_mod.ref_map_frame(ref_grid, rows, GM, grid.MAXLEVEL, view, W, H, cam7,
                                   bgr=bgr, stars=(pos, mg, tree, tl), lr=True, hor=hor,
                                   ver=ver)
    R = bt.Renderer(W, H)
    out = R.render(grid, viewer, cam, env=bt.Environment(bgr), stars=sp, lr=True, hor=hor,
                   ver=ver)
    sc = {k: v.cpu().numpy() for k, v in R.scratch().items()}
    assert np.array_equal(sc["thphi"], ref["thphi"]), "corner interpolation differs"
    assert np.array_equal(sc["gap"], ref["gap"])
    assert np.array_equal(sc["bh"], ref["bh"])
    compare_img(out.cpu().numpy(), ref["image"].reshape(H, W, 4), f"perspective {view_args}")
