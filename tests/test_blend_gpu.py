"""Blending between two grids (the reference's Gr > 1 movement path) against
the reference's own kernels compiled for the host: the black hole's box and
smoothed border (findBhCenter, findBhBorders, smoothBorder x 4) and the
blended corner interpolation (pixInterpolation with Gr = 2).

Tolerances: border 1e-5 rad, corners 1e-4 rad at p99.9 with the same
capture classification for >= 99.9% (the border walk steps by sinf/cosf,
which differ by an ulp between the device and the host libm).

The reference's border walk has no bound, so the host run only happens
when the device reports that every walk ended inside the lattice.  Where the
reference reads lattice rows past the first grid it reads the second grid's
rows (they are stored one after the other); this build reads absent
vertices there, as it does for single grids -- those corners (the last rows
of the view, at theta ~ pi) are left out of the comparison."""
import math

import numpy as np
import pytest

from parity import synthetic_stars, value_noise_bgr

pytestmark = pytest.mark.gpu

ML, SL = 8, 5


@pytest.fixture(scope="module")
def two_grids(bt, cuda):
    ca = bt.Camera(math.pi / 2, 0.0, 5.0, 0.0, 0.0, 1.0, a=0.999)
    cb = bt.Camera(math.pi / 2, 0.0, 6.0, 0.0, 0.0, 1.0, a=0.999)
    ga = bt.Grid(ML, SL, True, ca, opts="fast")
    gb = bt.Grid(ML, SL, True, cb, opts="fast")
    return ca, cb, ga, gb


def map_grid_host(g):
    p, rows, cols, _ = g.map_grid()
    import torch
    from blacktracer_b200.render import _device_view
    return _device_view(p, (rows * cols, 2), torch.float32).cpu().numpy(), rows, cols


@pytest.mark.parametrize("alpha", [0.0, 0.3, 0.75])
def test_blend_vs_reference(bt, cuda, oracle_mod, two_grids, alpha):
    ca, cb, ga, gb = two_grids
    B = bt.Blend()
    B.prepare(ga, gb)
    border, nang, at_edge = B.info()
    assert nang == 1000
    if at_edge:
        pytest.skip(f"{at_edge} border walks reached the lattice edge (unbounded in the reference)")
    W, H = 256, 128
    view = bt.Viewer(math.pi / 2, 0, 0, W, H, True)
    R = bt.Renderer(W, H)
    R.render(ga, view, ca, grid2=gb, cam2=cb, alpha=alpha, blend=B)
    sc = R.scratch()
    A, rows, cols = map_grid_host(ga)
    Bg, _, _ = map_grid_host(gb)
    thphi, gap, ref_border = oracle_mod.ref_map_blend(A, Bg, rows, cols, ML,
                                                      view.viewMatrix.cpu().numpy(), W, H, alpha)
    got_border = border.cpu().numpy()
    # the walk steps by sinf/cosf of the direction, a few hundred times: the
    # device's and the host's sinf/cosf differ by an ulp
    assert np.abs(got_border - ref_border).max() < 1e-5
    keep = np.arange((H + 1) * (W + 1)) < (H - 1) * (W + 1)  # all but the last two rows
    got = sc["thphi"].cpu().numpy()[keep]
    ref = thphi[keep]
    cap_g, cap_r = got[:, 0] == -1, ref[:, 0] == -1
    both = ~cap_g & ~cap_r
    dth = np.abs(got[both, 0] - ref[both, 0])
    dph = np.abs((got[both, 1] - ref[both, 1] + np.pi) % (2 * np.pi) - np.pi)
    err = np.maximum(dth, dph)
    gaps = (sc["gap"].cpu().numpy()[keep] == gap[keep]).mean()
    print(f"alpha {alpha}: classification equal {(cap_g == cap_r).mean():.5f}, "
          f"exact {(err == 0).mean():.5f}, p99.9 {np.percentile(err, 99.9):.2e}, gaps {gaps:.5f}")
    assert (cap_g == cap_r).mean() >= 0.999
    assert np.percentile(err, 99.9) <= 1e-4 and gaps >= 0.999


def test_blend_frame(bt, cuda, two_grids):
    ca, cb, ga, gb = two_grids
    B = bt.Blend()
    B.prepare(ga, gb)
    W, H = 256, 128
    view = bt.Viewer(math.pi / 2, 0, 0, W, H, True)
    env = bt.Environment(value_noise_bgr(128, 256, seed=2))
    sp = bt.StarProcessor(*synthetic_stars(4000, seed=1, tmax=15000.0), treeLevel=7)
    R = bt.Renderer(W, H)
    kw = dict(env=env, stars=sp, grid2=gb, cam2=cb, blend=B)
    a = R.render(ga, view, ca, alpha=0.5, **kw).cpu().numpy()
    b = R.render(ga, view, ca, alpha=0.5, **kw).cpu().numpy()
    assert np.array_equal(a, b)
    c = R.render(ga, view, ca, alpha=0.0, **kw).cpu().numpy()
    assert not np.array_equal(a, c)
    with pytest.raises(bt.BtError):
        R.render(ga, view, ca, grid2=gb, cam2=cb, alpha=0.5, blend=bt.Blend())  # unprepared
