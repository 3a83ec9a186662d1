"""The work census of a frame (bt_map_census) that the map roofline and the
star-candidate report use: environment columns per pixel against a numpy
restatement of distortEnvironmentMap's span (BT/MakeImageKernel.cu:645-657,
retrievePixelCorners and piCheck), and the reference's star candidates
(starsToCheck, :265-275) against the reference's own searchTree run per
pixel on the host.  Both exact."""
import math
import os

import numpy as np
import pytest

from parity import synthetic_stars, value_noise_bgr

pytestmark = pytest.mark.gpu

F = np.float32
PI, PI2 = F(np.pi), F(2 * np.pi)


def corners(thphi, M, N):
    """(t, p, ok, picheck) of every pixel, as pixel_corners / retrievePixelCorners."""
    M1 = M + 1
    tp = thphi.reshape(N + 1, M1, 2)
    t = np.stack([tp[1:, :-1, 0], tp[:-1, :-1, 0], tp[:-1, 1:, 0], tp[1:, 1:, 0]], -1)
    p = np.stack([tp[1:, :-1, 1], tp[:-1, :-1, 1], tp[:-1, 1:, 1], tp[1:, 1:, 1]], -1)
    ok = (p >= 0).all(-1) & (t >= 0).all(-1)
    p = np.fmod(p + F(0), PI2).astype(F)
    hi = (p > PI2 * (F(1) - F(.2))).any(-1)
    lo = p < PI2 * F(.2)
    add = hi[..., None] & lo
    p = np.where(add, p + PI2, p).astype(F)
    return t.reshape(-1, 4), p.reshape(-1, 4), ok.reshape(-1), add.any(-1).reshape(-1)


def env_columns(thphi, bh, M, N, rows):
    t, p, ok, _ = corners(thphi, M, N)
    ind = (np.arange(N)[:, None] * (M + 1) + np.arange(M)[None, :]).reshape(-1)
    use = ok & (ind > 0) & (bh == 0)
    pix = F(PI / F(rows))
    phmax, phmin = p.max(1), p.min(1)
    pmax = (phmax / pix).astype(np.int64)
    pmin = (phmin / pix).astype(np.int64)
    num = pmax - pmin + 1
    num = np.where((num > 1) & ((pmax * pix).astype(F) > phmax), num - 1, num)
    return int((num[use] + 1).sum()), int(use.sum())


def test_census_vs_restatement_and_reference_search(bt, cuda, oracle_mod):
    if not oracle_mod.have_ref_map():
        pytest.skip("reference map harness not built")
    cam = bt.Camera(1.2, 0.0, 8.0, 0.0, a=0.99)
    grid = bt.Grid(8, 5, True, cam, opts="fast")
    W, H, TL = 128, 64, 9
    view = bt.Viewer(math.pi / 2, 0, 0, W, H, True)
    env = bt.Environment(value_noise_bgr(256, 512, seed=3))
    stars = synthetic_stars(60000, seed=4)
    sp = bt.StarProcessor(*stars, treeLevel=TL)
    R = bt.Renderer(W, H)
    R.render(grid, view, cam, env=env, stars=sp)
    c = R.census()
    sc = R.scratch()
    thphi = sc["thphi"].cpu().numpy()
    bh = sc["bh"].cpu().numpy()
    cols, px = env_columns(thphi, bh, W, H, 256)
    assert (c["env_columns"], c["env_pixels"]) == (cols, px)
    # starsToCheck per pixel: the reference's searchTree on each pixel's box
    t, p, ok, _ = corners(thphi, W, H)
    lib = oracle_mod._refmaplib()
    import ctypes as C
    lib.btref_search_tree.argtypes = [oracle_mod._i32, oracle_mod._f32p, oracle_mod._f32p,
                                      C.c_int, oracle_mod._i32, C.c_int]
    tree = sp.binaryStarTree
    nodes = np.empty(1 << 16, np.int32)
    ref, npx = 0, 0
    for k in np.nonzero(bh == 0)[0]:  # distortStarMap does not check the corners
        mn = np.array([t[k].min(), p[k].min()], F)
        mx = np.array([t[k].max(), p[k].max()], F)
        n = lib.btref_search_tree(tree, mn, mx, TL, nodes, len(nodes))
        npx += 1
        for node in nodes[:n]:
            start = tree[node - 1] if node != 0 and ((node + 1) & node) != 0 else 0
            ref += int(tree[node] - start)
    assert c["star_pixels"] == npx
    assert c["star_candidates_ref"] == ref
    assert 0 < c["star_candidates"] <= ref
    print(f"candidates per pixel: reference {ref / npx:.1f}, pruned {c['star_candidates'] / npx:.1f}")
