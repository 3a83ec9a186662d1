"""Pins the CPU oracle (plain-C restatement, oracle/bt_oracle.c) to the
reference's own code: against the committed golden fixtures (made by the
reference compiled in place, tests/golden/make_golden.py) and, where the
reference harness is built, directly against it on fresh seeded inputs."""
import os

import numpy as np
import pytest

from parity import CAMERAS, ang_err, oracle_camera, seeded_rays

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", sorted(CAMERAS))
def test_camera_matches_reference(oracle_mod, name):
    if not oracle_mod.have_ref():
        pytest.skip("reference harness not built here")
    c0, _ = oracle_camera(oracle_mod, name)
    c1, _ = oracle_camera(oracle_mod, name, ref=True)
    assert np.array_equal(c0, c1)


@pytest.mark.parametrize("name", sorted(CAMERAS))
def test_rays_bit_exact_vs_golden(oracle_mod, name):
    g = np.load(os.path.join(GOLD, f"rays_{name}.npz"))
    to, po, st, status = oracle_mod.integrate_rays(g["cam"], float(g["a"]), g["theta"], g["phi"])
    assert np.array_equal(to, g["theta_out"])
    assert np.array_equal(po, g["phi_out"])
    assert np.array_equal(st, g["steps"])
    # captured rays are (-1, -1, 0) with status CAPTURED
    cap = status == 1
    assert np.all(to[cap] == -1) and np.all(st[cap] == 0)


@pytest.mark.parametrize("name", ["g_c1_l6u", "g_c2_l7s4", "g_c2_l7s4h", "g_c5_l7s5"])
def test_grid_bit_exact_vs_golden(oracle_mod, name):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    args = (int(g["maxlevel"]), int(g["startlevel"]), bool(g["angle"]), g["cam"], float(g["a"]))
    raw = oracle_mod.grid_build(*args, tfix=0)
    assert np.array_equal(raw["theta"], g["theta_raw"])
    assert np.array_equal(raw["phi"], g["phi_raw"])
    fix = oracle_mod.grid_build(*args, tfix=1)
    for k in ("theta", "phi", "exists", "steps", "blevel"):
        assert np.array_equal(fix[k], g[k]), k


def test_rays_bit_exact_vs_reference_fresh(oracle_mod):
    if not oracle_mod.have_ref():
        pytest.skip("reference harness not built here")
    th, ph = seeded_rays(4000, seed=7)
    for name in sorted(CAMERAS):
        cam, a = oracle_camera(oracle_mod, name)
        r0 = oracle_mod.integrate_rays(cam, a, th, ph)
        r1 = oracle_mod.integrate_rays(cam, a, th, ph, ref=True, nthreads=4)
        for x, y in zip(r0[:3], r1[:3]):
            assert np.array_equal(x, y)


def test_grid_native_order_difference_is_bounded(oracle_mod):
    """The reference's own T-vertex order (libstdc++ unordered_map) vs the
    canonical order: same topology and traced values; fixed T-vertices may
    differ, and the difference is recorded here (not a tolerance)."""
    if not oracle_mod.have_ref():
        pytest.skip("reference harness not built here")
    cam, a = oracle_camera(oracle_mod, "c2")
    nat = oracle_mod.grid_build(8, 5, True, cam, a, tfix=2, ref=True)
    can = oracle_mod.grid_build(8, 5, True, cam, a, tfix=1)
    assert np.array_equal(nat["exists"], can["exists"])
    assert np.array_equal(nat["blevel"], can["blevel"])
    assert np.array_equal(nat["steps"], can["steps"])
    e = nat["exists"] == 1
    d = ang_err(nat["theta"][e], nat["phi"][e], can["theta"][e], can["phi"][e])
    frac = float((d > 0).mean())
    assert frac < 0.02, frac


def test_newton_cap_reports_status(oracle_mod):
    """a = 0 makes the capture test's b0/q0 divide by zero (BT/Metric.h:133-143);
    the restatement must terminate and classify every ray."""
    cam = oracle_mod.camera_static(0.0, np.pi / 2, 0.0, 20.0, 0.0)
    th, ph = seeded_rays(200, seed=3)
    to, po, st, status = oracle_mod.integrate_rays(cam, 0.0, th, ph)
    assert set(np.unique(status)) <= {0, 1, 2, 3}


def test_ref_frame_rows_equal_whole_frame(oracle_mod):
    """The reference map kernels run on host threads with the colour passes
    restricted to listed rows (ref_map_frame_rows, used for the full-size
    frames) give the same corners, mask, areas and row colours as the
    whole-frame single-thread run."""
    if not oracle_mod.have_ref_map():
        pytest.skip("reference map harness not built here")
    from parity import map_grid_from_dense, sphere_view, synthetic_stars, value_noise_bgr
    g = np.load(os.path.join(GOLD, "g_c2_l7s4.npz"))
    grid, rows, GM = map_grid_from_dense(g["theta"], g["phi"], g["exists"], True)
    W, H, tl = 256, 128, 7
    bgr = value_noise_bgr(256, 512, seed=256)
    stars = synthetic_stars(4000, seed=4000, tmax=15000.0)
    pos, mg, tree = oracle_mod.ref_star_tree(*stars, tl)
    cam7 = np.array([0.3, 0.9, 0.1, 1.2, 0.0, 0.0, 1.0], np.float32)
    view = sphere_view(W, H)
    ml = int(g["maxlevel"])
    ref = oracle_mod.ref_map_frame(grid, rows, GM, ml, view, W, H, cam7, bgr=bgr,
                                   stars=(pos, mg, tree, tl), lr=True)
    sat = oracle_mod.ref_map_sat(bgr)
    assert np.array_equal(sat, ref["sat"])
    for sel in (np.arange(H), np.arange(3, H, 16)):
        r = oracle_mod.ref_map_frame_rows(grid, rows, GM, ml, view, W, H, cam7, sel, sat=sat,
                                          env_shape=bgr.shape[:2], stars=(pos, mg, tree, tl),
                                          lr=True, nthreads=4)
        for k in ("thphi", "gap", "bh", "area"):
            assert np.array_equal(r[k], ref[k]), k
        assert np.array_equal(r["env"], ref["env"].reshape(H, W, 4)[sel])
        assert np.array_equal(r["stars"], ref["stars"].reshape(H, W, 4)[sel])
        assert np.array_equal(r["image"], ref["image"].reshape(H, W, 4)[sel])
    # solid angles passed in are the ones the colour passes use
    r2 = oracle_mod.ref_map_frame_rows(grid, rows, GM, ml, view, W, H, cam7, sel, sat=sat,
                                       env_shape=bgr.shape[:2], stars=(pos, mg, tree, tl),
                                       lr=True, nthreads=4, area=ref["area"])
    assert np.array_equal(r2["image"], r["image"])
    r3 = oracle_mod.ref_map_frame_rows(grid, rows, GM, ml, view, W, H, cam7, sel, sat=sat,
                                       env_shape=bgr.shape[:2], lr=True, nthreads=4,
                                       area=ref["area"] * np.float32(1.5))
    assert not np.array_equal(r3["env"], r["env"])


@pytest.mark.parametrize("name", sorted(CAMERAS))
def test_early_refinement_rule_holds_on_test_grids(oracle_mod, name):
    """The one-launch build refines a block as soon as one traced diagonal's
    squared separation is above refineCheck's threshold (BT/Grid.h:410-445).
    That equals the full rule, the larger of both diagonals by std::max,
    unless the (0, 3) separation is NaN.  On the raw grids (before the
    T-vertex fix) of the test cameras no vertex is NaN, and no leaf block has
    a diagonal that would alone have refined it."""
    cam, a = oracle_camera(oracle_mod, name)
    maxlevel = 9
    r = oracle_mod.grid_build(maxlevel, 6, True, cam, a, tfix=0)
    th, ph, ex, bl = r["theta"], r["phi"], r["exists"] == 1, r["blevel"]
    assert not np.isnan(th[ex]).any() and not np.isnan(ph[ex]).any()
    M = r["M"]
    ii, jj = np.nonzero((bl >= 0) & (bl < maxlevel))
    assert ii.size > 0
    lv = bl[ii, jj].astype(np.int64)
    gap = 2 ** (maxlevel - lv)
    kk, ll = ii + gap, (jj + gap) % M
    d03 = (th[ii, jj] - th[kk, ll]) ** 2 + (ph[ii, jj] - ph[kk, ll]) ** 2
    d12 = (th[kk, jj] - th[ii, ll]) ** 2 + (ph[kk, jj] - ph[ii, ll]) ** 2
    thr = np.where(lv < 6, 1e-10, 0.015)
    assert not (d03 > thr).any() and not (d12 > thr).any()
