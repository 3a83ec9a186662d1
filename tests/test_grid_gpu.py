"""GPU parity of the device grid builder against the reference.

Topology (which vertices exist = the reference's CamToCel keys, and the
block levels) must be bit-exact; traced values and steps follow the plain
integrator's tolerance (1e-9 rad); T-vertex-fixed values are compared with
the reference's own fixTvertices run in the same canonical order.
"""
import os

import numpy as np
import pytest

from parity import ang_err, oracle_camera

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-9
pytestmark = pytest.mark.gpu


def build(bt, cam12, a, ml, sl, ang, prec="plain"):
    cam = bt.Camera.from_array(cam12, a)
    g = bt.Grid(ml, sl, ang, cam, opts=prec)
    d = {k: v.cpu().numpy() for k, v in g.dense().items()}
    return g, d


def compare(d, ref, label):
    assert np.array_equal(d["exists"], ref["exists"]), f"{label}: vertex set differs"
    assert np.array_equal(d["blevel"], ref["blevel"]), f"{label}: block levels differ"
    e = ref["exists"] == 1
    err = ang_err(d["theta"][e], d["phi"][e], ref["theta"][e], ref["phi"][e])
    same_steps = float((d["steps"] == ref["steps"]).mean())
    print(f"{label}: {e.sum()} vertices, within {TOL}: {(err <= TOL).mean():.4f}, "
          f"p99 {np.percentile(err, 99):.2e} max {err.max():.2e}, same steps {same_steps:.4f}")
    assert (err <= TOL).mean() >= 0.99
    return err


@pytest.mark.parametrize("name", ["g_c1_l6u", "g_c2_l7s4", "g_c2_l7s4h", "g_c5_l7s5"])
def test_grid_vs_reference_golden(bt, cuda, name):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    grid, d = build(bt, g["cam"], float(g["a"]), int(g["maxlevel"]), int(g["startlevel"]),
                    bool(g["angle"]))
    ref = {k: g[k] for k in ("theta", "phi", "exists", "steps", "blevel")}
    compare(d, ref, name)
    assert grid.info().flags == 0


@pytest.mark.parametrize("ml,sl,ang,camname", [(9, 5, True, "c2"), (9, 6, True, "c5"),
                                               (8, 4, False, "c2"), (8, 8, True, "c1")])
def test_grid_vs_oracle(bt, cuda, oracle_mod, ml, sl, ang, camname):
    cam, a = oracle_camera(oracle_mod, camname)
    ref = oracle_mod.grid_build(ml, sl, ang, cam, a, tfix=1)
    grid, d = build(bt, cam, a, ml, sl, ang)
    compare(d, ref, f"L{ml}s{sl}{camname}")
    assert grid.traced == ref["count"]


def test_grid_rebuild_in_place(bt, cuda, oracle_mod):
    cam, a = oracle_camera(oracle_mod, "c1")
    cam2, a2 = oracle_camera(oracle_mod, "c2")
    grid, _ = build(bt, cam, a, 7, 4, True)
    grid.build(bt.Camera.from_array(cam2, a2), a2)
    d = {k: v.cpu().numpy() for k, v in grid.dense().items()}
    ref = oracle_mod.grid_build(7, 4, True, cam2, a2, tfix=1)
    compare(d, ref, "rebuild")


def test_grid_mixed_topology(bt, cuda, oracle_mod):
    cam, a = oracle_camera(oracle_mod, "c2")
    ref = oracle_mod.grid_build(9, 5, True, cam, a, tfix=1)
    grid, d = build(bt, cam, a, 9, 5, True, prec="mixed")
    e = ref["exists"] == 1
    topo = np.array_equal(d["exists"], ref["exists"]) and np.array_equal(d["blevel"], ref["blevel"])
    if topo:
        err = ang_err(d["theta"][e], d["phi"][e], ref["theta"][e], ref["phi"][e])
        print(f"mixed grid: p99 {np.percentile(err, 99):.2e} max {err.max():.2e}")
    assert topo, "mixed-precision grid topology must match the FP64 reference"


def test_compact_export_matches_dense(bt, cuda, oracle_mod):
    cam, a = oracle_camera(oracle_mod, "c2")
    grid, d = build(bt, cam, a, 8, 5, True)
    ex = grid.export()
    ii, jj = np.nonzero(d["exists"])  # row-major = key order
    assert np.array_equal(ex["vi"].numpy(), ii) and np.array_equal(ex["vj"].numpy(), jj)
    assert np.array_equal(ex["theta"].numpy(), d["theta"][ii, jj])
    assert np.array_equal(ex["phi"].numpy(), d["phi"][ii, jj])
    assert np.array_equal(ex["steps"].numpy(), d["steps"][ii, jj])
    bi, bj = np.nonzero(d["blevel"] >= 0)
    assert np.array_equal(ex["bi"].numpy(), bi) and np.array_equal(ex["bj"].numpy(), bj)
    assert np.array_equal(ex["level"].numpy(), d["blevel"][bi, bj])
    # the reference's CamToCel holds exactly these keys
    ref = oracle_mod.grid_build(8, 5, True, cam, a, tfix=1)
    assert len(ii) == int(ref["exists"].sum())


@pytest.mark.parametrize("ml,sl,camname", [(9, 6, "c2"), (9, 6, "c5")])
def test_fast_grid_topology_matches_plain(bt, cuda, oracle_mod, ml, sl, camname):
    """The fast FP64 form builds the same grid (vertex set, block levels) as
    the plain form, with values within the 1e-6 rad target."""
    cam, a = oracle_camera(oracle_mod, camname)
    _, dp = build(bt, cam, a, ml, sl, True, "plain")
    _, df = build(bt, cam, a, ml, sl, True, "fast")
    assert np.array_equal(dp["exists"], df["exists"]), "vertex set differs"
    assert np.array_equal(dp["blevel"], df["blevel"]), "block levels differ"
    e = (dp["exists"] == 1) & (dp["theta"] >= 0)
    err = ang_err(df["theta"][e], df["phi"][e], dp["theta"][e], dp["phi"][e])
    print(f"fast grid L{ml}{camname}: p99 {np.percentile(err, 99):.2e} max {err.max():.2e}")
    assert np.percentile(err, 99) <= 1e-6


@pytest.mark.parametrize("coop", [True, False])
def test_tfix_nonconvergence_is_reported(bt, cuda, oracle_mod, coop):
    """With one T-vertex pass per level the fix cannot see a pass that
    changed nothing, so the build must report it as not converged: flag 1
    in bt_grid_info.flags and BT_ERR_NUMERIC from bt_grid_query.  The
    default pass count converges on the same grid.  Both launch forms of
    the fix (one cooperative launch per level, a launch per pass)."""
    import ctypes as C

    from blacktracer_b200 import _lib as L
    cam, a = oracle_camera(oracle_mod, "c2")
    g = bt.Grid(9, 6, True, bt.Camera.from_array(cam, a), opts="plain")
    g.set_tfix_launch(coop)
    g.build()
    assert g.info().flags == 0
    g.set_tfix_passes(1)
    g.build()
    inf = L.bt_grid_info()
    rc = L.lib().bt_grid_query(g._h, C.byref(inf), None)
    assert rc == L.BT_ERR_NUMERIC
    assert inf.flags & 1
    assert b"T-vertex" in L.lib().bt_last_error()
    with pytest.raises(L.BtError):
        g.info()
    g.set_tfix_passes(8)
    g.build()
    assert g.info().flags == 0
    with pytest.raises(L.BtError):
        g.set_tfix_passes(0)


@pytest.mark.parametrize("prec", ["plain", "fast"])
def test_tfix_launch_forms_agree(bt, cuda, oracle_mod, prec):
    """The T-vertex fix as one cooperative launch per level and as a launch
    per pass give the same grid, bit for bit (C2 camera, L6 -> L10)."""
    cam, a = oracle_camera(oracle_mod, "c2")
    c = bt.Camera.from_array(cam, a)
    g1 = bt.Grid(10, 6, True, c, opts=prec)
    g2 = bt.Grid(10, 6, True, c, opts=prec)
    g2.set_tfix_launch(False)
    g2.build()
    d1 = {k: v.cpu().numpy() for k, v in g1.dense().items()}
    d2 = {k: v.cpu().numpy() for k, v in g2.dense().items()}
    for k in d1:
        np.testing.assert_array_equal(d1[k], d2[k], err_msg=k)
    assert g1.info().flags == 0 and g2.info().flags == 0
