"""Grid sets (bt_batch): G grids with their own cameras and spins built
together must give, grid by grid, exactly what a lone build of the same
camera and spin gives -- the set only shares launches and the ray queue --
in eager mode, replayed from a CUDA graph, after the autotuner, and in the
mixed form.  One member is also checked against the oracle."""
import math

import numpy as np
import pytest

from test_grid_gpu import compare

pytestmark = pytest.mark.gpu

POSES = [  # (theta, phi, r, motion, a)
    (math.pi / 2, 0.0, 5.0, (0.0, 0.0, 1.0), 0.999),   # circular orbit
    (1.2, 0.0, 8.0, (0.0,), 0.99),                     # static
    (math.pi / 2, 0.0, 30.0, (0.0,), 0.6),             # static, far
    (0.5, 0.0, 12.0, (0.0,), 0.3),                     # static, high latitude
]
ML, SL = 8, 5


def cameras(bt, poses):
    return [bt.Camera(t, p, r, *mv, a=a) for t, p, r, mv, a in poses], [p[4] for p in poses]


def dense(g):
    return {k: v.cpu().numpy() for k, v in g.dense().items()}


def alone(bt, cam, a, prec="plain"):
    g = bt.Grid(ML, SL, True, cam, opts=prec)
    return dense(g), g.traced


def assert_same(a, b, label):
    for k in ("exists", "blevel", "steps", "status"):
        assert np.array_equal(a[k], b[k]), f"{label}: {k} differs"
    e = a["exists"] == 1
    for k in ("theta", "phi"):
        assert np.array_equal(a[k][e], b[k][e]), f"{label}: {k} differs"


@pytest.mark.parametrize("prec", ["plain", "mixed"])
def test_set_members_equal_lone_builds(bt, cuda, prec):
    cams, spins = cameras(bt, POSES)
    S = bt.GridSet(ML, SL, True, len(cams), opts=prec)
    S.build(cams, spins)
    total = 0
    for k, (c, a) in enumerate(zip(cams, spins)):
        ref, traced = alone(bt, c, a, prec)
        assert_same(dense(S.grids[k]), ref, f"{prec} member {k}")
        assert S.grids[k].traced == traced
        total += traced
    assert S.traced == total
    assert S.info().flags == 0


def test_set_member_vs_oracle(bt, cuda, oracle_mod):
    cams, spins = cameras(bt, POSES)
    S = bt.GridSet(ML, SL, True, len(cams))
    S.build(cams, spins)
    for k in (0, 3):
        cam12 = cams[k].as_array()
        ref = oracle_mod.grid_build(ML, SL, True, cam12, spins[k], tfix=1)
        compare(dense(S.grids[k]), ref, f"member {k}")


def test_set_graph_replay_equals_eager(bt, cuda):
    cams, spins = cameras(bt, POSES)
    eager = bt.GridSet(ML, SL, True, len(cams))
    eager.build(cams, spins)
    ref = [dense(g) for g in eager.grids]
    S = bt.GridSet(ML, SL, True, len(cams))
    S.set_graph(True)
    order = [2, 0, 3, 1]
    S.build([cams[k] for k in order], [spins[k] for k in order])  # captures
    S.build(cams, spins)                                          # replays
    assert S.info().graph == 1
    for k in range(len(cams)):
        assert_same(dense(S.grids[k]), ref[k], f"graph member {k}")
    S.build([cams[k] for k in order], [spins[k] for k in order])
    for slot, k in enumerate(order):
        assert_same(dense(S.grids[slot]), ref[k], f"graph permuted {slot}")


def test_autotune_keeps_results(bt, cuda):
    cams, spins = cameras(bt, POSES)
    S = bt.GridSet(ML, SL, True, len(cams))
    S.build(cams, spins)
    ref = [dense(g) for g in S.grids]
    (threads, per_sm), ms = S.autotune(cams, spins, repeats=1)
    assert threads in (64, 128, 256) and 0 <= per_sm <= 32 and ms > 0
    assert (S.info().shape.threads, S.info().shape.blocks_per_sm) == (threads, per_sm)
    S.build(cams, spins)
    for k in range(len(cams)):
        assert_same(dense(S.grids[k]), ref[k], f"tuned member {k}")


def test_full_tuner(bt, cuda):
    """bt_batch_tune: the configuration it keeps (level shape with refill size,
    or one launch) builds the same grids; for the mixed form the FP64 band is
    picked by its error against the plain form: the narrowest band meets a
    loose target, none meets an impossible one (the smallest-error band is
    reported), and the error reported is the one of the band chosen."""
    cams, spins = cameras(bt, POSES)
    S = bt.GridSet(ML, SL, True, len(cams), opts="fast")
    S.build(cams, spins)
    ref = [dense(g) for g in S.grids]
    r = S.tune(cams, spins, repeats=1)
    assert r["candidates"] == 23 and r["best_ms"] > 0 and r["level_ms"] > 0
    assert r["flow_ms"] > 0 and r["best_ms"] == min(r["level_ms"], r["flow_ms"])
    assert r["band_p99_rad"] == -1.0
    sh = S.info().shape
    if r["flow"] == 0:
        assert (sh.threads, sh.blocks_per_sm, sh.refill) == r["shape"]
        assert r["shape"][2] in (4, 8, 16)
    S.build(cams, spins)
    assert S.info().flags == 0
    for k in range(len(cams)):
        assert_same(dense(S.grids[k]), ref[k], f"tuned member {k}")
    M = bt.GridSet(ML, SL, True, len(cams), opts="mixed")
    loose = M.tune(cams, spins, p99_target=1.0, repeats=1)
    assert loose["band_met"] and loose["fp64_band"] == 0.05
    assert 0 <= loose["band_p99_rad"] <= 1.0
    tight = M.tune(cams, spins, p99_target=1e-15, repeats=1)
    assert not tight["band_met"] and tight["fp64_band"] in (0.05, 0.1, 0.2, 0.5, 1.0, 2.0, 5.0)
    assert tight["band_p99_rad"] <= loose["band_p99_rad"]
    assert M.opts._o.fp64_band == tight["fp64_band"]
    print(f"tuned: fast {r}; mixed band {tight['fp64_band']} p99 {tight['band_p99_rad']:.2e}")


def test_lone_grid_tuner(bt, cuda):
    """bt_grid_tune on a lone grid keeps a configuration that builds the same
    grid; tuning a member of a set is refused."""
    cams, spins = cameras(bt, POSES)
    g = bt.Grid(ML, SL, True, cams[0], opts="fast")
    ref = dense(g)
    r = g.tune(repeats=1)
    assert r["candidates"] == 23 and r["best_ms"] > 0
    g.build()
    assert g.info().flags == 0
    assert_same(dense(g), ref, "tuned lone grid")
    S = bt.GridSet(ML, SL, True, 2, opts="fast")
    S.build(cams[:2], spins[:2])
    with pytest.raises(bt.BtError):
        S.grids[0].tune(repeats=1)


def test_lone_grid_graph_replay(bt, cuda):
    cams, spins = cameras(bt, POSES)
    ref, _ = alone(bt, cams[1], spins[1])
    g = bt.Grid(ML, SL, True, cams[0], opts="plain")
    g.set_graph(True)
    g.build(cams[1], spins[1])
    g.build(cams[1], spins[1])
    assert_same(dense(g), ref, "lone graph")


def test_member_misuse(bt, cuda):
    cams, spins = cameras(bt, POSES[:2])
    S = bt.GridSet(ML, SL, True, 2)
    with pytest.raises(ValueError):
        S.build(cams[:1], spins[:1])
    S.build(cams, spins)
    with pytest.raises(bt.BtError):
        S.grids[0].build(cams[0], spins[0])
    bt.lib().bt_grid_destroy(S.grids[1]._h)  # ignored for members
    assert S.grids[1].traced > 0


@pytest.mark.parametrize("prec", ["plain", "fast", "mixed"])
def test_flow_builds_equal_level_builds(bt, cuda, prec):
    """The refinement levels run as one persistent launch (bt_batch_set_flow:
    a block is checked as soon as its corners are traced, or refined as soon
    as one traced diagonal decides it) give the grids of the level-by-level
    build, bit for bit: a set of poses (and one member replayed from a CUDA
    graph), the C2 grid L6 -> L10 alone, and L4 -> L12, whose eight levels are
    more than early refinement's waiter bits hold (blocks then wait for all
    four corners)."""
    cams, spins = cameras(bt, POSES)
    lvl = bt.GridSet(ML, SL, True, len(cams), opts=prec)
    lvl.build(cams, spins)
    flo = bt.GridSet(ML, SL, True, len(cams), opts=prec)
    flo.set_flow(True)
    for graph in (False, True):
        flo.set_graph(graph)
        flo.build(cams, spins)
        assert flo.info().flags == 0
        for k in range(len(cams)):
            assert_same(dense(flo.grids[k]), dense(lvl.grids[k]), f"{prec} flow member {k}")
            assert flo.grids[k].traced == lvl.grids[k].traced
    cam = bt.Camera(math.pi / 2, 0.0, 5.0, 0.0, 0.0, 1.0, a=0.999)
    a = bt.Grid(10, 6, True, cam, opts=prec)
    b = bt.Grid(10, 6, True, cam, opts=prec)
    for bps in (1, 2):  # launch shapes: blocks of 256 threads per SM
        b.set_flow(True, blocks_per_sm=bps)
        b.build()
        assert b.info().flags == 0 and b.traced == a.traced
        assert_same(dense(b), dense(a), f"{prec} flow C2 L10, {bps} blocks per SM")
    a = bt.Grid(12, 4, True, cam, opts=prec)
    b = bt.Grid(12, 4, True, cam, opts=prec)
    b.set_flow(True)
    b.build()
    assert b.info().flags == 0 and b.traced == a.traced
    assert_same(dense(b), dense(a), f"{prec} flow C2 L4 -> L12")


def test_flow_gives_up_when_a_ray_is_lost(bt, cuda):
    """The one-launch build's waits are bounded: with one ray lost on purpose
    (counted as in flight, never traced; bt_grid_set_flow_drop) nothing can
    end the flow, its warps give up after about two seconds without
    progress, and the build reports flag 8 (BT_ERR_NUMERIC, "the flow gave up
    waiting").  The context stays usable: the next build, with nothing lost,
    gives the level build's grid."""
    import time

    from blacktracer_b200 import _lib as L
    cam = bt.Camera(math.pi / 2, 0.0, 5.0, 0.0, 0.0, 1.0, a=0.999)
    ref = bt.Grid(9, 6, True, cam, opts="fast")
    g = bt.Grid(9, 6, True, cam, opts="fast")
    g.set_flow(True)
    L.check(L.lib().bt_grid_set_flow_drop(g._h))
    import ctypes as C
    t0 = time.time()
    g.build()
    inf = L.bt_grid_info()
    rc = L.lib().bt_grid_query(g._h, C.byref(inf), None)
    waited = time.time() - t0
    assert rc == L.BT_ERR_NUMERIC and inf.flags & 8, (rc, inf.flags)
    assert b"flow gave up" in L.lib().bt_last_error()
    assert 1.5 < waited < 60, waited
    g.build()
    assert g.info().flags == 0
    assert_same(dense(g), dense(ref), "flow after a lost ray")
    g.set_graph(True)
    with pytest.raises(L.BtError):
        L.check(L.lib().bt_grid_set_flow_drop(g._h))
