"""The frame server (bt_server): every result is the same alone and in a mix
of requests of other resolutions, spins and poses -- bit-identical, since a
set member equals a lone grid build and the map is deterministic -- and equal
to the direct Grid + Renderer path; resident grids are reused, evicted under
a small budget, and no request is lost under backpressure."""
import math

import numpy as np
import pytest

from parity import synthetic_stars, value_noise_bgr

pytestmark = pytest.mark.gpu

ML, SL = 8, 5
POSES = [  # theta, phi, r, motion, spin
    (math.pi / 2, 0.0, 5.0, (0.0, 0.0, 1.0), 0.999),
    (math.pi / 2, 1.0, 6.0, (0.0, 0.0, 1.0), 0.7),
    (1.2, 0.0, 8.0, (0.0,), 0.99),
    (0.6, 0.3, 12.0, (0.0,), 0.3),
    (2.0, 2.0, 20.0, (0.0,), 0.5),
]
SIZES = [(128, 64), (256, 128), (192, 96)]


@pytest.fixture(scope="module")
def scene(bt, cuda):
    env = bt.Environment(value_noise_bgr(256, 512, seed=7))
    sp = bt.StarProcessor(*synthetic_stars(5000, seed=9), treeLevel=8)
    cams = [(bt.Camera(t, p, r, *mv, a=a), a) for t, p, r, mv, a in POSES]
    return env, sp, cams


def out_buf(cuda, W, H):
    return cuda.zeros((H, W, 4), dtype=cuda.uint8, pin_memory=True)


def drain(S, n, timeout_s=60.0):
    import time
    got, t0 = [], time.time()
    while len(got) < n and time.time() - t0 < timeout_s:
        got += S.poll(wait_ms=50)
    assert len(got) == n, f"{len(got)} of {n} completed"
    assert all(c["status"] == 0 for c in got), got
    return {c["id"]: c for c in got}


def serve(bt, scene, reqs, **kw):
    import torch
    env, sp, cams = scene
    S = bt.Server(env=env, stars=sp, maxlevel=ML, startlevel=SL, precision="fast", **kw)
    outs = {}
    for rid, (pose, (W, H)) in enumerate(reqs):
        outs[rid] = out_buf(torch, W, H)
        cam, a = cams[pose]
        S.submit(rid, W, H, cam, a, outs[rid])
    comp = drain(S, len(reqs))
    st = S.stats()
    S.close()
    return {k: v.numpy().copy() for k, v in outs.items()}, comp, st


def test_alone_equals_in_mix_and_direct(bt, cuda, scene):
    env, sp, cams = scene
    target = (2, SIZES[1])
    alone, _, _ = serve(bt, scene, [target])
    mix = [(0, SIZES[0]), (1, SIZES[2]), target, (3, SIZES[0]), (4, SIZES[1]),
           (0, SIZES[1]), (2, SIZES[0])]
    mixed, comp, st = serve(bt, scene, mix)
    assert np.array_equal(alone[0], mixed[2]), "result differs in the mix"
    # the direct path: a lone grid build of the same camera, then the map
    cam, a = cams[2]
    g = bt.Grid(ML, SL, True, cam, opts="fast")
    W, H = SIZES[1]
    view = bt.Viewer(math.pi / 2, 0, 0, W, H, True)
    ref = bt.Renderer(W, H).render(g, view, cam, env=env, stars=sp, lr=True).cpu().numpy()
    assert np.array_equal(alone[0], ref), "server frame differs from Grid + Renderer"
    assert st["grid_misses"] == 5 and st["grid_hits"] == 2
    assert comp[5]["grid_reused"] or comp[6]["grid_reused"]


def test_eviction_under_small_budget(bt, cuda, scene):
    import blacktracer_b200 as btm
    N, M = btm.grid_dims(ML, True)
    reqs = [(k % 5, SIZES[k % 2]) for k in range(12)]
    outs, comp, st = serve(bt, scene, reqs, grid_cache_bytes=2 * N * M * 8 + 16,
                           max_build_batch=2)
    assert st["evictions"] > 0 and st["completed"] == 12
    ref, _, _ = serve(bt, scene, reqs)
    for k in outs:
        assert np.array_equal(outs[k], ref[k]), f"request {k} differs under eviction"


def test_request_that_cannot_fit_fails(bt, cuda, scene):
    """A request whose frame needs more than the whole render budget fails
    with BT_ERR_NOMEM instead of waiting forever (it used to hold every
    request behind it, and the server's shutdown, which drains the queue);
    a request that fits is served after it."""
    import time

    import torch

    from blacktracer_b200 import _lib as L
    env, sp, cams = scene
    S = bt.Server(env=env, stars=sp, maxlevel=ML, startlevel=SL, precision="fast",
                  render_bytes=24 << 20)
    big, small = (1920, 960), SIZES[0]
    bufs = [out_buf(torch, *big), out_buf(torch, *small)]
    cam, a = cams[0]
    S.submit(0, *big, cam, a, bufs[0])
    S.submit(1, *small, cam, a, bufs[1])
    got, t0 = [], time.time()
    while len(got) < 2 and time.time() - t0 < 60.0:
        got += S.poll(wait_ms=50)
    st = {c["id"]: c["status"] for c in got}
    assert st == {0: L.BT_ERR_NOMEM, 1: L.BT_OK}, st
    S.close()  # returns: nothing is left waiting


def test_backpressure_keeps_every_request(bt, cuda, scene):
    reqs = [(k % 5, SIZES[k % 3]) for k in range(24)]
    outs, comp, st = serve(bt, scene, reqs, max_inflight=2, max_build_batch=3,
                           render_bytes=64 << 20)
    assert st["completed"] == 24 and st["failed"] == 0
    for c in comp.values():
        assert c["t_submit"] <= c["t_admit"] <= c["t_done"]
