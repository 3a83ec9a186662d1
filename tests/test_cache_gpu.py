"""Cache files on the device: a .grid file expanded into the map grid
(makeGrid from the perfect hash, BT/MakeImageKernel.cu:369-384), a built
grid saved for the reference, and star files, all against the reference's
own bytes and lookups (golden fixtures from tests/golden/make_golden.py, and
the reference harness where it was built).  Everything here is exact: the
file path moves the same float values the map grid holds."""
import math
import os
import tempfile

import numpy as np
import pytest

from parity import synthetic_stars, value_noise_bgr

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def mirrored(dense, N, M):
    """makeGrid's layout of a dense N x M decode: with M / N > 3 the lower
    hemisphere mirrors the upper one (theta -> pi - theta)."""
    if M / N <= 3:
        return dense.reshape(N * M, 2).copy()
    rows = 2 * N - 1
    g = np.empty((rows, M, 2), np.float32)
    d = dense.reshape(N, M, 2)
    g[:N] = d
    m = d.copy()
    t = m[..., 0]
    keep = (t != -1) & (t != -2)
    t[keep] = np.float32(np.pi) - t[keep]
    for i in range(N):
        g[rows - i - 1] = m[i]
    return g.reshape(-1, 2)


def u32(a):
    return np.ascontiguousarray(a).view(np.uint32)


def test_reference_grid_file_to_map_grid(bt, cuda):
    ref = np.load(os.path.join(GOLD, "ref_c2_l6s4_decoded.npz"))
    gf = bt.GridFile(os.path.join(GOLD, "ref_c2_l6s4.grid"))
    N, M = int(ref["N"]), int(ref["M"])
    assert gf.MAXLEVEL == int(ref["maxlevel"]) and gf.cols == M
    got = gf.grid.cpu().numpy()
    assert np.array_equal(u32(got), u32(mirrored(ref["dense"], N, M)))


@pytest.mark.parametrize("angle", [True, False])
def test_saved_grid_loads_everywhere(bt, cuda, oracle_mod, angle):
    cam = bt.Camera(math.pi / 2, 0.0, 5.0, 0.0, 0.0, 1.0, a=0.999)
    g = bt.Grid(7, 4, angle, cam, opts="fast")
    ptr, rows, cols, sym = g.map_grid()
    from blacktracer_b200.render import _device_view
    mine = _device_view(ptr, (rows * cols, 2), cuda.float32).cpu().numpy()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.grid")
        g.save(p)
        gf = bt.GridFile(p)
        assert (gf.rows, gf.cols, gf.sym) == (rows, cols, sym)
        assert np.array_equal(u32(gf.grid.cpu().numpy()), u32(mine))
        t = bt.read_grid_file(p)
        assert (t["N"], t["M"], t["MAXLEVEL"]) == (g.N, g.M, 7)
        # the device expansion from tables handed over directly
        dev = {k: cuda.from_numpy(np.ascontiguousarray(t[k])).cuda()
               for k in ("hash_table", "pos_tag", "offset_table")}
        out = cuda.empty((rows * cols, 2), dtype=cuda.float32, device="cuda")
        import blacktracer_b200._lib as L
        L.check(L.lib().bt_grid_map_from_psh(dev["hash_table"].data_ptr(),
                                             dev["pos_tag"].data_ptr(),
                                             dev["offset_table"].data_ptr(), t["hash_width"],
                                             t["offset_width"], t["N"], t["M"],
                                             out.data_ptr(), rows, None))
        assert np.array_equal(u32(out.cpu().numpy()), u32(mine))
        if oracle_mod.have_ref():
            back = oracle_mod.ref_grid_file_decode(p)
            N, M = back["N"], back["M"]
            assert np.array_equal(u32(back["dense"]), u32(mine.reshape(-1, M, 2)[:N].reshape(-1, 2)))


def test_render_from_file_equals_render_from_grid(bt, cuda):
    cam = bt.Camera(1.2, 0.0, 8.0, 0.0, a=0.99)
    g = bt.Grid(7, 5, True, cam, opts="fast")
    W, H = 192, 96
    view = bt.Viewer(math.pi / 2, 0, 0, W, H, True)
    env = bt.Environment(value_noise_bgr(128, 256, seed=5))
    th, ph, mag, bv = synthetic_stars(3000, seed=6, tmax=15000.0)
    sp = bt.StarProcessor(th, ph, mag, bv, treeLevel=7)
    R = bt.Renderer(W, H)
    a = R.render(g, view, cam, env=env, stars=sp).cpu().numpy()
    with tempfile.TemporaryDirectory() as d:
        gp, spath = os.path.join(d, "g.grid"), os.path.join(d, "s.star")
        g.save(gp)
        sp.save(spath)
        b = R.render(bt.GridFile(gp), view, cam, env=env,
                     stars=bt.StarProcessor.load(spath)).cpu().numpy()
    assert np.array_equal(a, b)


def test_load_map_argument_errors(bt, cuda):
    gf = os.path.join(GOLD, "ref_c2_l6s4.grid")
    import blacktracer_b200._lib as L
    out = cuda.empty(16, dtype=cuda.float32, device="cuda")
    with pytest.raises(bt.BtError):  # wrong shape
        L.check(L.lib().bt_grid_file_load_map(gf.encode(), out.data_ptr(), 3, 4, None))
