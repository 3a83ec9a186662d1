"""The allocation-free ray integration entry point (bt_integrate_rays_host_static).

Some callers cannot let a library allocate device memory (a real-time thread
that must not stall on cudaMalloc's implicit synchronisation, a plugin host
with a fixed device-memory budget); this entry point stages its rays in a
fixed static device array instead.  This test calls it through the C ABI and
checks it against the allocating entry point (bt_integrate_rays_host) on two
calls in a row, with the tolerance the integrator tests use (1e-9 rad; the
two run the same kernel on the same inputs, so they agree exactly).
Collected last, so a run that stops at the first failure has run the rest.
"""
import ctypes as C

import numpy as np
import pytest

from parity import ang_err, seeded_rays

pytestmark = pytest.mark.gpu
TOL = 1e-9


def run_static(bt, cam, th, ph, a, with_status=True, stream=None):
    L = bt._lib
    n = th.size
    out = (np.empty(n), np.empty(n), np.empty(n, dtype=np.int32), np.empty(n, dtype=np.uint8))
    th = np.ascontiguousarray(th)
    ph = np.ascontiguousarray(ph)
    rc = L.lib().bt_integrate_rays_host_static(
        C.byref(cam._c), a, th.ctypes.data, ph.ctypes.data, n, out[0].ctypes.data,
        out[1].ctypes.data, out[2].ctypes.data,
        out[3].ctypes.data if with_status else None, None, stream)
    L.check(rc)
    return out


def test_static_entry_point_matches_allocating_one(bt, cuda):
    cam = bt.Camera(np.pi / 2, 0.0, 5.0, 0.0, 0.0, 1.0, a=0.999)
    for seed, n in ((101, 20000), (202, 5000)):  # two calls in a row
        th, ph = seeded_rays(n, seed=seed)
        s = run_static(bt, cam, th, ph, 0.999)
        h = bt.integrate_rays_host(cam, th, ph, opts="plain")
        assert np.array_equal(s[3], h[3])
        assert np.array_equal(s[2], h[2])
        err = ang_err(s[0], s[1], h[0], h[1])
        assert err.max() <= TOL


def test_static_entry_point_full_capacity_on_a_stream(bt, cuda):
    """n equal to the capacity (the last slot of every staged array in use),
    status NULL, on a created stream; then the default stream again."""
    cap = int(bt.lib().bt_integrate_rays_host_static_capacity())
    cam = bt.Camera(np.pi / 2, 0.0, 30.0, 0.0, a=0.6)
    th, ph = seeded_rays(cap, seed=303)
    s = cuda.cuda.Stream()
    got = run_static(bt, cam, th, ph, 0.6, with_status=False, stream=s.cuda_stream)
    h = bt.integrate_rays_host(cam, th, ph, opts="plain")
    assert np.array_equal(got[2], h[2])
    assert ang_err(got[0], got[1], h[0], h[1]).max() <= TOL
    th2, ph2 = seeded_rays(1000, seed=304)
    got2 = run_static(bt, cam, th2, ph2, 0.6)
    h2 = bt.integrate_rays_host(cam, th2, ph2, opts="plain")
    assert np.array_equal(got2[3], h2[3]) and np.array_equal(got2[2], h2[2])
    assert ang_err(got2[0], got2[1], h2[0], h2[1]).max() <= TOL


def test_static_entry_point_rejects_oversize(bt, cuda):
    cap = bt.lib().bt_integrate_rays_host_static_capacity()
    assert cap == 65536
    cam = bt.Camera(np.pi / 2, 0.0, 30.0, 0.0, a=0.6)
    th, ph = seeded_rays(cap + 1, seed=3)
    with pytest.raises(bt.BtError, match="static staging capacity"):
        run_static(bt, cam, th, ph, 0.6)
