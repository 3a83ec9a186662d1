"""The C-ABI library loads and exports every symbol include/*.h declares
(no GPU needed), and the host-only entry points agree with the oracle."""
import os
import re

import numpy as np
import pytest

from parity import CAMERAS, oracle_camera

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bt_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(bt):
    import ctypes
    lib = ctypes.CDLL(bt._lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_errors(bt):
    lib = bt.lib()
    assert b"sm_100a" in lib.bt_version()


@pytest.mark.parametrize("name", sorted(CAMERAS))
def test_camera_host_matches_oracle(bt, oracle_mod, name):
    c = CAMERAS[name]
    ref, a = oracle_camera(oracle_mod, name)
    if c["kind"] == "static":
        cam = bt.Camera(c["theta"], c["phi"], c["r"], c["speed"], a=a)
    else:
        cam = bt.Camera(c["theta"], c["phi"], c["r"], c["br"], c["btheta"], c["bphi"], a=a)
    assert np.array_equal(cam.as_array(), ref)


def test_blackhole_sets_current_spin(bt):
    bh = bt.BlackHole(0.42)
    cam = bt.Camera(np.pi / 2, 0.0, 10.0, 0.0)
    assert cam.a == 0.42 and bh.getAngVel(2.0) == 0.84


def test_grid_dims(bt, oracle_mod):
    for ml in (3, 6, 11):
        for ang in (True, False):
            assert bt.grid_dims(ml, ang) == oracle_mod.grid_dims(ml, ang)


def test_bad_arguments_raise(bt):
    with pytest.raises(bt.BtError):
        bt.grid_dims(0, True)
    with pytest.raises(bt.BtError):
        bt.Camera(np.pi / 2, 0.0, -1.0, 0.0, a=0.5)
