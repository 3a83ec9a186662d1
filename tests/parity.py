"""Shared parity helpers for the tests (angles, tolerances, seeded inputs)."""
import numpy as np

TWO_PI = 2 * np.pi

# Seeded synthetic cameras of the benchmark configurations:
#   C1 static camera at r = 30M, theta = pi/2, a = 0.6      (Camera.h:27)
#   C2 Keplerian orbit at r = 5M, theta = pi/2, a = 0.999  (Camera.h:40)
#   C5 Keplerian orbit at r = 8M, theta = 1.2,  a = 0.99
CAMERAS = {
    "c1": dict(kind="static", a=0.6, theta=np.pi / 2, phi=0.0, r=30.0, speed=0.0),
    "c2": dict(kind="orbit", a=0.999, theta=np.pi / 2, phi=0.0, r=5.0, br=0.0, btheta=0.0, bphi=1.0),
    "c5": dict(kind="orbit", a=0.99, theta=1.2, phi=0.0, r=8.0, br=0.0, btheta=0.0, bphi=1.0),
}


def oracle_camera(oracle, name, ref=False):
    c = CAMERAS[name]
    if c["kind"] == "static":
        return oracle.camera_static(c["a"], c["theta"], c["phi"], c["r"], c["speed"], ref=ref), c["a"]
    return oracle.camera_orbit(c["a"], c["theta"], c["phi"], c["r"], c["br"], c["btheta"],
                               c["bphi"], ref=ref), c["a"]


def seeded_rays(n, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, np.pi, n), rng.uniform(0, TWO_PI, n)


def ang_err(t0, p0, t1, p1):
    """Per-ray angular disagreement: max(|dtheta|, |dphi| wrapped to [-pi, pi])."""
    dt = np.abs(np.asarray(t0) - np.asarray(t1))
    dp = np.asarray(p0) - np.asarray(p1)
    dp = np.abs((dp + np.pi) % TWO_PI - np.pi)
    return np.maximum(dt, dp)
