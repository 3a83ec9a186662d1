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


def value_noise_bgr(rows, cols, seed, cell=16, octaves=3, dtype=np.float64):
    """Seeded 2-D value noise in [0, 255] per channel, BGR8 (rows, cols, 3);
    the synthetic environment map of the benchmark configurations (dtype:
    the arithmetic of the interpolation; float32 for the largest maps)."""
    rng = np.random.default_rng(seed)
    img = np.zeros((rows, cols, 3), dtype)
    amp, tot = 1.0, 0.0
    for o in range(octaves):
        c = max(2, cell >> o)
        gr, gc = rows // c + 2, cols // c + 2
        lat = rng.uniform(0, 1, (gr, gc, 3)).astype(dtype)
        y = np.arange(rows) / c
        x = np.arange(cols) / c
        y0, x0 = np.floor(y).astype(int), np.floor(x).astype(int)
        fy = (y - y0)[:, None, None].astype(dtype)
        fx = (x - x0)[None, :, None].astype(dtype)
        fy, fx = fy * fy * (3 - 2 * fy), fx * fx * (3 - 2 * fx)
        a = lat[y0][:, x0]
        b = lat[y0][:, x0 + 1]
        cc = lat[y0 + 1][:, x0]
        d = lat[y0 + 1][:, x0 + 1]
        img += amp * ((a * (1 - fx) + b * fx) * (1 - fy) + (cc * (1 - fx) + d * fx) * fy)
        tot += amp
        amp *= 0.5
    return np.clip(img / tot * 255.0, 0, 255).astype(np.uint8)


def synthetic_stars(n, seed, tmin=3000.0, tmax=30000.0):
    """n stars: uniform on the sphere, magnitude ~ Exp(mean 2), temperature
    ~ U(3000, 30000) K expressed as the B-V index the reference's colour
    formula (46*(1/(0.92bv+1.7) + 1/(0.92bv+0.62)), BT/MakeImageKernel.cu:295)
    maps back to that temperature / 100."""
    rng = np.random.default_rng(seed)
    theta = np.arccos(1 - 2 * rng.uniform(0, 1, n))
    phi = 2 * np.pi * rng.uniform(0, 1, n)
    mag = rng.exponential(2.0, n)
    T = rng.uniform(tmin, tmax, n)
    c = T / 4600.0
    # c = 1/(u+1.7) + 1/(u+0.62), u = 0.92 bv
    A, B, Cc = c, 2.32 * c - 2.0, 1.054 * c - 2.32
    u = (-B + np.sqrt(B * B - 4 * A * Cc)) / (2 * A)
    bv = u / 0.92
    return (theta.astype(np.float32), phi.astype(np.float32), mag.astype(np.float32),
            bv.astype(np.float32))


def map_grid_from_dense(theta, phi, exists, angle):
    """makeGrid (BT/MakeImageKernel.cu:369-384) from a dense grid: float2
    values, (-2,-2) where no vertex exists, the lower hemisphere mirrored for
    half grids (GM/GN > 3).  Returns (grid (rows*GM, 2) float32, rows, GM)."""
    GN, GM = theta.shape
    sym = (GM / GN) > 3
    rows = 2 * GN - 1 if sym else GN
    g = np.full((rows, GM, 2), -2.0, np.float32)
    t = np.where(exists == 1, theta, -2.0).astype(np.float32)
    p = np.where(exists == 1, phi, -2.0).astype(np.float32)
    g[:GN, :, 0], g[:GN, :, 1] = t, p
    if sym:
        for i in range(GN):
            x = rows - i - 1
            tt = t[i].copy()
            m = (tt != -1) & (tt != -2)
            tt[m] = np.float32(np.pi).astype(np.float32) - tt[m]
            g[x, :, 0], g[x, :, 1] = tt, p[i]
    return g.reshape(-1, 2), rows, GM


def sphere_view(width, height):
    """Viewer::makeSphereView (BT/Viewer.h:82-88): float32 corners."""
    i = np.arange(height + 1, dtype=np.float64)[:, None]
    j = np.arange(width + 1, dtype=np.float64)[None, :]
    th = (np.float32(1.0) * i * np.pi / height) * np.ones_like(j)
    ph = (np.float32(1.0) * j * (2 * np.pi) / width) * np.ones_like(i)
    return np.stack([th.astype(np.float32), ph.astype(np.float32)], -1).reshape(-1, 2)
