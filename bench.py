#!/usr/bin/env python
"""Benchmark of the BlackTracer hot path on B200.

Headline (value): geodesics/s of building the adaptive camera-sky grid of the
"single large adaptive grid" configuration -- Kerr a/M = 0.999, camera on a
circular equatorial orbit at r = 5M boosted at Keplerian velocity, adaptive
refinement from level 6 (64x128) to level 11 (2048x4096 equivalent) --
through the C ABI (bt_grid_build), in the fast FP64 form by default (the
reference's method with its equations of motion reassociated, Newton-refined
reciprocals and FP32 step control: same grid topology, p99 ~1e-10 rad against
the plain form); the plain form (the
reference's operation order) and the FP32-bulk mixed form are reported beside
it, each with its error against plain.  One step = one complete grid build
(all levels + T-vertex fix).  Also reported: 4K frames (3840x1920 BGRA8 from
an 8192x4096 environment map and 10^6 stars, lensing + redshift on) per
second and p50/p99 frame latency, and the 64-pose batched grid set.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Multi-GPU (torchrun, one rank per GPU): every rank builds its own grid
(replicas; the path has no data exchange), value = all ranks' rays / the
slowest rank's time.  `--impl reference` times the reference's own CPU
integrator on the box's host cores on the same ray set.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("geodesics/s & 4K frames/s, mixed vs plain FP64 on 1 B200 @≤1e-6 rad; p99 ms")
# Algorithmic FP64 work of the plain integrator, counted once from the
# reference's equations (BT/Metric.h:198-270; +,-,*,/,sqrt,sin,cos = 1 flop):
F_EOM = 130          # derivs
F_COMBINE = 270      # the Cash-Karp stage combinations of one attempt
F_CONTROL = 45       # scale, error norm, step-size update
F_ATTEMPT = 6 * F_EOM + F_COMBINE + F_CONTROL
F_SETUP = 1000       # ray set-up + capture test (Newton + golden section), approx.
# The fast form's equations of motion (kerr_fast.cuh), counted the same way:
# 104 flops (3 reciprocals instead of 16 divisions); FMA = 2 flops.
F_EOM_FAST = 104
F_ATTEMPT_FORM = {"plain": F_ATTEMPT, "mixed": F_ATTEMPT,
                  "fast": 6 * F_EOM_FAST + F_COMBINE + F_CONTROL}
WORKLOAD = dict(maxlevel=11, startlevel=6, a=0.999, r=5.0, theta=np.pi / 2)
SEAM_RAYS = 200_000


def replica_rate(units_local, secs_local, dist=None, device="cpu"):
    """Whole-job rate of replicas (one process per GPU, no data exchange):
    the units all ranks processed over the slowest rank's time.  Returns
    (rate, slowest seconds).  With dist None or one rank, the local rate."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return units_local / secs_local, secs_local
    import torch
    t = torch.tensor([secs_local], dtype=torch.float64, device=device)
    u = torch.tensor([float(units_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(u.item()) / float(t.item()), float(t.item())


def hbm_peak():
    """Measured copy bandwidth of this pool's B200s (GB/s), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s)"


def c2_camera(bt):
    return bt.Camera(WORKLOAD["theta"], 0.0, WORKLOAD["r"], 0.0, 0.0, 1.0, a=WORKLOAD["a"])


# Batched grids: 64 camera poses, each an adaptive grid L6 -> L9 (64x128 ->
# 512x1024 equivalent), static cameras at r in [4M, 40M], theta in
# [0.1, pi - 0.1], spins in [0, 0.999], seeded.
BATCH = dict(count=64, maxlevel=9, startlevel=6, seed=20261206)


def batch_poses(bt, count=BATCH["count"], seed=BATCH["seed"]):
    rng = np.random.default_rng(seed)
    r = rng.uniform(4.0, 40.0, count)
    th = rng.uniform(0.1, np.pi - 0.1, count)
    a = rng.uniform(0.0, 0.999, count)
    return [bt.Camera(float(th[k]), 0.0, float(r[k]), 0.0, a=float(a[k]))
            for k in range(count)], [float(x) for x in a]


def latency_floor(bt, torch, grid, d, cam, prec, reps=5):
    """The build's latency floor: each refinement level waits for its longest
    ray, so a level-synchronous build takes at least the sum over levels of
    the time the level's longest ray takes alone.  Each such ray (the one
    with the most steps among the level's integrated vertices; a vertex
    belongs to the level at which its lattice position first appears) is
    integrated alone through bt_integrate_rays, the best of `reps` runs."""
    N, M = grid.N, grid.M
    ml, sl = grid.MAXLEVEL, grid.STARTLVL
    ii = torch.arange(N, device="cuda")[:, None].expand(N, M)
    jj = torch.arange(M, device="cuda")[None, :].expand(N, M)

    def tz(x):
        t = torch.zeros_like(x)
        for b in range(ml - sl):
            t += ((x % (2 << b)) == 0).to(x.dtype)
        return t
    lvl = ml - torch.minimum(torch.minimum(tz(ii), tz(jj)), torch.full_like(ii, ml - sl))
    live = (d["exists"] == 1) & (d["status"] != 1)
    st = torch.where(live, d["steps"].to(torch.int64), torch.full_like(ii, -1))
    stream = torch.cuda.current_stream()
    levels, total_ms, attempts = [], 0.0, 0
    for level in range(sl, ml + 1):
        s_l = torch.where(lvl == level, st, torch.full_like(st, -1))
        k = int(torch.argmax(s_l))
        if int(s_l.view(-1)[k]) < 0:
            continue
        i, j = k // M, k % M
        th = torch.tensor([i / (N - 1) * np.pi], dtype=torch.float64, device="cuda")
        ph = torch.tensor([j / M * 2 * np.pi], dtype=torch.float64, device="cuda")
        best = 1e30
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            bt.integrate_rays(cam, th, ph, opts=prec)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        n_att = int(s_l.view(-1)[k]) + 1
        levels.append({"level": level, "attempts": n_att, "alone_ms": best})
        total_ms += best
        attempts += n_att
    return {"floor_ms": total_ms, "critical_path_attempts": attempts,
            "us_per_attempt_alone": total_ms * 1e3 / max(1, attempts), "levels": levels}


def set_error_vs(Sp, Sm):
    """Per-vertex angular difference of a mixed set against the plain set
    (vertices both hold and both traced to the sky), p99 and max, and whether
    every member's topology (vertex set, block levels) is the same."""
    import torch
    errs, topo = [], True
    for gp, gm in zip(Sp.grids, Sm.grids):
        dp, dm = gp.dense(), gm.dense()
        topo = topo and bool(torch.equal(dp["exists"], dm["exists"]) and
                             torch.equal(dp["blevel"], dm["blevel"]))
        both = ((dp["exists"] == 1) & (dm["exists"] == 1) & (dp["theta"] >= 0) &
                (dm["theta"] >= 0))
        dth = (dp["theta"][both] - dm["theta"][both]).abs()
        dph = ((dp["phi"][both] - dm["phi"][both] + np.pi).remainder(2 * np.pi) - np.pi).abs()
        errs.append(torch.maximum(dth, dph).float().cpu())
    e = torch.cat(errs)
    return float(torch.quantile(e, 0.99)), float(e.max()), topo


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev_index):
        self.dev = dev_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            import tempfile
            fd, self.path = tempfile.mkstemp(prefix="bt_clocks_", suffix=".csv")
            self.f = os.fdopen(fd, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def value_noise_env(torch, rows, cols, seed, cell=64, octaves=4):
    """Seeded value noise in [0, 255], BGR8 (rows, cols, 3) on the device."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    img = torch.zeros((rows, cols, 3), device="cuda", dtype=torch.float32)
    amp, tot = 1.0, 0.0
    for o in range(octaves):
        c = max(2, cell >> o)
        lat = torch.rand((rows // c + 2, cols // c + 2, 3), device="cuda", generator=g)
        y = torch.arange(rows, device="cuda", dtype=torch.float32) / c
        x = torch.arange(cols, device="cuda", dtype=torch.float32) / c
        y0, x0 = y.floor().long(), x.floor().long()
        fy = (y - y0)[:, None, None]
        fx = (x - x0)[None, :, None]
        fy, fx = fy * fy * (3 - 2 * fy), fx * fx * (3 - 2 * fx)
        a = lat[y0][:, x0]
        b = lat[y0][:, x0 + 1]
        cc = lat[y0 + 1][:, x0]
        d = lat[y0 + 1][:, x0 + 1]
        img += amp * ((a * (1 - fx) + b * fx) * (1 - fy) + (cc * (1 - fx) + d * fx) * fy)
        tot += amp
        amp *= 0.5
    return (img / tot * 255.0).clamp(0, 255).to(torch.uint8).contiguous()


def synthetic_stars(n, seed, tmin=3000.0, tmax=30000.0):
    rng = np.random.default_rng(seed)
    theta = np.arccos(1 - 2 * rng.uniform(0, 1, n))
    phi = 2 * np.pi * rng.uniform(0, 1, n)
    mag = rng.exponential(2.0, n)
    T = rng.uniform(tmin, tmax, n)
    c = T / 4600.0
    A, B, Cc = c, 2.32 * c - 2.0, 1.054 * c - 2.32
    bv = ((-B + np.sqrt(B * B - 4 * A * Cc)) / (2 * A)) / 0.92
    return [x.astype(np.float32) for x in (theta, phi, mag, bv)]


def traffic_from_profiles(prec="plain"):
    """Per-launch DRAM bytes of the trace kernel of form `prec` from the
    committed ncu summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", f"k_trace_lattice_{prec}_c2.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


SERVE = dict(rates=(30.0, 60.0, 120.0), sizes=((512, 256), (1920, 960), (3840, 1920)),
             repeat=0.3, recent=10, seed=20261207, r=5.0, maxlevel=11, startlevel=6)


def serve_rates(bt, torch, env, sp, n):
    """The serving configuration: n frame requests per arrival rate, Poisson
    arrivals (seeded), resolution uniform over SERVE['sizes'], spin uniform in
    [0, 0.999], camera on the circular equatorial Keplerian orbit at r = 5M at a
    uniform orbital phase; 30% of requests repeat one of the 10 most recent
    poses.  Grid cache 40 GB, 10^6 resident stars.  Latency = completion -
    submission (the generator submits at the scheduled arrival times)."""
    out = {"workload": f"{n} requests per rate, Poisson arrivals, resolutions "
                       "512x256 / 1920x960 / 3840x1920, a in [0, 0.999], Keplerian orbit "
                       "r=5M at a uniform phase, 30% repeats of the 10 most recent poses; "
                       "grids L6->L11 fast FP64, 40 GB grid cache, 1e6 stars, 8192x4096 env",
           "rates": []}
    pools = {sz: [] for sz in SERVE["sizes"]}
    for rate in SERVE["rates"]:
        rng = np.random.default_rng(SERVE["seed"] + int(rate))
        t_arr = np.cumsum(rng.exponential(1.0 / rate, n))
        poses, recent = [], []
        for k in range(n):
            if recent and rng.uniform() < SERVE["repeat"]:
                poses.append(recent[rng.integers(len(recent))])
            else:
                p = (float(rng.uniform(0, 2 * np.pi)), float(rng.uniform(0.0, 0.999)))
                poses.append(p)
                recent = (recent + [p])[-SERVE["recent"]:]
        sizes = [SERVE["sizes"][i] for i in rng.integers(0, len(SERVE["sizes"]), n)]
        cams = {}
        S = bt.Server(env=env, stars=sp, maxlevel=SERVE["maxlevel"],
                      startlevel=SERVE["startlevel"], precision="fast",
                      grid_cache_bytes=40 << 30, render_bytes=40 << 30, max_inflight=16)
        # warm-up outside the timed schedule: render slots of every size (16 each)
        # and the generator's pinned output buffers
        wcam = bt.Camera(np.pi / 2, 0.0, SERVE["r"], 0.0, 0.0, 1.0, a=0.5)
        for (W, H) in SERVE["sizes"]:
            while len(pools[(W, H)]) < 32:
                pools[(W, H)].append(torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True))
            for q in range(16):
                S.submit(10**9 + q, W, H, wcam, 0.5, pools[(W, H)][q])
            got = 0
            while got < 16:
                got += len(S.poll(wait_ms=50))
        # objects of earlier measurements that sit in reference cycles are
        # freed here rather than by a collection inside the timed schedule,
        # where a cudaFree of gigabytes would hold up the server's launches
        gc.collect()
        torch.cuda.synchronize()
        st0 = S.stats()
        used = {}
        lat, done = {}, 0
        t0 = time.perf_counter()

        def collect(wait_ms=0):
            nonlocal done
            for c in S.poll(wait_ms=wait_ms):
                assert c["status"] == 0, c
                lat[c["id"]] = (c["t_done"] - c["t_submit"], c["grid_reused"],
                                c["t_admit"] - c["t_submit"])
                pools[used.pop(c["id"])[0]].append(used_buf.pop(c["id"]))
                done += 1

        used_buf = {}
        for k in range(n):
            while time.perf_counter() - t0 < t_arr[k]:
                collect()
                time.sleep(0.0002)
            W, H = sizes[k]
            ph, a = poses[k]
            if poses[k] not in cams:
                cams[poses[k]] = bt.Camera(np.pi / 2, ph, SERVE["r"], 0.0, 0.0, 1.0, a=a)
            buf = pools[(W, H)].pop() if pools[(W, H)] else torch.empty(
                (H, W, 4), dtype=torch.uint8, pin_memory=True)
            used[k] = ((W, H),)
            used_buf[k] = buf
            S.submit(k, W, H, cams[poses[k]], a, buf)
        while done < n:
            collect(wait_ms=20)
        wall = time.perf_counter() - t0
        st = S.stats()
        S.close()
        L = np.array([lat[k][0] for k in range(n)]) * 1e3
        Wt = np.array([lat[k][2] for k in range(n)]) * 1e3
        reused = np.array([lat[k][1] for k in range(n)], bool)
        by_size = {}
        for (W, H) in SERVE["sizes"]:
            sel = np.array([sizes[k] == (W, H) for k in range(n)])
            if sel.any():
                by_size[f"{W}x{H}"] = {"p50_ms": float(np.percentile(L[sel], 50)),
                                       "p99_ms": float(np.percentile(L[sel], 99))}
        out["rates"].append({
            "rate_rps": rate, "requests": n, "throughput_rps": n / wall,
            "p50_ms": float(np.percentile(L, 50)), "p99_ms": float(np.percentile(L, 99)),
            "mean_ms": float(L.mean()), "by_size": by_size,
            "admission_wait_p99_ms": float(np.percentile(Wt, 99)),
            "p99_ms_grid_reused": float(np.percentile(L[reused], 99)) if reused.any() else None,
            "p99_ms_grid_built": float(np.percentile(L[~reused], 99)) if (~reused).any() else None,
            "grid_hits": st["grid_hits"] - st0["grid_hits"],
            "grid_misses": st["grid_misses"] - st0["grid_misses"],
            "grid_sets_built": st["build_sets"] - st0["build_sets"],
            "evictions": st["evictions"] - st0["evictions"], "wall_s": wall})
    return out


FULL = dict(a=0.99, r=8.0, theta=1.2, maxlevel=12, startlevel=6, W=7680, H=3840,
            env=(8192, 16384), stars=10_000_000, tree_level=18, psf=33, seed=20261208)


def full_frame(bt, torch, n_frames):
    """The full-frame configuration: Kerr a = 0.99, static camera at r = 8M,
    theta = 1.2; adaptive grid L6 -> L12 (4096x8192 equivalent) in the fast FP64
    form; 7680x3840 output from a 16384x8192 value-noise environment; 10^7
    stars (tree level 18) with a 33x33 Airy diffraction sprite whose footprint
    scales with the pixel's magnification; colours from the 1024-entry FP32
    blackbody table.  Grid build and frame timed separately (CUDA events)."""
    stream = torch.cuda.current_stream()
    cam = bt.Camera(FULL["theta"], 0.0, FULL["r"], 0.0, a=FULL["a"])
    g = bt.Grid(FULL["maxlevel"], FULL["startlevel"], True, cam, opts="fast")
    for _ in range(2):
        g.build()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    g.build()
    ev[1].record(stream)
    torch.cuda.synchronize()
    build_ms = ev[0].elapsed_time(ev[1])
    rays = g.traced
    t0 = time.perf_counter()
    rows, cols = FULL["env"]
    bgr = value_noise_env(torch, rows, cols, seed=FULL["seed"])
    env = bt.Environment(bgr)
    del bgr
    th, ph, mag, bv = synthetic_stars(FULL["stars"], seed=FULL["seed"] + 1)
    sp = bt.StarProcessor(th, ph, mag, bv, treeLevel=FULL["tree_level"],
                          psf=bt.psf_airy(FULL["psf"], 4.0))
    del th, ph, mag, bv
    setup_s = time.perf_counter() - t0
    W, H = FULL["W"], FULL["H"]
    viewer = bt.Viewer(np.pi / 2, 0.0, 0.0, W, H, True)
    R = bt.Renderer(W, H)
    out = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    kw = dict(env=env, stars=sp, lr=True, diffraction=True, psf_scale=True, bb_table=1, out=out)
    for _ in range(2):
        R.render(g, viewer, cam, **kw)
    torch.cuda.synchronize()
    lat = []
    for _ in range(n_frames):
        ev[0].record(stream)
        R.render(g, viewer, cam, **kw)
        ev[1].record(stream)
        torch.cuda.synchronize()
        lat.append(ev[0].elapsed_time(ev[1]))
    lat = np.array(lat)
    res = {"workload": "Kerr a=0.99, static camera r=8M theta=1.2; grid L6->L12 fast FP64; "
                       "7680x3840 from 16384x8192 value-noise env; 1e7 stars (tree level 18), "
                       "33x33 Airy PSF scaled by sqrt(magnification), 1024-entry FP32 "
                       "blackbody table",
           "grid_build_ms": build_ms, "grid_rays": rays,
           "grid_geodesics_per_s": rays / (build_ms / 1e3),
           "frame_p50_ms": float(np.percentile(lat, 50)),
           "frame_p99_ms": float(np.percentile(lat, 99)), "frames": n_frames,
           "frame_plus_grid_ms": float(np.percentile(lat, 50)) + build_ms,
           "setup_s": setup_s}
    t0 = time.perf_counter()
    cen = R.census()
    res["star_census"] = {
        "pixels": cen["star_pixels"],
        "candidates_per_pixel_reference": cen["star_candidates_ref"] / max(1, cen["star_pixels"]),
        "candidates_per_pixel": cen["star_candidates"] / max(1, cen["star_pixels"]),
        "hits_per_pixel": cen["star_hits"] / max(1, cen["star_pixels"]),
        "heavy_share_of_candidates": cen["heavy_candidates"] / max(1, cen["star_candidates"]),
        "heavy_share_of_hits": cen["heavy_hits"] / max(1, cen["star_hits"]),
        "census_s": time.perf_counter() - t0}
    del R, out, sp, env, g
    torch.cuda.empty_cache()
    return res


def cpu_reference_arm(args):
    """--impl reference: the reference's own CPU integrator
    (Grid::integration_wrapper, compiled in place into oracle/_ref) on all
    host cores, over the rays the workload's grid traces."""
    import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not oracle.have_ref():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libbtref.so was not built (the reference tree was "
                          "absent when the library was built)"}))
        return 0
    cam = oracle.camera_orbit(WORKLOAD["a"], WORKLOAD["theta"], 0.0, WORKLOAD["r"], 0, 0, 1)
    g = oracle.grid_build(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, cam,
                          WORKLOAD["a"], tfix=0)
    # the ray set of the grid: every traced vertex (pole copies are not traced)
    ii, jj = np.nonzero(g["exists"])
    keep = ~(((ii == 0) | (ii == g["N"] - 1)) & (jj != 0))
    ii, jj = ii[keep], jj[keep]
    th = ii / (g["N"] - 1) * np.pi
    ph = jj / g["M"] * 2 * np.pi
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle.integrate_rays(cam, WORKLOAD["a"], th[:2000], ph[:2000], ref=True, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.integrate_rays(cam, WORKLOAD["a"], th, ph, ref=True, nthreads=cores)
    el = time.perf_counter() - t0
    v = len(th) * args.steps / el
    line = {
        "metric": METRIC, "value": v, "unit": "geodesics/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "adaptive grid L6->L11, a=0.999, r=5M equatorial Keplerian "
                               "camera: the grid's traced rays", "rays": int(len(th)),
                   "parallelism": f"{cores} host threads"},
        "cpu_baseline": {"value": v, "unit": "geodesics/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"{len(th)} rays of the workload's grid per step "
                                   "through Grid::integration_wrapper, split over host threads"},
        "e2e": {"value": v, "unit": "geodesics/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=20, help="4K frames to time (0 = skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fast", choices=["fast", "plain", "mixed"],
                    help="integrator form of the headline value")
    ap.add_argument("--launch", default=None,
                    help="THREADS,BLOCKS_PER_SM,REFILL for the headline grid's trace launch "
                         "instead of the autotuner's choice (for reproducible profiles)")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="skip the 64-pose batched-grid measurement")
    ap.add_argument("--no-c5", dest="c5", action="store_false",
                    help="skip the full-frame measurement (L12, 8K, 10^7 stars, diffraction)")
    ap.add_argument("--frames-c5", type=int, default=5, help="timed full 8K frames")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests per arrival rate of the serving measurement (0 = skip)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return cpu_reference_arm(args)

    import torch
    import torch.distributed as dist

    import blacktracer_b200 as bt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    stream = torch.cuda.current_stream()
    cam = c2_camera(bt)
    prec_main = args.precision
    opts = bt.IntegOpts(prec_main)
    grid = bt.Grid(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, cam, opts=opts)
    grid.set_timing(True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)

    # algorithmic FP64 work of one build (identical every build)
    grid.build()
    d = grid.dense()
    steps = d["steps"][d["status"] <= 2].to(torch.int64)
    st_all = d["steps"].to(torch.int64)
    integrated = (d["exists"] == 1) & (d["status"] != 1)
    traced = int(grid.info().traced)
    flops_build = float(((st_all[integrated] + 1).sum().item()) * F_ATTEMPT_FORM[prec_main] +
                        traced * F_SETUP)
    latency = latency_floor(bt, torch, grid, d, cam, prec_main)
    del d, steps, st_all, integrated
    # the launch configuration from the project's autotuner (not timed), or a
    # fixed one
    if args.launch:
        t_, b_, r_ = (int(x) for x in args.launch.split(","))
        grid.set_shape(t_, b_, r_)
        tuned_main = {"shape": (t_, b_, r_), "flow": 0}
    else:
        tuned_main = grid.tune(repeats=3)

    # the trace launches' device time per build (the roofline's kernel time),
    # from eager builds with CUDA events around each trace launch
    for _ in range(args.warmup):
        grid.build()
    n_eager = max(3, args.steps // 4)
    trace_ms, launches = 0.0, 0
    for _ in range(n_eager):
        flush.zero_()
        grid.build()
        inf = grid.info()  # synchronises
        trace_ms += float(inf.trace_ms)
        launches += int(inf.trace_launches)
    trace_ms_build, launches_build = trace_ms / n_eager, launches / n_eager
    # the timed builds: each a replay of the build's CUDA graph
    grid.set_graph(True)
    for _ in range(args.warmup):
        grid.build()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    total_ms, all_launches = 0.0, 0
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        grid.build()
        e1.record(stream)
        inf = grid.info()  # synchronises
        total_ms += e0.elapsed_time(e1)
        all_launches += int(inf.launches)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    value, max_s = replica_rate(traced * args.steps, total_ms / 1e3,
                                dist if world > 1 else None, "cuda")
    max_ms = max_s * 1e3

    # the other two forms, same workload (reported beside the headline), with
    # their error against the plain form
    other = {}
    ref_dense = None
    for prec in [p_ for p_ in ("plain", "fast", "mixed") if p_ != prec_main]:
        gm = bt.Grid(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, cam, opts=prec)
        tuned_o = gm.tune(repeats=3)
        gm.set_graph(True)  # timed like the headline
        for _ in range(3):
            gm.build()
        torch.cuda.synchronize()
        t_o = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            gm.build()
            e1.record(stream)
            torch.cuda.synchronize()
            t_o += e0.elapsed_time(e1)
        o_value = int(gm.info().traced) * args.steps / (t_o / 1e3)
        if prec == "plain":
            ref_dense = gm.dense()
        dp = ref_dense if ref_dense is not None else grid.dense()
        dm = gm.dense() if prec != "plain" else grid.dense()
        both = (dp["exists"] == 1) & (dm["exists"] == 1) & (dp["theta"] >= 0) & (dm["theta"] >= 0)
        dth = (dp["theta"][both] - dm["theta"][both]).abs()
        dph = (dp["phi"][both] - dm["phi"][both] + np.pi).remainder(2 * np.pi) - np.pi
        err = torch.maximum(dth, dph.abs()).float().cpu()
        other[prec] = {
            "value": o_value, "unit": "geodesics/s",
            "ratio_to_headline": o_value / (traced * args.steps / (total_ms / 1e3)),
            "p99_rad_vs_plain": float(torch.quantile(err, 0.99)) if err.numel() else None,
            "max_rad_vs_plain": float(err.max()) if err.numel() else None,
            "topology_exact": bool(torch.equal(dp["exists"], dm["exists"]) and
                                   torch.equal(dp["blevel"], dm["blevel"])),
            "tuned": {"shape": tuned_o["shape"], "flow": tuned_o["flow"],
                      "fp64_band": tuned_o["fp64_band"] if prec == "mixed" else None}}
        if prec != "plain":
            other[prec]["error_vs"] = "plain"
        else:
            other[prec]["error_vs"] = prec_main + " (the headline form)"
        del dp, dm, gm
    del ref_dense

    # the refinement levels as one persistent launch (set_flow): the same grid,
    # timed like the forms above, against the level-by-level headline build
    flow_grid = {}
    head = grid.dense()
    for bps in (1, 2):
        gf = bt.Grid(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, cam, opts=prec_main)
        gf.set_flow(True, blocks_per_sm=bps)
        gf.set_graph(True)  # timed like the headline
        for _ in range(3):
            gf.build()
        torch.cuda.synchronize()
        t_f = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            gf.build()
            e1.record(stream)
            torch.cuda.synchronize()
            t_f += e0.elapsed_time(e1)
        df = gf.dense()
        flow_grid[f"{bps}_blocks_per_sm"] = {
            "ms_per_build": t_f / args.steps,
            "level_build_ms": total_ms / args.steps,
            "speed_vs_level": (total_ms / args.steps) / (t_f / args.steps),
            "same_grid": bool(all(torch.equal(head[k], df[k]) for k in head)),
            "flags": int(gf.info().flags)}
        del gf, df
    del head

    # end to end through the C ABI with host buffers: every step builds the
    # grid and exports it (CamToCel / steps / blockLevels, compacted in key
    # order) into pinned host memory.  Two grids of the same configuration
    # alternate: the builds run one after another on `stream`, and each
    # build's export runs on a second stream while the next build runs
    ex = grid.export()
    nv, nb = len(ex["vi"]), len(ex["bi"])
    d2h = nv * (4 + 4 + 8 + 8 + 4) + nb * (4 + 4 + 1)
    h2d = 12 * 8 + 8  # camera fields + spin, passed by value
    twin = bt.Grid(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, cam, opts=prec_main)
    if tuned_main["flow"]:
        twin.set_flow(True, blocks_per_sm=tuned_main["flow"])
    else:
        twin.set_shape(*tuned_main["shape"])
    twin.set_graph(True)
    pair = (grid, twin)
    bufs = (ex["_buffers"], twin.export()["_buffers"])
    copy_stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        twin.build()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    built = [None, None]
    for step in range(args.steps + 1):
        if step < args.steps:
            pair[step % 2].build()
            built[step % 2] = torch.cuda.Event()
            built[step % 2].record(stream)
        if step:
            k = (step - 1) % 2
            copy_stream.wait_event(built[k])
            pair[k].export(out=bufs[k], stream=copy_stream)
    torch.cuda.synchronize()
    barrier()
    del twin, pair
    e2e_value, e2e_s = replica_rate(traced * args.steps, time.perf_counter() - t0,
                                    dist if world > 1 else None, "cuda")

    # the integration seam (bt_integrate_rays, device arrays): 2x10^5 rays of
    # the same camera, directions uniform on the camera sky (seeded), each
    # form timed with CUDA events; the rays are the same every step
    seam = {"workload": f"{SEAM_RAYS} rays, camera r=5M Keplerian a=0.999, directions "
                        "uniform on the camera sky (seeded), bt_integrate_rays on device "
                        "arrays", "rays": SEAM_RAYS}
    rng = np.random.default_rng(20261209)
    th_s = torch.tensor(np.arccos(1 - 2 * rng.uniform(0, 1, SEAM_RAYS)), device="cuda")
    ph_s = torch.tensor(rng.uniform(0, 2 * np.pi, SEAM_RAYS), device="cuda")
    for prec in ("plain", "fast"):
        for _ in range(2):
            bt.integrate_rays(cam, th_s, ph_s, opts=prec)
        torch.cuda.synchronize()
        reps = 5
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            bt.integrate_rays(cam, th_s, ph_s, opts=prec)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        seam[prec] = {"ms": ms, "geodesics_per_s": SEAM_RAYS / (ms / 1e3)}
    del th_s, ph_s

    # roofline of the dominant kernel (the ray-tracing launches)
    import ctypes as C
    pk = C.c_double()
    bt._lib.check(bt.lib().bt_probe_fp64_tflops(C.byref(pk), C.c_void_p(stream.cuda_stream)))
    peak = pk.value
    per_launch_ms = trace_ms_build / max(1.0, launches_build)
    achieved = flops_build / (trace_ms_build / 1e3) / 1e12
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "traffic": traffic_from_profiles(prec_main),
                "kernel": "k_trace_lattice<%sPolicy>" % prec_main.capitalize(),
                "peak_source": "measured in this run: independent-chain DFMA probe "
                               "(bt_probe_fp64_tflops); MEASURED_PEAKS.json has no FP64 entry",
                "flops_per_build": flops_build, "trace_ms_per_build": trace_ms_build,
                "trace_ms_from": f"{n_eager} eager builds with events around the trace launches",
                "launches_per_build": launches_build,
                "avg_launch_ms": per_launch_ms,
                # one grid is bound by its levels' longest rays, not the FP64 pipe
                "latency_roofline": {**latency,
                                     "frac": latency["floor_ms"] / trace_ms_build,
                                     "note": "sum over levels of the level's longest ray "
                                             "integrated alone, over the trace time per "
                                             "build"}}

    # resident environment (8192x4096) and star set (10^6 stars, tree level 14)
    env = sp = None
    if args.frames > 0 or args.serve_requests > 0:
        bgr = value_noise_env(torch, 4096, 8192, seed=20261204)
        env = bt.Environment(bgr)
        del bgr
        stars = synthetic_stars(1_000_000, seed=20261205)
        sp = bt.StarProcessor(*stars, treeLevel=14)

    # 4K frames with resident grid, environment and stars
    frames = None
    if args.frames > 0:
        W, H = 3840, 1920
        viewer = bt.Viewer(np.pi / 2, 0.0, 0.0, W, H, True)
        R = bt.Renderer(W, H)
        out = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
        host = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
        for _ in range(3):
            R.render(grid, viewer, cam, env=env, stars=sp, lr=True, out=out)
        torch.cuda.synchronize()
        lat = []
        for _ in range(args.frames):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            R.render(grid, viewer, cam, env=env, stars=sp, lr=True, out=out)
            e1.record(stream)
            torch.cuda.synchronize()
            lat.append(e0.elapsed_time(e1))
        lat_e2e = []
        for _ in range(args.frames):
            t0 = time.perf_counter()
            R.render(grid, viewer, cam, env=env, stars=sp, lr=True, out=out)
            host.copy_(out, non_blocking=True)
            torch.cuda.synchronize()
            lat_e2e.append((time.perf_counter() - t0) * 1e3)
        lat = np.array(lat)
        # map roofline: algorithmic bytes of the frame over its p50 time
        cen = R.census()
        gptr, grows, gcols, _ = grid.map_grid()
        n_stars = int(sp.starSize)
        algo = (8 * grows * gcols + 8 * (W + 1) * (H + 1) + 32 * cen["env_columns"] +
                16 * n_stars + 4 * W * H)
        hbm, hbm_src = hbm_peak()
        ach = algo / (float(np.percentile(lat, 50)) / 1e3) / 1e9
        map_roofline = {
            "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "peak_source": hbm_src, "algorithmic_bytes": int(algo),
            "bytes_formula": "8*GN*GM (map grid) + 8*(W+1)(H+1) (view) + 32*sum(pixNum+1) "
                             "(summed-area pairs) + 16*N_stars + 4*W*H (BGRA8 out)",
            "env_columns": cen["env_columns"], "note": "whole frame (every map kernel) at "
                                                       "the p50 frame time"}
        star_census = {
            "pixels": cen["star_pixels"],
            "candidates_per_pixel_reference": cen["star_candidates_ref"] / max(1, cen["star_pixels"]),
            "candidates_per_pixel": cen["star_candidates"] / max(1, cen["star_pixels"]),
            "hits_per_pixel": cen["star_hits"] / max(1, cen["star_pixels"]),
            "heavy_share_of_candidates": cen["heavy_candidates"] / max(1, cen["star_candidates"]),
            "heavy_share_of_hits": cen["heavy_hits"] / max(1, cen["star_hits"]),
            "note": "reference: stars of the kd-tree nodes its search emits (starsToCheck); "
                    "this build: stars of the leaves left after node-box pruning; hits: stars "
                    "inside the pixel's quad; heavy: pixels with more than 2048 candidates"}
        cpu_map = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            import oracle
            if oracle.have_ref_map():
                from blacktracer_b200.render import _device_view
                gmap = _device_view(gptr, (grows * gcols, 2), torch.float32).cpu().numpy()
                sat = env.sat().cpu().numpy()
                cores = os.cpu_count() or 1
                rt = oracle.ref_map_time(gmap, grows, gcols, grid.MAXLEVEL,
                                         viewer.viewMatrix.cpu().numpy(), W, H,
                                         cam.getParamArray(), sat, env.rows, env.cols,
                                         (sp.starPos, sp.starMag, sp.binaryStarTree,
                                          sp.treeLevel), row_stride=16, nthreads=cores)
                del gmap, sat
                cpu_map = {"value": 1.0 / rt["frame_s"], "unit": "frames/s", "cores": cores,
                           "kind": "reference", "phases_s": rt,
                           "sample": f"the reference's map kernels (BT/MakeImageKernel.cu) "
                                     f"compiled for the host, OpenMP over rows: corners and "
                                     f"areas over the whole 4K frame, environment and stars "
                                     f"over every 16th row ({rt['rows_sampled']} rows) scaled "
                                     f"to the frame; the per-pixel sums and the composite "
                                     f"are not timed"}
        frames = {"fps": float(1e3 / lat.mean()), "p50_ms": float(np.percentile(lat, 50)),
                  "p99_ms": float(np.percentile(lat, 99)),
                  "e2e_fps": float(1e3 / np.mean(lat_e2e)),
                  "e2e_p99_ms": float(np.percentile(lat_e2e, 99)),
                  "d2h_bytes_per_frame": W * H * 4, "width": W, "height": H,
                  "env": "8192x4096 BGR8 value noise", "stars": 1_000_000, "tree_level": 14,
                  "lensing_redshift": True, "roofline": map_roofline,
                  "star_census": star_census, "cpu_baseline": cpu_map}

    # batched grids (64 poses, L6 -> L9): one set, graph-captured, launch shape
    # from the autotuner; plain and mixed; the sets are larger than L2
    batched = None
    if args.batch:
        cams_b, spins_b = batch_poses(bt)
        res = {}
        sets = {}
        for prec in ("plain", "fast", "mixed"):
            Sb = bt.GridSet(BATCH["maxlevel"], BATCH["startlevel"], True, BATCH["count"],
                            opts=prec)
            tuned = Sb.tune(cams_b, spins_b, p99_target=1e-6, repeats=1)
            if tuned["flow"]:
                Sb.set_flow(True, blocks_per_sm=tuned["flow"])
            shape = tuned["shape"]
            Sb.set_graph(True)
            for _ in range(3):
                Sb.build(cams_b, spins_b)
            torch.cuda.synchronize()
            nb_steps = max(2, args.steps // 4)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(nb_steps):
                Sb.build(cams_b, spins_b)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / nb_steps
            rays = Sb.traced
            res[prec] = {"value": rays / (ms / 1e3), "unit": "geodesics/s",
                         "ms_per_set": ms, "rays_per_set": rays,
                         "trace_shape": {"threads": shape[0], "blocks_per_sm": shape[1],
                                         "refill": shape[2]},
                         "tuner": {k: tuned[k] for k in ("flow", "level_ms", "flow_ms",
                                                         "candidates", "fp64_band",
                                                         "band_met", "band_p99_rad")},
                         "launches_per_set": int(Sb.info().launches)}
            if prec != "mixed":
                # FP64 work of the set per build over the whole build time
                attempts = 0
                for gq in Sb.grids:
                    dq = gq.dense()
                    live = (dq["exists"] == 1) & (dq["status"] != 1)
                    attempts += int((dq["steps"][live].to(torch.int64) + 1).sum().item())
                    del dq
                fl = float(attempts * F_ATTEMPT_FORM[prec] + rays * F_SETUP)
                ach = fl / (ms / 1e3) / 1e12
                res[prec]["roofline"] = {
                    "bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                    "frac": ach / peak if peak else None, "flops_per_set": fl,
                    "note": "whole set build time (all kernels), FP64 peak as the headline's"}
            if prec == "fast":
                # the same set as one persistent launch per build
                Sb.set_flow(True, blocks_per_sm=2)
                for _ in range(3):
                    Sb.build(cams_b, spins_b)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for _ in range(nb_steps):
                    Sb.build(cams_b, spins_b)
                e1.record(stream)
                torch.cuda.synchronize()
                ms_f = e0.elapsed_time(e1) / nb_steps
                res[prec]["one_launch"] = {
                    "ms_per_set": ms_f, "value": rays / (ms_f / 1e3),
                    "speed_vs_level": ms / ms_f if not tuned["flow"] else None,
                    "blocks_per_sm": 2, "flags": int(Sb.info().flags)}
                Sb.set_flow(bool(tuned["flow"]), blocks_per_sm=tuned["flow"] or 2)
            sets[prec] = Sb
        for prec in ("fast", "mixed"):
            p99, mx, topo = set_error_vs(sets["plain"], sets[prec])
            res[prec].update({"p99_rad_vs_plain": p99, "max_rad_vs_plain": mx,
                              "topology_exact": topo})
        batched = {"workload": f"{BATCH['count']} poses, adaptive L6->L9 (512x1024 "
                               "equivalent), static cameras r in [4M,40M], theta in "
                               "[0.1, pi-0.1], a in [0, 0.999], seeded; one set per step, "
                               "CUDA graph replay, configuration from the autotuner "
                               "(bt_batch_tune: trace shape x refill, level or one-launch "
                               "build; the mixed form's FP64 band by a 1e-6 rad p99 target)",
                   "plain": res["plain"], "fast": res["fast"], "mixed": res["mixed"],
                   "speedup_vs_plain_set": {
                       k: res[k]["value"] / res["plain"]["value"] for k in ("fast", "mixed")}}
        del sets, Sb

    # full frame at scale: L12 grid, 7680x3840 from a 16384x8192 environment,
    # 10^7 stars, Airy PSF diffraction scaled by magnification, 1024-entry table
    full = None
    if args.c5 and rank == 0:
        full = full_frame(bt, torch, args.frames_c5)

    # serving loop: Poisson arrivals at 30, 60 and 120 requests/s
    serving = None
    if args.serve_requests > 0 and rank == 0:
        serving = serve_rates(bt, torch, env, sp, args.serve_requests)

    # CPU baseline: the reference's own Grid constructor, one thread, full workload
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.have_ref():
            camr = oracle.camera_orbit(WORKLOAD["a"], WORKLOAD["theta"], 0.0, WORKLOAD["r"], 0, 0, 1,
                                       ref=True)
            secs, n = oracle.ref_grid_time(WORKLOAD["maxlevel"], WORKLOAD["startlevel"], True, camr,
                                           WORKLOAD["a"])
            cpu = {"value": traced / secs, "unit": "geodesics/s", "cores": 1, "kind": "reference",
                   "sample": f"one full grid build (Grid::Grid, L6->L11, {traced} rays, "
                             f"{secs:.2f} s incl. its perfect hash) on one host thread"}
            # 8-way: the grid's rays split into 8 disjoint slices, integration_wrapper
            # on 8 threads (it only reads the camera and the spin)
            d = grid.dense()
            ii, jj = np.nonzero((d["exists"] == 1).cpu().numpy())
            del d
            keep = ~(((ii == 0) | (ii == grid.N - 1)) & (jj != 0))
            th8 = ii[keep] / (grid.N - 1) * np.pi
            ph8 = jj[keep] / grid.M * 2 * np.pi
            t0 = time.perf_counter()
            oracle.integrate_rays(camr, WORKLOAD["a"], th8, ph8, ref=True, nthreads=8)
            s8 = time.perf_counter() - t0
            cpu["eight_way"] = {"value": len(th8) / s8, "unit": "geodesics/s", "cores": 8,
                                "kind": "reference",
                                "sample": f"the grid's {len(th8)} traced rays through "
                                          f"Grid::integration_wrapper on 8 threads "
                                          f"({s8:.2f} s)"}

    # the speed target of the path (at least 5x the plain FP64 form at <= 1e-6 rad
    # p99), like for like: the form that meets 1e-6 rad against plain on the same work
    head = traced * args.steps / (total_ms / 1e3)
    plain_v = other["plain"]["value"] if "plain" in other else head
    target = {"form": prec_main, "goal": ">= 5x plain FP64 at <= 1e-6 rad p99",
              "single_grid_vs_plain": (head if prec_main != "plain" else plain_v) / plain_v}
    if batched is not None:
        target["set_vs_plain_set"] = (batched[prec_main]["value"] /
                                      batched["plain"]["value"])
        target["set_p99_rad_vs_plain"] = batched[prec_main].get("p99_rad_vs_plain")
    if "plain" in other:
        target["single_grid_p99_rad_vs_plain"] = other["plain"]["p99_rad_vs_plain"]
        target["single_grid_max_rad_vs_plain"] = other["plain"]["max_rad_vs_plain"]

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "geodesics/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "adaptive grid L6->L11 (64x128 -> 2048x4096 equivalent), "
                                   "Kerr a=0.999, camera r=5M theta=pi/2 Keplerian orbit; "
                                   f"{prec_main} integrator",
                       "integrator": {"fast": "FP64, reference method with reassociated "
                                              "equations of motion, Newton-refined "
                                              "reciprocals, FP32 error ratio and step "
                                              "factor, FMA (error vs plain under 'plain')",
                                      "plain": "FP64, reference operation order, no FMA",
                                      "mixed": "FP32 bulk, FP64 guards"}[prec_main],
                       "rays_per_build": traced, "l2": "flushed (256 MB write) before every step",
                       "graph": "each timed build replays the build's CUDA graph",
                       "launch": {"from": "--launch" if args.launch else
                                  "bt_grid_tune (the project's autotuner), before timing",
                                  "threads": tuned_main["shape"][0],
                                  "blocks_per_sm": tuned_main["shape"][1],
                                  "refill": tuned_main["shape"][2],
                                  "one_launch_build": tuned_main["flow"]},
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "geodesics/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "api": "bt_grid_build + bt_grid_export to pinned host (CamToCel, steps, "
                           "blockLevels as key-ordered lists) every step; two grids of the "
                           "tuned configuration alternate, builds one after another on one "
                           "stream, each export on a second stream beside the next build"},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": all_launches,
            # the long blocks first: the numbers read most come last
            "serving": serving,
            "full_frame_8k": full,
            "integration_seam": seam,
            "one_launch_build": {"workload": "the headline grid built with set_flow: every "
                                             "refinement level in one persistent launch",
                                 **flow_grid},
            "batched": batched,
            "frames_4k": frames,
            **other,
            "target_5x": target,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
