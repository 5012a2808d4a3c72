"""Seeded synthetic 2D LiDAR scenes for the SDF-SLAM LM path.

The reference ships no generator and its headline workloads are synthetic, so
this module builds worlds of wall segments, drives a robot through them, ray
casts every beam and integrates noisy odometry. The output has exactly the
shape of the reference's ``Dataset`` (src/core/scan.hpp:24-28): one scan of
sensor-frame points per frame and one pose per frame (odometry-integrated, as
for real data), plus the ground-truth poses for error reporting.

Workloads (all seeded with numpy's PCG64):

* ``room``     -- 10-pose closed loop in a room with 4 axis-aligned boxes,
                  180 beams / 360 deg, 40x40 grid at 0.25 m;
* ``floorplan``-- 76-pose loop along a ring corridor of a floor plan with 6-10
                  rooms, 360 beams / 360 deg, 100x100 grid at 0.2 m;
* ``office``   -- 910-pose, 3-lap trajectory through an office with a ring and
                  a cross corridor (1.5-2 m wide, 20-30 rooms), 180 beams /
                  180 deg, 200x200 grid at 0.15 m;
* ``batch``    -- 64 room-style scenes of uneven grid size, pose and beam
                  count, half of them with an active-region state;
* ``request``  -- one room-style scene of log-uniform size for the serving loop.

A grid of n nodes at spacing s spans (n - 1) * s metres
(src/core/grid_map.hpp:18-19), so each world is shrunk by half a metre against
that span and centred in it: e.g. the 10 m room becomes a 9.25 m room inside
the 9.75 m of a 40x40 grid at 0.25 m.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    name: str
    seed: int
    nx: int
    ny: int
    min_corner: tuple
    max_corner: tuple
    segments: np.ndarray            # (S, 4) world walls x0 y0 x1 y1
    gt_poses: np.ndarray            # (F, 3) ground truth
    poses: np.ndarray               # (F, 3) odometry-integrated start poses
    odometry: np.ndarray            # (F-1, 3) relative measurements
    scans: list                     # F arrays (n_i, 2), sensor frame
    options: dict = field(default_factory=dict)   # ProblemOptions fields
    solver: dict = field(default_factory=dict)    # SolverOptions fields

    @property
    def num_frames(self) -> int:
        return len(self.scans)

    @property
    def num_beam_returns(self) -> int:
        return int(sum(len(s) for s in self.scans))


# ------------------------------------------------------------- geometry --

def _box(x0, y0, x1, y1):
    return [(x0, y0, x1, y0), (x1, y0, x1, y1), (x1, y1, x0, y1), (x0, y1, x0, y0)]


def _wall_with_doors(a, b, doors):
    """Axis-aligned wall from a to b with door gaps [(t0, t1)] in wall
    parameter units (metres from a)."""
    ax, ay = a
    bx, by = b
    length = math.hypot(bx - ax, by - ay)
    ux, uy = (bx - ax) / length, (by - ay) / length
    cuts = sorted(doors)
    segs = []
    t = 0.0
    for d0, d1 in cuts:
        if d0 > t + 1e-9:
            segs.append((ax + ux * t, ay + uy * t, ax + ux * d0, ay + uy * d0))
        t = max(t, d1)
    if t < length - 1e-9:
        segs.append((ax + ux * t, ay + uy * t, bx, by))
    return segs


def ray_cast(segments, origins, dirs, max_range, chunk=8192):
    """Nearest hit distance along each ray (inf when nothing within range)."""
    segs = np.asarray(segments, dtype=np.float64)
    a = segs[:, :2]
    e = segs[:, 2:] - a
    out = np.full(len(origins), np.inf)
    for s in range(0, len(origins), chunk):
        o = origins[s:s + chunk, None, :]
        d = dirs[s:s + chunk, None, :]
        denom = d[..., 0] * e[None, :, 1] - d[..., 1] * e[None, :, 0]
        w = a[None, :, :] - o
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (w[..., 0] * e[None, :, 1] - w[..., 1] * e[None, :, 0]) / denom
            u = (w[..., 0] * d[..., 1] - w[..., 1] * d[..., 0]) / denom
        ok = (np.abs(denom) > 1e-12) & (t > 1e-6) & (u >= -1e-12) & (u <= 1 + 1e-12) & (t <= max_range)
        t = np.where(ok, t, np.inf)
        out[s:s + chunk] = t.min(axis=1)
    return out


def _wrap(a):
    return np.arctan2(np.sin(a), np.cos(a))


def _relative(pa, pb):
    """pose.hpp:40-43 on arrays of poses."""
    c, s = np.cos(pa[..., 2]), np.sin(pa[..., 2])
    dx, dy = pb[..., 0] - pa[..., 0], pb[..., 1] - pa[..., 1]
    return np.stack([c * dx + s * dy, -s * dx + c * dy, _wrap(pb[..., 2] - pa[..., 2])], axis=-1)


def _compose(pa, rel):
    """pose.hpp:33-36."""
    c, s = math.cos(pa[2]), math.sin(pa[2])
    return np.array([c * rel[0] - s * rel[1] + pa[0], s * rel[0] + c * rel[1] + pa[1],
                     math.atan2(math.sin(pa[2] + rel[2]), math.cos(pa[2] + rel[2]))])


def _scans(rng, segments, gt, beams, fov, max_range, sigma_r):
    n = len(gt)
    if fov >= 2 * math.pi - 1e-9:
        rel = np.arange(beams) * (2 * math.pi / beams)
    else:
        # beam i at -fov/2 + i * fov / beams (tools/viz/carmen_to_pcd.py:57-70)
        rel = -fov / 2 + np.arange(beams) * (fov / beams)
    ang = gt[:, 2:3] + rel[None, :]
    origins = np.repeat(gt[:, :2], beams, axis=0)
    dirs = np.stack([np.cos(ang), np.sin(ang)], axis=-1).reshape(-1, 2)
    ranges = ray_cast(segments, origins, dirs, max_range).reshape(n, beams)
    noise = rng.normal(0.0, sigma_r, size=ranges.shape)
    scans = []
    for f in range(n):
        hit = np.isfinite(ranges[f])
        r = ranges[f, hit] + noise[f, hit]
        a = rel[hit]
        scans.append(np.stack([r * np.cos(a), r * np.sin(a)], axis=-1))
    return scans


def _odometry(rng, gt, sigma_t, sigma_theta):
    true_rel = _relative(gt[:-1], gt[1:])
    noisy = true_rel + np.stack([rng.normal(0, sigma_t, len(true_rel)),
                                 rng.normal(0, sigma_t, len(true_rel)),
                                 rng.normal(0, sigma_theta, len(true_rel))], axis=-1)
    poses = [gt[0].copy()]
    for r in noisy:
        poses.append(_compose(poses[-1], r))
    poses = np.array(poses)
    # the reference derives odometry from the dataset poses
    # (src/pipeline/runner.cpp:52-59)
    return poses, _relative(poses[:-1], poses[1:])


def _grid(n, spacing, origin=0.0):
    span = (n - 1) * spacing
    return span, (origin, origin), (origin + span, origin + span)


# --------------------------------------------------------------- worlds --

def _loop_poses(center, rx, ry, n, rng, wobble=0.05):
    t = np.arange(n) * (2 * math.pi / n)
    x = center[0] + rx * np.cos(t) + rng.normal(0, wobble, n)
    y = center[1] + ry * np.sin(t) + rng.normal(0, wobble, n)
    heading = np.arctan2(ry * np.cos(t), -rx * np.sin(t)) + rng.normal(0, 0.05, n)
    return np.stack([x, y, _wrap(heading)], axis=-1)


def room_scene(seed=0, grid=40, spacing=0.25, frames=10, beams=180, max_range=8.0,
               sigma_r=0.01, sigma_t=0.01, sigma_theta=0.005, boxes=4, active_region=False,
               hallucination_points=4, iterations=10, name="room"):
    rng = np.random.default_rng(seed)
    span, mn, mx = _grid(grid, spacing)
    lo, hi = mn[0] + 0.25, mx[0] - 0.25
    size = hi - lo
    c = (lo + hi) / 2
    rx, ry = 0.3 * size, 0.27 * size
    gt = _loop_poses((c, c), rx, ry, frames, rng)
    path = _loop_poses((c, c), rx, ry, 256, np.random.default_rng(seed + 1), wobble=0.0)
    segs = _box(lo, lo, hi, hi)
    placed = 0
    tries = 0
    while placed < boxes and tries < 10000:
        tries += 1
        w, h = rng.uniform(0.5, 2.0, size=2) * max(1.0, size / 9.25) ** 0.5
        x0 = rng.uniform(lo + 0.3, hi - 0.3 - w)
        y0 = rng.uniform(lo + 0.3, hi - 0.3 - h)
        dx = np.maximum(np.maximum(x0 - path[:, 0], path[:, 0] - (x0 + w)), 0)
        dy = np.maximum(np.maximum(y0 - path[:, 1], path[:, 1] - (y0 + h)), 0)
        if np.min(np.hypot(dx, dy)) < 0.6:
            continue
        segs += _box(x0, y0, x0 + w, y0 + h)
        placed += 1
    segs = np.array(segs)
    scans = _scans(rng, segs, gt, beams, 2 * math.pi, max_range, sigma_r)
    poses, odo = _odometry(rng, gt, sigma_t, sigma_theta)
    return Scene(name=name, seed=seed, nx=grid, ny=grid, min_corner=mn, max_corner=mx,
                 segments=segs, gt_poses=gt, poses=poses, odometry=odo, scans=scans,
                 options=dict(hallucination_points=hallucination_points, hallucination_step=0.1,
                              active_region=active_region),
                 solver=dict(max_iterations=iterations))


def _ring_loop(lo, hi, n, rng, laps=1, wobble=0.15):
    """Poses along a square ring centre line [lo, hi]^2, counter-clockwise."""
    side = hi - lo
    per = 4 * side
    s = (np.arange(n) * (laps * per / n)) % per
    x = np.empty(n)
    y = np.empty(n)
    hd = np.empty(n)
    for i, d in enumerate(s):
        k = int(d // side)
        u = d - k * side
        if k == 0:
            x[i], y[i], hd[i] = lo + u, lo, 0.0
        elif k == 1:
            x[i], y[i], hd[i] = hi, lo + u, math.pi / 2
        elif k == 2:
            x[i], y[i], hd[i] = hi - u, hi, math.pi
        else:
            x[i], y[i], hd[i] = lo, hi - u, -math.pi / 2
    x += rng.normal(0, wobble, n)
    y += rng.normal(0, wobble, n)
    hd = _wrap(hd + rng.normal(0, 0.08, n))
    return np.stack([x, y, hd], axis=-1)


def _band_rooms(rng, lo, hi, depth, rooms_per_side, door=1.0):
    """Rooms in the outer band of a square building [lo, hi]^2: perpendicular
    partitions plus a corridor-side wall with one door per room."""
    segs = _box(lo, lo, hi, hi)
    inner_lo, inner_hi = lo + depth, hi - depth
    count = 0
    sides = [
        ((lo, inner_lo), (hi, inner_lo), lambda t: [(lo + t, lo, lo + t, inner_lo)]),
        ((lo, inner_hi), (hi, inner_hi), lambda t: [(lo + t, inner_hi, lo + t, hi)]),
        ((inner_lo, inner_lo), (inner_lo, inner_hi), lambda t: [(lo, inner_lo + t, inner_lo, inner_lo + t)]),
        ((inner_hi, inner_lo), (inner_hi, inner_hi), lambda t: [(inner_hi, inner_lo + t, hi, inner_lo + t)]),
    ]
    for (a, b, partition), k in zip(sides, rooms_per_side):
        length = math.hypot(b[0] - a[0], b[1] - a[1])
        edges = np.linspace(0, length, k + 1)
        doors = []
        for r in range(k):
            d0 = rng.uniform(edges[r] + 0.3, max(edges[r] + 0.31, edges[r + 1] - 0.3 - door))
            doors.append((d0, d0 + door))
            if r > 0:
                segs += partition(edges[r])
            count += 1
        segs += _wall_with_doors(a, b, doors)
    return segs, count


def floorplan_scene(seed=1, grid=100, spacing=0.2, frames=76, beams=360, max_range=20.0,
                    sigma_r=0.02, sigma_t=0.02, sigma_theta=0.01, iterations=100,
                    name="floorplan"):
    rng = np.random.default_rng(seed)
    span, mn, mx = _grid(grid, spacing)
    lo, hi = mn[0] + 0.25, mx[0] - 0.25
    size = hi - lo
    corridor = 2.0
    depth = 0.22 * size
    total = int(rng.integers(6, 11))
    per_side = [1, 1, 1, 1]
    for _ in range(total - 4):
        per_side[int(rng.integers(0, 4))] += 1
    segs, _ = _band_rooms(rng, lo, hi, depth, per_side)
    ilo, ihi = lo + depth + corridor, hi - depth - corridor
    segs += _box(ilo, ilo, ihi, ihi)
    segs = np.array(segs)
    c0, c1 = lo + depth + corridor / 2, hi - depth - corridor / 2
    gt = _ring_loop(c0, c1, frames, rng, laps=1, wobble=0.12)
    scans = _scans(rng, segs, gt, beams, 2 * math.pi, max_range, sigma_r)
    poses, odo = _odometry(rng, gt, sigma_t, sigma_theta)
    return Scene(name=name, seed=seed, nx=grid, ny=grid, min_corner=mn, max_corner=mx,
                 segments=segs, gt_poses=gt, poses=poses, odometry=odo, scans=scans,
                 options=dict(hallucination_points=6, hallucination_step=0.1),
                 solver=dict(max_iterations=iterations))


def office_scene(seed=2, grid=200, spacing=0.15, frames=910, beams=180, max_range=30.0,
                 sigma_r=0.01, sigma_t=0.01, sigma_theta=0.005, laps=3, iterations=100,
                 name="office"):
    rng = np.random.default_rng(seed)
    span, mn, mx = _grid(grid, spacing)
    lo, hi = mn[0] + 0.25, mx[0] - 0.25
    size = hi - lo
    corridor = float(rng.uniform(1.5, 2.0))
    depth = 0.17 * size
    per_side = [4, 4, 4, 4]
    segs, rooms = _band_rooms(rng, lo, hi, depth, per_side)
    ilo, ihi = lo + depth + corridor, hi - depth - corridor
    mid = (ilo + ihi) / 2
    half = corridor / 2
    # four inner blocks split by a cross corridor, two rooms each
    for bx0, bx1 in ((ilo, mid - half), (mid + half, ihi)):
        for by0, by1 in ((ilo, mid - half), (mid + half, ihi)):
            segs += _box(bx0, by0, bx1, by1)
            xm = (bx0 + bx1) / 2
            segs.append((xm, by0, xm, by1))
            rooms += 2
    segs = np.array(segs)
    c0, c1 = lo + depth + corridor / 2, hi - depth - corridor / 2
    gt = _ring_loop(c0, c1, frames, rng, laps=laps, wobble=0.1)
    scans = _scans(rng, segs, gt, beams, math.pi, max_range, sigma_r)
    poses, odo = _odometry(rng, gt, sigma_t, sigma_theta)
    return Scene(name=name, seed=seed, nx=grid, ny=grid, min_corner=mn, max_corner=mx,
                 segments=segs, gt_poses=gt, poses=poses, odometry=odo, scans=scans,
                 options=dict(hallucination_points=6, hallucination_step=0.1),
                 solver=dict(max_iterations=iterations))


def batch_scenes(seed=3, count=64):
    """Uneven room-style instances: grid side U[40,150], poses U[10,200],
    beams U[90,360], every other instance with an active-region state."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        g = int(rng.integers(40, 151))
        f = int(rng.integers(10, 201))
        b = int(rng.integers(90, 361))
        out.append(room_scene(seed=seed * 1000 + i, grid=g, spacing=0.25, frames=f, beams=b,
                              max_range=min(30.0, 0.4 * g * 0.25 + 4), active_region=(i % 2 == 1),
                              hallucination_points=4, iterations=20, name=f"batch{i}"))
    return out


def request_scene(seed, grid_range=(40, 200), pose_range=(10, 400), iterations=20):
    """One serving request: log-uniform grid side and pose count."""
    rng = np.random.default_rng(seed)
    g = int(round(math.exp(rng.uniform(math.log(grid_range[0]), math.log(grid_range[1])))))
    f = int(round(math.exp(rng.uniform(math.log(pose_range[0]), math.log(pose_range[1])))))
    return room_scene(seed=seed, grid=g, spacing=0.25, frames=f, beams=180,
                      max_range=min(30.0, 0.4 * g * 0.25 + 4), hallucination_points=4,
                      iterations=iterations, name=f"request{seed}")


WORKLOADS = {
    "room": room_scene,
    "floorplan": floorplan_scene,
    "office": office_scene,
}
