"""Seeded synthetic scenes in the reference's file formats (.scn, .json, task file).

There is no public data set for this path; these generators stand in for
the benchmark fields.  Conventions: x = east, y = up, z = north; the tower
stands at the origin and the field lies north of it.  The sun direction is
the direction of travel, -(cos e sin a, sin e, cos e cos a) for azimuth a
(clockwise from north) and elevation e.

  small_field   50 flat 4x4 m heliostats on a jittered 10x5 lattice (8 m
                pitch), 8x6 m rectangle receiver at 80 m (vertical, facing
                the field: the scene format has no receiver tilt), 0.05 m
                micro-facets (6400 per heliostat), 10 m grid cells,
                0.05 m receiver pixels (160x120).
  large_field   624 focus-flat 12.84x9.45 m heliostats (4x7 sub-heliostats,
                no gap, focal length = slant range) on radial-staggered rings
                100-750 m over +-70 degrees, cylinder receiver r = 4 m,
                h = 12 m at 115 m, 0.02 m micro-facets (300,664 per
                heliostat), 20 m grid cells, 0.02 m receiver pixels (1257x600).
  uneven_field  one of the batch's seeded fields of uneven size: 200-2500
                square 6-12 m heliostats on radial-staggered rings sized to
                the count, a rectangle (flat heliostats) or cylinder
                (focus-flat 2x2 heliostats) receiver, 0.05 m micro-facets,
                grid cells scaled to the heliostat size.
  huge_field    10,000 flat 10x10 m heliostats on radial-staggered rings
                150-1800 m over +-70 degrees, cylinder receiver r = 10 m,
                h = 20 m at 200 m, 0.05 m micro-facets (40,000 per
                heliostat), 20 m grid cells, 0.05 m receiver pixels.
  two_receiver_field  two towers, each with its receiver and its own grid:
                flat heliostats on a rectangle receiver to the north,
                focus-flat heliostats on a cylinder to the south (the
                reference's multi-receiver, multi-grid scene layout).
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np


def sun_direction(azimuth_deg: float, elevation_deg: float) -> list[float]:
    a, e = math.radians(azimuth_deg), math.radians(elevation_deg)
    return [-(math.cos(e) * math.sin(a)), -math.sin(e), -(math.cos(e) * math.cos(a))]


def sun_positions(days: int = 12, hours: int = 8, latitude_deg: float = 37.0, min_elevation_deg: float = 15.0,
                  max_elevation_deg: float = 80.0) -> np.ndarray:
    """Sun directions (direction of travel) for `days` days spread over a year
    (the 15th of each month for 12) x `hours` hours spread over the day
    (hour angles -52.5..+52.5 degrees for 8), from the standard declination /
    hour-angle formulas at `latitude_deg`, elevations clamped to
    [min_elevation_deg, max_elevation_deg].  Shape (days * hours, 3), float32."""
    lat = math.radians(latitude_deg)
    out = []
    for d in range(days):
        day = 15 + round(365 * d / days)
        decl = math.radians(23.45) * math.sin(2 * math.pi * (284 + day) / 365)
        for k in range(hours):
            h = math.radians(-52.5 + 105.0 * k / max(hours - 1, 1))
            el = math.asin(math.sin(lat) * math.sin(decl) + math.cos(lat) * math.cos(decl) * math.cos(h))
            el = min(max(el, math.radians(min_elevation_deg)), math.radians(max_elevation_deg))
            az = math.atan2(-math.sin(h) * math.cos(decl),
                            math.cos(lat) * math.sin(decl) - math.sin(lat) * math.cos(decl) * math.cos(h))
            out.append(sun_direction(math.degrees(az), math.degrees(el)))
    return np.array(out, np.float32)


@dataclass
class SceneFiles:
    scene: Path
    config: Path
    tasks: Path
    num_heliostats: int


def _fmt(x: float) -> str:
    return f"{x:.6f}"


def _write(out_dir: Path, name: str, recv_lines: list[str], grid: dict, helio_block: list[str],
           positions: np.ndarray, size: tuple, config: dict) -> SceneFiles:
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    lines = ["# synthetic scene " + name, "ground\t4096.000000\t4096.000000", "ngrid\t1", ""]
    lines += recv_lines + [""]
    lines += ["Grid\t0",
              "pos\t\t" + "\t".join(_fmt(v) for v in grid["pos"]),
              "size\t" + "\t".join(_fmt(v) for v in grid["size"]),
              "inter\t" + "\t".join(_fmt(v) for v in grid["inter"]),
              f"n\t\t{len(positions)}", f"type\t{grid['helio_type']}", "end", ""]
    lines += helio_block
    for p in positions:
        lines.append("helio\t" + "\t".join(_fmt(v) for v in p))
        lines.append("\t\t" + "\t".join(_fmt(v) for v in size))
    scene = out_dir / f"{name}_scene.scn"
    scene.write_text("\n".join(lines) + "\n")
    cfg = out_dir / f"{name}_configuration.json"
    cfg.write_text(json.dumps(config, indent=2) + "\n")
    tasks = out_dir / f"{name}_heliostat_index.txt"
    tasks.write_text(f"{len(positions)}\n" + " ".join(str(i) for i in range(len(positions))) + "\n")
    return SceneFiles(scene, cfg, tasks, len(positions))


def small_field(out_dir, seed: int = 0, helio_pixel: float = 0.05, receiver_pixel: float = 0.05,
                groups: int = 128, per_group: int = 2048, rows: int = 5, cols: int = 10) -> SceneFiles:
    """The 50-heliostat flat field (optionally coarser facets / smaller lattice for tests)."""
    rng = np.random.default_rng(seed)
    pitch = 8.0
    xs = (np.arange(cols) - (cols - 1) / 2.0) * pitch
    zs = 40.0 + np.arange(rows) * pitch
    pos = []
    for z in zs:
        for x in xs:
            jx, jz = rng.uniform(-0.5, 0.5, 2)
            pos.append([x + jx, 2.5, z + jz])
    pos = np.array(pos)
    recv = ["Recv\t0", "pos\t\t0.000000\t80.000000\t0.000000", "size\t8.000000\t6.000000\t0.100000",
            "norm\t0.000000\t0.000000\t1.000000", "face\t0", "end"]
    x0 = float(np.floor(pos[:, 0].min() - 10.0))
    z0 = float(np.floor(pos[:, 2].min() - 10.0))
    grid = {"pos": [x0, 0.0, z0], "size": [float(np.ceil(pos[:, 0].max() + 10.0 - x0)), 10.0,
                                            float(np.ceil(pos[:, 2].max() + 10.0 - z0))],
            "inter": [10.0, 10.0, 10.0], "helio_type": 0}
    config = {"sun_dir": sun_direction(180.0, 60.0), "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": groups,
              "num_per_sunshape_group": per_group, "inverse_transform_sampling_groups": 1024,
              "receiver_pixel_length": receiver_pixel, "helio_disturb_std": 0.002,
              "helio_pixel_length": helio_pixel, "helio_reflected_rate": 0.88}
    return _write(out_dir, "small", recv, grid, ["gap\t0.000000\t0.000000", "matrix\t1\t1"], pos,
                  (4.0, 0.1, 4.0), config)


def radial_staggered(n: int, r_min: float, r_max: float, span_deg: float, seed: int) -> np.ndarray:
    """n (x, z) positions on staggered rings between r_min and r_max over +-span_deg
    around north, with seeded jitter."""
    rng = np.random.default_rng(seed)
    ring_step = 30.0
    radii = np.arange(r_min, r_max + 1e-6, ring_step)
    span = math.radians(2 * span_deg)
    arc_total = span * radii.sum()
    spacing = arc_total / n
    pos = []
    for k, r in enumerate(radii):
        m = max(1, int(round(span * r / spacing)))
        offset = 0.5 if k % 2 else 0.0
        for j in range(m):
            az = -math.radians(span_deg) + span * (j + 0.25 + 0.5 * offset) / m
            pos.append((r, az))
    pos = np.array(pos)
    if len(pos) > n:
        keep = np.sort(rng.choice(len(pos), n, replace=False))
        pos = pos[keep]
    while len(pos) < n:  # top up on the outermost ring
        az = rng.uniform(-math.radians(span_deg), math.radians(span_deg))
        pos = np.vstack([pos, [r_max, az]])
    r = pos[:, 0] + rng.uniform(-1.0, 1.0, n)
    az = pos[:, 1] + rng.uniform(-1.0, 1.0, n) / pos[:, 0]
    return np.stack([r * np.sin(az), r * np.cos(az)], axis=1)


def large_field(out_dir, seed: int = 0, num_heliostats: int = 624, helio_pixel: float = 0.02,
                receiver_pixel: float = 0.02, groups: int = 128, per_group: int = 2048,
                rows: int = 4, cols: int = 7, keep_every: int = 1) -> SceneFiles:
    """The 624-heliostat focus-flat field with a cylinder receiver
    (keep_every = k keeps every k-th of its heliostats: a slice of the same
    field, spread over it, with the same grid)."""
    xz = radial_staggered(num_heliostats, 100.0, 750.0, 70.0, seed)
    pos = np.stack([xz[:, 0], np.full(len(xz), 5.5), xz[:, 1]], axis=1)
    recv = ["Recv\t1", "pos\t\t0.000000\t115.000000\t0.000000", "size\t4.000000\t12.000000\t0.000000",
            "norm\t0.000000\t1.000000\t0.000000", "face\t0", "end"]
    x0 = float(np.floor(pos[:, 0].min() - 20.0))
    z0 = float(np.floor(pos[:, 2].min() - 20.0))
    grid = {"pos": [x0, 0.0, z0], "size": [float(np.ceil(pos[:, 0].max() + 20.0 - x0)), 20.0,
                                            float(np.ceil(pos[:, 2].max() + 20.0 - z0))],
            "inter": [20.0, 20.0, 20.0], "helio_type": 1}
    config = {"sun_dir": sun_direction(180.0, 60.0), "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": groups,
              "num_per_sunshape_group": per_group, "inverse_transform_sampling_groups": 1024,
              "receiver_pixel_length": receiver_pixel, "helio_disturb_std": 0.0029,
              "helio_pixel_length": helio_pixel, "helio_reflected_rate": 0.88}
    block = ["gap\t0.000000\t0.000000", f"matrix\t{rows}\t{cols}", "surface_property -1 -1 -1 -1 -1 -1"]
    return _write(out_dir, "large", recv, grid, block, pos[::keep_every], (12.84, 0.1, 9.45), config)


def uneven_field(out_dir, index: int, seed: int = 0, helio_pixel: float = 0.05, receiver_pixel: float = 0.05,
                 groups: int = 128, per_group: int = 2048) -> SceneFiles:
    """Field `index` of the batch's uneven fields (seeded by seed and index).

    Even indexes: flat square heliostats and a vertical rectangle receiver
    facing the field; odd indexes: focus-flat 2x2 heliostats (focal length =
    slant range) and a cylinder receiver.  Heliostat count uniform in
    [200, 2500], side uniform in [6, 12] m, rings from 60 m + 3 sides out to
    the radius that leaves about (3 sides)^2 of ground per heliostat over
    +-70 degrees.
    """
    rng = np.random.default_rng([seed, index, 0x5EED])
    n = int(rng.integers(200, 2501))
    side = float(rng.uniform(6.0, 12.0))
    r_min = 60.0 + 3.0 * side
    span = math.radians(140.0)
    r_max = math.sqrt(r_min ** 2 + n * (3.0 * side) ** 2 / (0.5 * span))
    xz = radial_staggered(n, r_min, r_max, 70.0, int(rng.integers(1 << 30)))
    pos = np.stack([xz[:, 0], np.full(n, 0.5 * side + 0.5), xz[:, 1]], axis=1)
    tower = 40.0 + 0.08 * r_max
    cylinder = index % 2 == 1
    if cylinder:
        r, h = float(rng.uniform(3.0, 8.0)), float(rng.uniform(8.0, 16.0))
        recv = ["Recv\t1", f"pos\t\t0.000000\t{_fmt(tower)}\t0.000000", f"size\t{_fmt(r)}\t{_fmt(h)}\t0.000000",
                "norm\t0.000000\t1.000000\t0.000000", "face\t0", "end"]
        block = ["gap\t0.000000\t0.000000", "matrix\t2\t2", "surface_property -1 -1 -1 -1 -1 -1"]
    else:
        w, h = float(rng.uniform(8.0, 14.0)), float(rng.uniform(6.0, 10.0))
        recv = ["Recv\t0", f"pos\t\t0.000000\t{_fmt(tower)}\t0.000000", f"size\t{_fmt(w)}\t{_fmt(h)}\t0.100000",
                "norm\t0.000000\t0.000000\t1.000000", "face\t0", "end"]
        block = ["gap\t0.000000\t0.000000", "matrix\t1\t1"]
    cell = float(max(10.0, round(1.6 * side)))
    margin = cell
    x0 = float(np.floor(pos[:, 0].min() - margin))
    z0 = float(np.floor(pos[:, 2].min() - margin))
    grid = {"pos": [x0, 0.0, z0], "size": [float(np.ceil(pos[:, 0].max() + margin - x0)), cell,
                                            float(np.ceil(pos[:, 2].max() + margin - z0))],
            "inter": [cell, cell, cell], "helio_type": 1 if cylinder else 0}
    config = {"sun_dir": sun_direction(float(rng.uniform(120.0, 240.0)), float(rng.uniform(25.0, 75.0))),
              "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": groups, "num_per_sunshape_group": per_group,
              "inverse_transform_sampling_groups": 1024, "receiver_pixel_length": receiver_pixel,
              "helio_disturb_std": 0.002, "helio_pixel_length": helio_pixel, "helio_reflected_rate": 0.88}
    return _write(out_dir, f"uneven{index:02d}", recv, grid, block, pos, (side, 0.1, side), config)


def huge_field(out_dir, seed: int = 0, num_heliostats: int = 10_000, helio_pixel: float = 0.05,
               receiver_pixel: float = 0.05, groups: int = 128, per_group: int = 2048) -> SceneFiles:
    """The large batched-adjoint field: flat 10x10 m heliostats, cylinder receiver."""
    xz = radial_staggered(num_heliostats, 150.0, 1800.0, 70.0, seed)
    pos = np.stack([xz[:, 0], np.full(len(xz), 5.5), xz[:, 1]], axis=1)
    recv = ["Recv\t1", "pos\t\t0.000000\t200.000000\t0.000000", "size\t10.000000\t20.000000\t0.000000",
            "norm\t0.000000\t1.000000\t0.000000", "face\t0", "end"]
    x0 = float(np.floor(pos[:, 0].min() - 20.0))
    z0 = float(np.floor(pos[:, 2].min() - 20.0))
    grid = {"pos": [x0, 0.0, z0], "size": [float(np.ceil(pos[:, 0].max() + 20.0 - x0)), 20.0,
                                            float(np.ceil(pos[:, 2].max() + 20.0 - z0))],
            "inter": [20.0, 20.0, 20.0], "helio_type": 0}
    config = {"sun_dir": sun_direction(180.0, 60.0), "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": groups,
              "num_per_sunshape_group": per_group, "inverse_transform_sampling_groups": 1024,
              "receiver_pixel_length": receiver_pixel, "helio_disturb_std": 0.002,
              "helio_pixel_length": helio_pixel, "helio_reflected_rate": 0.88}
    return _write(out_dir, "huge", recv, grid, ["gap\t0.000000\t0.000000", "matrix\t1\t1"], pos,
                  (10.0, 0.1, 10.0), config)


def two_receiver_field(out_dir, seed: int = 0, helio_pixel: float = 0.25, receiver_pixel: float = 0.05,
                       groups: int = 4, per_group: int = 128) -> SceneFiles:
    """Two receivers, one grid each: 12 flat 5x5 m heliostats north of a
    rectangle receiver at (0, 40, 0) facing north, 12 focus-flat 6x4 m (2x2)
    heliostats south of a cylinder receiver (r 2 m, h 4 m) at (0, 40, -200)."""
    out_dir = Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    lines = ["# synthetic scene two receivers", "ground\t1024.000000\t1024.000000", "ngrid\t2", ""]
    north = [[(c - 1.5) * 10.0 + rng.uniform(-0.5, 0.5), 3.0, 40.0 + r * 10.0 + rng.uniform(-0.5, 0.5)]
             for r in range(3) for c in range(4)]
    south = [[(c - 1.5) * 10.0 + rng.uniform(-0.5, 0.5), 3.0, -240.0 - r * 10.0 + rng.uniform(-0.5, 0.5)]
             for r in range(3) for c in range(4)]
    blocks = [
        (["Recv\t0", "pos\t\t0.000000\t40.000000\t0.000000", "size\t6.000000\t5.000000\t0.100000",
          "norm\t0.000000\t0.000000\t1.000000", "face\t0", "end"],
         0, ["gap\t0.000000\t0.000000", "matrix\t1\t1"], north, (5.0, 0.1, 5.0)),
        (["Recv\t1", "pos\t\t0.000000\t40.000000\t-200.000000", "size\t2.000000\t4.000000\t0.000000",
          "norm\t0.000000\t1.000000\t0.000000", "face\t0", "end"],
         1, ["gap\t0.000000\t0.000000", "matrix\t2\t2", "surface_property -1 -1 -1 -1 -1 -1"], south,
         (6.0, 0.1, 4.0)),
    ]
    n_total = 0
    for recv, htype, block, pos, size in blocks:
        pos = np.array(pos)
        lines += recv + [""]
        x0 = float(np.floor(pos[:, 0].min() - 10.0))
        z0 = float(np.floor(pos[:, 2].min() - 10.0))
        sx = float(np.ceil(pos[:, 0].max() + 10.0 - x0))
        sz = float(np.ceil(pos[:, 2].max() + 10.0 - z0))
        lines += ["Grid\t0", f"pos\t\t{_fmt(x0)}\t0.000000\t{_fmt(z0)}", f"size\t{_fmt(sx)}\t10.000000\t{_fmt(sz)}",
                  "inter\t10.000000\t10.000000\t10.000000", f"n\t\t{len(pos)}", f"type\t{htype}", "end", ""]
        lines += block
        for p in pos:
            lines.append("helio\t" + "\t".join(_fmt(v) for v in p))
            lines.append("\t\t" + "\t".join(_fmt(v) for v in size))
        lines.append("")
        n_total += len(pos)
    scene = out_dir / "two_scene.scn"
    scene.write_text("\n".join(lines) + "\n")
    config = {"sun_dir": sun_direction(150.0, 50.0), "dni": 1000.0, "csr": 0.1, "num_of_sunshape_groups": groups,
              "num_per_sunshape_group": per_group, "inverse_transform_sampling_groups": 1024,
              "receiver_pixel_length": receiver_pixel, "helio_disturb_std": 0.002,
              "helio_pixel_length": helio_pixel, "helio_reflected_rate": 0.88}
    cfg = out_dir / "two_configuration.json"
    cfg.write_text(json.dumps(config, indent=2) + "\n")
    tasks = out_dir / "two_heliostat_index.txt"
    tasks.write_text(f"{n_total}\n" + " ".join(str(i) for i in range(n_total)) + "\n")
    return SceneFiles(scene, cfg, tasks, n_total)
