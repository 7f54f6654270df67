"""Seeded synthetic scenes and cameras for the benchmark configurations.

The reference measured on laser scans that are not part of it; these seeded
scenes stand in for them with the shapes and sizes the benchmark
configurations name:

* ``menger``    -- Menger sponge level 5 (243^3 cells) in a depth-8 octree
                   (256^3), one treelet, colour = hash(x, y, z); 512x512 view
                   from a seeded camera outside the cube, 60 degree fov.
* ``icosphere`` -- icosphere subdivided 6 times (81,920 triangles), radius
                   0.4 displaced radially by 3-octave value noise of amplitude
                   0.05, depth-11 octree cut into 6-level treelets, colour from
                   the face normal; one 1920x1080 view from an orbit of radius
                   2.5.  The configuration names no field of view; 25 degrees
                   (vertical) makes the sphere fill the frame height, so most
                   rays enter the octree.
* ``terrain``   -- 1024 x 1024 height-field grid (2,093,058 triangles), heights
                   from 6-octave fBm in [-0.45, -0.15] (0.3 of the extent),
                   depth-12 octree cut into 6-level treelets; 64 square views
                   with sides drawn log-uniformly from 256 to 2048 pixels,
                   eyes above the terrain looking at seeded points on it,
                   60 degree fov.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import Camera, Scene, icosphere as icosphere_mesh, orbit_camera, terrain as terrain_mesh


@dataclass
class Workload:
    name: str
    scene: Scene
    cameras: list
    stack_size: int = 13
    description: str = ""

    @property
    def rays_per_step(self) -> int:
        return sum(c.width * c.height for c in self.cameras)


def menger(level=5, depth=8, seed=1, width=512, height=512) -> Workload:
    scene = Scene.menger(level=level, depth=depth, seed=seed)
    cam = orbit_camera(seed, width, height, radius=(1.5, 2.5), fov_deg=60.0)
    return Workload("menger_l5_d8_512", scene, [cam],
                    description=f"Menger level {level}, depth {depth}, one treelet, {width}x{height}")


def orbit_pose(radius: float, angle_deg: float, elevation_deg: float, width: int, height: int,
               fov_deg=60.0) -> Camera:
    a, e = math.radians(angle_deg), math.radians(elevation_deg)
    eye = (radius * math.cos(e) * math.cos(a), radius * math.sin(e), radius * math.cos(e) * math.sin(a))
    return Camera(eye, (0.0, 0.0, 0.0), width, height, fov_deg)


def icosphere(subdivisions=6, depth=11, treelet_levels=6, seed=1, width=1920, height=1080,
              fov_deg=25.0, radius=2.5) -> Workload:
    v, t = icosphere_mesh(subdivisions, radius=0.4, octaves=3, amplitude=0.05, frequency=2.0, seed=seed)
    scene = Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels)
    rng = np.random.default_rng(seed)
    cam = orbit_pose(radius, float(rng.uniform(0, 360)), float(rng.uniform(-30, 30)), width, height,
                     fov_deg)
    return Workload(f"icosphere_s{subdivisions}_d{depth}_{width}x{height}", scene, [cam],
                    description=f"icosphere {subdivisions}x subdivided ({t.shape[0]} triangles), 3-octave "
                                f"noise 0.05, depth {depth}, {treelet_levels}-level treelets, {width}x{height}, "
                                f"orbit radius {radius}, fov {fov_deg}")


def terrain(grid=1024, depth=12, treelet_levels=6, seed=1, views=64, min_side=256, max_side=2048,
            fov_deg=60.0) -> Workload:
    v, t = terrain_mesh(grid, octaves=6, base=-0.45, height=0.3, frequency=2.0, seed=seed)
    scene = Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels)
    rng = np.random.default_rng(seed + 1000)
    cams = []
    for _ in range(views):
        side = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        eye = (rng.uniform(-0.45, 0.45), rng.uniform(-0.05, 0.35), rng.uniform(-0.45, 0.45))
        target = (rng.uniform(-0.35, 0.35), -0.3, rng.uniform(-0.35, 0.35))
        up = (0.0, 1.0, 0.0)
        cams.append(Camera(eye, target, side, side, fov_deg, up))
    return Workload(f"terrain_g{grid}_d{depth}_{views}views", scene, cams,
                    description=f"terrain {grid}x{grid} grid ({t.shape[0]} triangles), 6-octave fBm, "
                                f"depth {depth}, {treelet_levels}-level treelets, {views} views "
                                f"{min_side}^2..{max_side}^2 log-uniform, fov {fov_deg}")
