"""Seeded synthetic scenes and cameras for the benchmark configurations.

The reference measured on laser scans that are not part of it; these seeded
scenes stand in for them with the shapes and sizes the benchmark
configurations name:

* ``menger``    -- Menger sponge level 5 (243^3 cells) in a depth-8 octree
                   (256^3), one treelet, colour = hash(x, y, z); 512x512 view
                   from a seeded camera outside the cube, 60 degree fov.
* ``icosphere`` -- icosphere subdivided 6 times (81,920 triangles), radius
                   0.4 displaced radially by 3-octave value noise of amplitude
                   0.05, depth-11 octree cut into 6-level treelets, leaf colour
                   from the face normal (colour = normal * 0.5 + 0.5 of the
                   normalised sum of the overlapping faces' normals, as the
                   configuration asks; ``colour="vertex"`` interpolates seeded
                   per-vertex attributes as the reference's attribute
                   generator does instead); one 1920x1080 view from an orbit of
                   radius 2.5.  The configuration names no field of view; 25
                   degrees (vertical) makes the sphere fill the frame height, so
                   most rays enter the octree.
* ``terrain``   -- 1024 x 1024 height-field grid (2,093,058 triangles), heights
                   from 6-octave fBm in [-0.45, -0.15] (0.3 of the extent),
                   depth-12 octree cut into 6-level treelets; 64 square views
                   with sides drawn log-uniformly from 256 to 2048 pixels,
                   eyes above the terrain looking at seeded points on it,
                   60 degree fov.
* ``large_shadowed`` -- icosphere subdivided 9 times (5,242,880 triangles),
                   4-octave noise, depth-14 octree (16384^3) cut into 8-level
                   treelets, built on the GPU (DeviceScene, about 40 GB of
                   pool); one 3840x2160 view from the icosphere orbit, primary
                   rays plus one shadow ray per hit toward a seeded
                   directional light, stack size 15 (depth 14 + 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import (Camera, DeviceScene, Scene, icosphere as icosphere_mesh, orbit_camera, seeded_light,
               terrain as terrain_mesh, vertex_attributes)


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
              fov_deg=25.0, radius=2.5, colour="face") -> Workload:
    v, t = icosphere_mesh(subdivisions, radius=0.4, octaves=3, amplitude=0.05, frequency=2.0, seed=seed)
    if colour == "face":
        scene = Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels)
    else:
        n, c = vertex_attributes(v, t, seed)
        scene = Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels, normals=n, colors=c)
    rng = np.random.default_rng(seed)
    cam = orbit_pose(radius, float(rng.uniform(0, 360)), float(rng.uniform(-30, 30)), width, height,
                     fov_deg)
    return Workload(f"icosphere_s{subdivisions}_d{depth}_{width}x{height}", scene, [cam],
                    description=f"icosphere {subdivisions}x subdivided ({t.shape[0]} triangles), 3-octave "
                                f"noise 0.05, depth {depth}, {treelet_levels}-level treelets, colour from the "
                                f"{'face normal' if colour == 'face' else 'vertex attributes'}, {width}x{height}, "
                                f"orbit radius {radius}, fov {fov_deg}")


def terrain(grid=1024, depth=12, treelet_levels=6, seed=1, views=64, min_side=256, max_side=2048,
            fov_deg=60.0) -> Workload:
    v, t = terrain_mesh(grid, octaves=6, base=-0.45, height=0.3, frequency=2.0, seed=seed)
    n, c = vertex_attributes(v, t, seed)
    scene = Scene.from_mesh(v, t, depth, treelet_levels=treelet_levels, normals=n, colors=c)
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


@dataclass
class LargeShadowedWorkload:
    name: str
    scene: DeviceScene
    camera: Camera
    light: np.ndarray
    stack_size: int
    description: str = ""


def large_shadowed(subdivisions=9, depth=14, treelet_levels=8, seed=1, width=3840, height=2160,
                   fov_deg=25.0, radius=2.5, stream=None) -> LargeShadowedWorkload:
    v, t = icosphere_mesh(subdivisions, radius=0.4, octaves=4, amplitude=0.05, frequency=2.0, seed=seed)
    n, c = vertex_attributes(v, t, seed)
    scene = DeviceScene(v, t, depth, treelet_levels=treelet_levels, stream=stream, normals=n, colors=c)
    rng = np.random.default_rng(seed)
    cam = orbit_pose(radius, float(rng.uniform(0, 360)), float(rng.uniform(-30, 30)), width, height, fov_deg)
    return LargeShadowedWorkload(
        f"icosphere_s{subdivisions}_d{depth}_{width}x{height}_shadow", scene, cam, seeded_light(seed),
        depth + 1,
        description=f"icosphere {subdivisions}x subdivided ({t.shape[0]} triangles), 4-octave noise 0.05, "
                    f"depth {depth}, {treelet_levels}-level treelets built on the GPU, {width}x{height} "
                    f"primary rays + 1 shadow ray per hit toward a seeded directional light, "
                    f"orbit radius {radius}, fov {fov_deg}")


@dataclass
class ServingWorkload:
    name: str
    scenes: list          # Scene per octree
    stack_sizes: list
    description: str = ""


# (kind, size, depth, treelet levels, seed, radius): displaced icospheres and
# fBm terrains of depths 9..13.  The depth-13 octree is a smaller sphere
# (radius 0.15) so that its host build stays in seconds.
SERVING_OCTREES = [
    ("icosphere", 5, 9, 4, 11, 0.4), ("terrain", 257, 9, 4, 12, None),
    ("icosphere", 5, 10, 5, 13, 0.4), ("terrain", 513, 10, 5, 14, None),
    ("icosphere", 6, 11, 6, 15, 0.4), ("terrain", 1024, 11, 6, 16, None),
    ("icosphere", 6, 12, 6, 17, 0.3), ("icosphere", 6, 13, 6, 18, 0.15),
]


def serving(octrees=SERVING_OCTREES) -> ServingWorkload:
    scenes = []
    for kind, size, depth, levels, seed, radius in octrees:
        if kind == "icosphere":
            v, t = icosphere_mesh(size, radius=radius, octaves=3, amplitude=0.05 * radius / 0.4,
                                  frequency=2.0, seed=seed)
        else:
            v, t = terrain_mesh(size, octaves=6, base=-0.45, height=0.3, frequency=2.0, seed=seed)
        n, c = vertex_attributes(v, t, seed)
        scenes.append(Scene.from_mesh(v, t, depth, treelet_levels=levels, normals=n, colors=c))
    depths = [o[2] for o in octrees]
    return ServingWorkload("serving_8_octrees", scenes, [13] * len(scenes),
                           description=f"{len(scenes)} octrees (icospheres and terrains, depths "
                                       f"{min(depths)}..{max(depths)}), requests 64x64..1920x1080 "
                                       f"log-uniform, Poisson arrivals")


def serving_requests(n, num_octrees, seed=0, min_wh=(64, 64), max_wh=(1920, 1080)):
    """Seeded request mix: (octree, Camera) pairs; each axis of the resolution
    interpolates log-linearly between 64x64 and 1920x1080 with one uniform
    draw, cameras on an orbit around the octree."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        o = int(rng.integers(0, num_octrees))
        u = rng.uniform()
        w = int(round(min_wh[0] * (max_wh[0] / min_wh[0]) ** u))
        h = int(round(min_wh[1] * (max_wh[1] / min_wh[1]) ** u))
        cam = orbit_pose(float(rng.uniform(1.2, 2.5)), float(rng.uniform(0, 360)),
                         float(rng.uniform(-40, 40)), w, h, fov_deg=float(rng.uniform(25, 60)))
        out.append((o, cam))
    return out


def poisson_arrivals(n, rate_per_s, seed=0):
    rng = np.random.default_rng(seed + 7)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))
