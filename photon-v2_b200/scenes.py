"""Seeded procedural scenes for the BNEEPT/BVPT workloads, written out as Photon SDL (.p2) text.

Every workload this library is measured on is generated here, in code, from a seed:

* ``cornell``      -- Cornell box: 5 wall quads of a 555-unit box, two rotated boxes, one ceiling
                      quad light of radiance (17, 12, 4); Lambertian albedos 0.73 / (0.65, 0.05,
                      0.05) / (0.12, 0.45, 0.15); pinhole camera, 40 degree FOV.
* ``ggx_sphere``   -- icosphere subdivided ``level`` times (20 * 4**level triangles), radially
                      displaced by 3-octave value noise (amplitude 5 % of the radius) on a 2-triangle
                      ground; GGX conductors in 64 material groups with roughness ~ U[0.05, 0.5]
                      and F0 ~ U[0.5, 1]; 2 quad lights and a constant environment of 0.1.
* ``slit_room``    -- 10 x 10 x 4 room filled with seeded boxes, lit only by a 1 x 1 quad behind a
                      wall with a 0.05-wide slit; 70 % Lambertian / 30 % GGX dielectric groups.
* ``city``         -- grid city of boxes with lognormal heights and many small emissive quads.

The scene is described once (triangles, materials, emitters, camera) and serialised to SDL in
the form the reference parser reads (``#version 1.1.0`` command syntax, see the reference's
Engine/Source/SDL/SdlCommandParser.cpp:84-560 and SdlInlinePacketInterface.cpp:48-200), so the
same text drives the reference CPU renderer and this library's ``phLoadCommands``/
``phEnterCommand``.  All geometry is emitted in world space with identity actor transforms:
the reference then intersects plain ``PTriangle`` primitives (Engine/Source/Actor/AModel.cpp:
43-81 only wraps them in a transformed intersectable when the actor has a transform).
"""

from __future__ import annotations

import dataclasses
import os
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

RGB = Tuple[float, float, float]


@dataclasses.dataclass
class Material:
    """One surface material.

    kind: "matte" (Lambertian, ``albedo``), "conductor" (GGX + Schlick, ``roughness``, ``f0``)
    or "dielectric" (GGX + exact dielectric Fresnel, ``roughness``, ``ior_outer``,
    ``ior_inner``).
    """

    kind: str
    albedo: RGB = (0.5, 0.5, 0.5)
    roughness: float = 0.5
    f0: RGB = (1.0, 1.0, 1.0)
    ior_outer: float = 1.0
    ior_inner: float = 1.5


@dataclasses.dataclass
class MeshGroup:
    """Triangles sharing one material; ``radiance`` set means the group is an area emitter."""

    tris: np.ndarray  # float32 [N, 3, 3]
    material: Material
    radiance: Optional[RGB] = None


@dataclasses.dataclass
class Scene:
    name: str
    width: int
    height: int
    spp: int
    max_bounces: int
    cam_pos: RGB
    cam_dir: RGB
    cam_up: RGB
    fov_deg: float
    groups: List[MeshGroup]
    estimator: str = "bneept"
    env_radiance: Optional[RGB] = None
    sample_filter: str = "box"      # box | gaussian | mn | bh (the reference's sample-filter enum)
    # lat-long dome image [H, W, 3] (row 0 = top), used instead of env_radiance when set, and the
    # dome's rotation (axis, degrees)
    env_image: Optional[np.ndarray] = None
    env_rotation: Optional[Tuple[RGB, float]] = None

    @property
    def has_env(self) -> bool:
        return self.env_radiance is not None or self.env_image is not None

    @property
    def num_tris(self) -> int:
        return int(sum(g.tris.shape[0] for g in self.groups))

    @property
    def num_paths(self) -> int:
        return self.width * self.height * self.spp


# ----------------------------------------------------------------------------------------------
# geometry helpers

def quad(a, b, c, d) -> np.ndarray:
    """Two triangles (a, b, c) and (a, c, d); the face normal follows (b - a) x (c - a)."""
    a, b, c, d = (np.asarray(v, np.float64) for v in (a, b, c, d))
    return np.array([[a, b, c], [a, c, d]], np.float32)


def box(center, size, yaw_deg: float = 0.0) -> np.ndarray:
    """12 outward-facing triangles of a box rotated about +y by ``yaw_deg``."""
    cx, cy, cz = center
    sx, sy, sz = (s * 0.5 for s in size)
    c, s = math.cos(math.radians(yaw_deg)), math.sin(math.radians(yaw_deg))

    def p(x, y, z):
        return (cx + c * x + s * z, cy + y, cz - s * x + c * z)

    v = [p(x, y, z) for x in (-sx, sx) for y in (-sy, sy) for z in (-sz, sz)]
    # v index = 4*ix + 2*iy + iz
    faces = [
        (0, 1, 3, 2),  # -x
        (4, 6, 7, 5),  # +x
        (0, 4, 5, 1),  # -y
        (2, 3, 7, 6),  # +y
        (0, 2, 6, 4),  # -z
        (1, 5, 7, 3),  # +z
    ]
    return np.concatenate([quad(v[f[0]], v[f[1]], v[f[2]], v[f[3]]) for f in faces])


def boxes_axis_aligned(mins: np.ndarray, maxs: np.ndarray) -> np.ndarray:
    """Vectorised outward-facing 12-triangle boxes for arrays of corners [K, 3] -> [12K, 3, 3]."""
    k = mins.shape[0]
    corners = np.empty((k, 8, 3), np.float64)
    for ix in range(2):
        for iy in range(2):
            for iz in range(2):
                corners[:, 4 * ix + 2 * iy + iz] = np.stack(
                    [(mins, maxs)[ix][:, 0], (mins, maxs)[iy][:, 1], (mins, maxs)[iz][:, 2]], 1)
    faces = np.array([(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1),
                      (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)])
    tri_idx = np.concatenate([faces[:, [0, 1, 2]], faces[:, [0, 2, 3]]], 0)  # [12, 3]
    tris = corners[:, tri_idx]  # [K, 12, 3, 3]
    return tris.reshape(-1, 3, 3).astype(np.float32)


def icosphere(level: int) -> np.ndarray:
    """Unit icosphere subdivided ``level`` times: [20 * 4**level, 3, 3] float64 outward-wound."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
                      (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                      (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
                      (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
                      (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
                      (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)])
    tris = verts[faces]
    for _ in range(level):
        a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        tris = np.stack([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1),
                         np.stack([ca, bc, c], 1), np.stack([ab, bc, ca], 1)], 1).reshape(-1, 3, 3)
    # make winding outward
    n = np.cross(tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0])
    flip = np.einsum("ij,ij->i", n, tris.mean(1)) < 0
    tris[flip] = tris[flip][:, [0, 2, 1]]
    return tris


def value_noise3(p: np.ndarray, seed: int, octaves: int = 3) -> np.ndarray:
    """Seeded 3-octave trilinear value noise in [-1, 1] at points p [N, 3]."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-1.0, 1.0, 4096)
    perm = rng.permutation(4096)
    total = np.zeros(p.shape[0])
    amp, freq, norm = 1.0, 2.0, 0.0
    for _ in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        f = f * f * (3 - 2 * f)
        acc = np.zeros(p.shape[0])
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    h = perm[(perm[(perm[(i0[:, 0] + dx) & 4095] + i0[:, 1] + dy) & 4095]
                              + i0[:, 2] + dz) & 4095]
                    w = ((f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1])
                         * (f[:, 2] if dz else 1 - f[:, 2]))
                    acc += w * table[h]
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


# ----------------------------------------------------------------------------------------------
# workloads

WHITE = Material("matte", albedo=(0.73, 0.73, 0.73))
RED = Material("matte", albedo=(0.65, 0.05, 0.05))
GREEN = Material("matte", albedo=(0.12, 0.45, 0.15))
BLACK = Material("matte", albedo=(0.0, 0.0, 0.0))


def cornell(width: int = 256, height: int = 256, spp: int = 64, max_bounces: int = 8,
            estimator: str = "bneept") -> Scene:
    """Cornell box (36 triangles) in a 555-unit box, camera looking down +z."""
    L = 555.0
    floor = quad((0, 0, 0), (0, 0, L), (L, 0, L), (L, 0, 0))            # normal +y
    ceiling = quad((0, L, 0), (L, L, 0), (L, L, L), (0, L, L))          # normal -y
    back = quad((0, 0, L), (0, L, L), (L, L, L), (L, 0, L))             # normal -z
    left = quad((L, 0, 0), (L, 0, L), (L, L, L), (L, L, 0))             # x = L, normal -x (red)
    right = quad((0, 0, 0), (0, L, 0), (0, L, L), (0, 0, L))            # x = 0, normal +x (green)
    short_box = box((185.5, 82.5, 169.0), (165.0, 165.0, 165.0), -18.0)
    tall_box = box((368.5, 165.0, 351.5), (165.0, 330.0, 165.0), 15.0)
    light = quad((213, 554, 227), (343, 554, 227), (343, 554, 332), (213, 554, 332))  # normal -y
    groups = [
        MeshGroup(np.concatenate([floor, ceiling, back]), WHITE),
        MeshGroup(left, RED),
        MeshGroup(right, GREEN),
        MeshGroup(np.concatenate([short_box, tall_box]), WHITE),
        MeshGroup(light, BLACK, radiance=(17.0, 12.0, 4.0)),
    ]
    return Scene("cornell", width, height, spp, max_bounces,
                 cam_pos=(278.0, 273.0, -800.0), cam_dir=(0.0, 0.0, 1.0), cam_up=(0.0, 1.0, 0.0),
                 fov_deg=40.0, groups=groups, estimator=estimator)


def cornell_glossy(width: int = 64, height: int = 64, spp: int = 64, max_bounces: int = 8,
                   estimator: str = "bneept") -> Scene:
    """Cornell box whose tall box is a rough GGX dielectric (IOR 1.5, roughness 0.1) and whose
    short box is a GGX conductor (roughness 0.3, gold-like F0): exercises every BSDF.

    The glass box floats one unit above the floor. Resting on it, its bottom face would be
    coplanar with the floor, and a ray leaving the glass downwards would hit both at (nearly) the
    same t: which one the reference reports depends on its BVH traversal order and last-ulp
    rounding, and the two answers (refract out of the glass vs. a diffuse bounce) carry different
    energy, so such a scene has no well-defined expected image."""
    sc = cornell(width, height, spp, max_bounces, estimator)
    L = 555.0
    floor = quad((0, 0, 0), (0, 0, L), (L, 0, L), (L, 0, 0))
    ceiling = quad((0, L, 0), (L, L, 0), (L, L, L), (0, L, L))
    back = quad((0, 0, L), (0, L, L), (L, L, L), (L, 0, L))
    short_box = box((185.5, 82.5, 169.0), (165.0, 165.0, 165.0), -18.0)
    tall_box = box((368.5, 166.0, 351.5), (165.0, 330.0, 165.0), 15.0)
    sc.groups[0] = MeshGroup(np.concatenate([floor, ceiling, back]), WHITE)
    sc.groups[3] = MeshGroup(short_box, Material("conductor", roughness=0.3, f0=(1.0, 0.77, 0.34)))
    sc.groups.insert(4, MeshGroup(tall_box, Material("dielectric", roughness=0.1, ior_outer=1.0, ior_inner=1.5)))
    sc.name = "cornell_glossy"
    return sc


def tessellated_boxes(mins: np.ndarray, maxs: np.ndarray, grid: int = 3) -> np.ndarray:
    """Outward-facing boxes whose 6 faces are each split into grid x grid quads:
    [K, 6 * grid^2 * 2, 3, 3] float32 (108 triangles per box at grid 3)."""
    k = mins.shape[0]
    u = np.linspace(0.0, 1.0, grid + 1)
    tris = []
    # each face: origin corner (in unit-box coordinates), two edge axes, sign for outward winding
    faces = [((0, 0, 0), 2, 1), ((1, 0, 0), 1, 2),   # -x, +x
             ((0, 0, 0), 0, 2), ((0, 1, 0), 2, 0),   # -y, +y
             ((0, 0, 0), 1, 0), ((0, 0, 1), 0, 1)]   # -z, +z
    ext = maxs - mins
    for origin, ea, eb in faces:
        for i in range(grid):
            for j in range(grid):
                def corner(a, b):
                    c = np.array(origin, np.float64)
                    c = np.broadcast_to(c, (k, 3)).copy()
                    c[:, ea] = a
                    c[:, eb] = b
                    return mins + c * ext
                p00, p10 = corner(u[i], u[j]), corner(u[i + 1], u[j])
                p11, p01 = corner(u[i + 1], u[j + 1]), corner(u[i], u[j + 1])
                tris.append(np.stack([p00, p10, p11], 1))
                tris.append(np.stack([p00, p11, p01], 1))
    return np.stack(tris, 1).astype(np.float32)


def city(width: int = 1920, height: int = 1080, spp: int = 1024, max_bounces: int = 12,
         blocks: int = 447, num_lights: int = 10_000, num_materials: int = 64, seed: int = 5,
         estimator: str = "bneept") -> Scene:
    """Many-light night city: a blocks x blocks grid of buildings (447^2 = 199,809) whose heights
    are lognormal(mu 2, sigma 0.6), each a box with 3 x 3-tessellated faces (108 triangles, so
    ~21.6M triangles), on a ground plane; GGX conductors with roughness ~ U[0.02, 0.8] in
    `num_materials` groups; lit only by `num_lights` small emissive quads whose radiance is
    lognormal (sigma 1), picked by the power alias table."""
    rng = np.random.default_rng(seed)
    lot = 12.0
    gx, gz = np.meshgrid(np.arange(blocks), np.arange(blocks), indexing="ij")
    gx, gz = gx.ravel(), gz.ravel()
    k = gx.size
    fw = rng.uniform(4.0, 9.0, (k, 2))
    off = rng.uniform(0.0, 1.0, (k, 2)) * (lot - 1.0 - fw)
    building_h = np.exp(rng.normal(2.0, 0.6, k))
    mins = np.stack([gx * lot + 0.5 + off[:, 0], np.zeros(k), gz * lot + 0.5 + off[:, 1]], 1)
    maxs = np.stack([mins[:, 0] + fw[:, 0], building_h, mins[:, 2] + fw[:, 1]], 1)
    boxes = tessellated_boxes(mins, maxs, 3)
    size = blocks * lot
    ground = quad((0, 0, 0), (0, 0, size), (size, 0, size), (size, 0, 0))
    group = rng.integers(0, num_materials, k)
    groups = [MeshGroup(ground, Material("matte", albedo=(0.3, 0.3, 0.3)))]
    for m in range(num_materials):
        sel = boxes[group == m].reshape(-1, 3, 3)
        if sel.shape[0]:
            groups.append(MeshGroup(sel, Material("conductor", roughness=float(rng.uniform(0.02, 0.8)),
                                                  f0=tuple(float(x) for x in rng.uniform(0.5, 1.0, 3)))))
    # street lights: 1 x 1 quads facing down, 6 m above the street between lots
    lx = (rng.integers(0, blocks, num_lights) + rng.uniform(0.0, 1.0, num_lights)) * lot
    lz = rng.integers(0, blocks, num_lights) * lot + 0.25
    radiance = np.exp(rng.normal(0.0, 1.0, num_lights)) * 400.0
    tint = rng.uniform(0.7, 1.0, (num_lights, 3))
    for i in range(num_lights):
        x, z = float(lx[i]), float(lz[i])
        q = quad((x, 6.0, z), (x + 1.0, 6.0, z), (x + 1.0, 6.0, z + 1.0), (x, 6.0, z + 1.0))  # normal -y
        groups.append(MeshGroup(q, BLACK, radiance=tuple(float(radiance[i] * t) for t in tint[i])))
    centre = size * 0.5
    return Scene("city", width, height, spp, max_bounces, cam_pos=(centre - 60.0, 25.0, centre - 60.0),
                 cam_dir=(0.7, -0.25, 0.7), cam_up=(0.0, 1.0, 0.0), fov_deg=60.0, groups=groups,
                 estimator=estimator)


def slit_room(width: int = 1024, height: int = 1024, spp: int = 64, max_bounces: int = 10,
              num_boxes: int = 166_667, seed: int = 3, estimator: str = "bneept",
              glass_fraction: float = 0.3) -> Scene:
    """Learned-guiding workload: a 10 x 10 x 4 room filled with seeded random furniture boxes
    (12 triangles each; 166,667 boxes = 2M triangles), lit only by a 1 x 1 quad light behind a
    dividing wall that has a single 0.05-wide vertical slit. 70 % of the boxes are Lambertian,
    30 % rough GGX glass (IOR 1.5, roughness 0.1). Almost all light enters the room through the
    slit, so BSDF sampling rarely finds it: the case path guiding is for. glass_fraction 0 makes
    every box Lambertian (the same boxes: the random draws do not change)."""
    rng = np.random.default_rng(seed)
    # room shell, faces pointing inwards
    shell = boxes_axis_aligned(np.array([[0.0, 0.0, 0.0]]), np.array([[10.0, 4.0, 10.0]]))[:, [0, 2, 1]]
    # dividing wall at x = 8 (0.1 thick) with a slit z in [4.975, 5.025], full height
    wall = boxes_axis_aligned(np.array([[7.95, 0.0, 0.0], [7.95, 0.0, 5.025]]),
                              np.array([[8.05, 4.0, 4.975], [8.05, 4.0, 10.0]]))
    # the light: 1 x 1 quad at x = 9.5 facing -x, towards the slit
    light = quad((9.5, 1.5, 4.5), (9.5, 1.5, 5.5), (9.5, 2.5, 5.5), (9.5, 2.5, 4.5))
    # furniture in the main part of the room (x < 7.9), standing on the floor or floating
    # box sizes shrink with the count so that the filled volume stays ~2 % of the room; the corner
    # around the camera is kept clear
    k = int(num_boxes)
    largest = float(np.clip(0.25 * (2000.0 / max(k, 1)) ** (1.0 / 3.0), 0.04, 0.25))
    size = rng.uniform(0.08 * largest, largest, (k, 3)) * np.array([1.0, 1.6, 1.0])
    # boxes "on the floor" stand 1 mm above it: a box bottom in the floor's plane would make the
    # closest hit of a ray inside a glass box an arbitrary pick between two coplanar triangles
    lo = np.stack([rng.uniform(0.1, 7.8, k), np.where(rng.random(k) < 0.6, 1e-3, rng.uniform(0.0, 3.5, k)),
                   rng.uniform(0.1, 9.9, k)], 1)
    near_camera = (lo[:, 0] < 1.6) & (lo[:, 2] < 1.6)
    lo[near_camera, 0] += 1.6
    hi = np.minimum(lo + size, np.array([7.9, 3.95, 9.95]))
    boxes = boxes_axis_aligned(lo, hi).reshape(k, 12, 3, 3)
    glass = rng.random(k) < glass_fraction
    groups = [
        MeshGroup(np.concatenate([shell, wall]).astype(np.float32), Material("matte", albedo=(0.7, 0.7, 0.7))),
        MeshGroup(boxes[~glass].reshape(-1, 3, 3), Material("matte", albedo=(0.6, 0.55, 0.5))),
        MeshGroup(boxes[glass].reshape(-1, 3, 3), Material("dielectric", roughness=0.1, ior_outer=1.0, ior_inner=1.5)),
        MeshGroup(light.astype(np.float32), BLACK, radiance=(400.0, 400.0, 400.0)),
    ]
    groups = [g for g in groups if g.tris.shape[0] > 0]
    return Scene("slit_room", width, height, spp, max_bounces, cam_pos=(0.6, 2.2, 0.6),
                 cam_dir=(0.55, -0.15, 0.8), cam_up=(0.0, 1.0, 0.0), fov_deg=70.0, groups=groups,
                 estimator=estimator)


def ggx_sphere(level: int = 8, width: int = 1024, height: int = 1024, spp: int = 256,
               max_bounces: int = 10, num_groups: int = 64, seed: int = 1,
               with_env: bool = True, estimator: str = "bneept") -> Scene:
    """Displaced GGX icosphere (20 * 4**level triangles) on a ground plane, 2 quad lights."""
    R = 1.0
    tris = icosphere(level)
    flat = tris.reshape(-1, 3)
    disp = 1.0 + 0.05 * value_noise3(flat, seed)
    flat = flat * (R * disp)[:, None]
    tris = flat.reshape(-1, 3, 3)
    tris[:, :, 1] += R * 1.05  # sit on the ground
    rng = np.random.default_rng(2)
    rough = rng.uniform(0.05, 0.5, num_groups)
    f0 = rng.uniform(0.5, 1.0, (num_groups, 3))
    gid = np.arange(tris.shape[0]) % num_groups
    groups = [MeshGroup(tris[gid == g].astype(np.float32),
                        Material("conductor", roughness=float(rough[g]),
                                 f0=tuple(float(x) for x in f0[g])))
              for g in range(num_groups)]
    G = 20.0
    groups.append(MeshGroup(quad((-G, 0, -G), (-G, 0, G), (G, 0, G), (G, 0, -G)),
                            Material("matte", albedo=(0.5, 0.5, 0.5))))
    groups.append(MeshGroup(quad((-3, 5, -1), (-1, 5, -1), (-1, 5, 1), (-3, 5, 1)), BLACK,
                            radiance=(8.0, 8.0, 8.0)))
    groups.append(MeshGroup(quad((2, 4, 1.5), (3.5, 4, 1.5), (3.5, 3, 3.0), (2, 3, 3.0)), BLACK,
                            radiance=(6.0, 6.0, 6.0)))
    return Scene(f"ggx_sphere_l{level}", width, height, spp, max_bounces,
                 cam_pos=(0.0, 1.6, -4.2), cam_dir=(0.0, -0.12, 1.0), cam_up=(0.0, 1.0, 0.0),
                 fov_deg=45.0, groups=groups, estimator=estimator,
                 env_radiance=(0.1, 0.1, 0.1) if with_env else None)


def furnace(spp: int = 1024, estimator: str = "bneept", sample_filter: str = "box") -> Scene:
    """Grey-furnace known answer (the reference's RenderTest test_gray_furnace_box.py): a convex
    Lambertian icosphere of albedo 0.5 under a constant unit dome, 32 x 32; with exact densities
    every pixel that sees only the sphere is 0.5."""
    sphere = icosphere(3).astype(np.float32)
    groups = [MeshGroup(sphere, Material("matte", albedo=(0.5, 0.5, 0.5)))]
    return Scene("furnace", 32, 32, spp, 10000, cam_pos=(0.0, 0.0, -4.0), cam_dir=(0.0, 0.0, 1.0),
                 cam_up=(0.0, 1.0, 0.0), fov_deg=30.0, groups=groups, estimator=estimator,
                 env_radiance=(1.0, 1.0, 1.0), sample_filter=sample_filter)


def batch_scene(index: int, max_bounces: int = 10, estimator: str = "bneept") -> Scene:
    """Scene `index` (0..63) of the batched workload: seeded by its index, ~U[1k, 500k] triangles
    of random boxes (even indices) or a displaced icosphere (odd indices; 20 * 4**level triangles,
    the level nearest the drawn count), resolution ~U{128..1024} squared, spp ~U{16..256}, eight
    material groups each Lambertian or GGX conductor with probability 1/2, 1-4 quad lights."""
    rng = np.random.default_rng(7000 + index)
    target = int(rng.integers(1000, 500_001))
    res = int(rng.integers(128, 1025))
    spp = int(rng.integers(16, 257))
    num_lights = int(rng.integers(1, 5))
    if index % 2 == 0:
        k = max(target // 12, 1)
        # boxes scattered over a 10 x 10 floor, sizes shrinking with the count (~5 % filled)
        largest = float(np.clip(1.2 * (300.0 / k) ** (1.0 / 3.0), 0.02, 1.2))
        size = rng.uniform(0.2 * largest, largest, (k, 3))
        lo = np.stack([rng.uniform(-5.0, 5.0, k), np.where(rng.random(k) < 0.5, 0.0, rng.uniform(0.0, 3.0, k)),
                       rng.uniform(-5.0, 5.0, k)], 1)
        tris = boxes_axis_aligned(lo, lo + size).reshape(-1, 3, 3)
        centre, extent = np.array([0.0, 1.0, 0.0]), 6.0
    else:
        level = int(np.clip(np.round(np.log(target / 20.0) / np.log(4.0)), 3, 7))
        tris = icosphere(level)
        flat = tris.reshape(-1, 3)
        flat = flat * (1.0 + 0.08 * value_noise3(flat * 2.0, index))[:, None] * 2.0
        tris = flat.reshape(-1, 3, 3)
        tris[:, :, 1] += 2.1
        centre, extent = np.array([0.0, 2.0, 0.0]), 3.5
    gid = rng.integers(0, 8, tris.shape[0])
    groups = []
    for g in range(8):
        sel = tris[gid == g].astype(np.float32)
        if sel.shape[0] == 0:
            continue
        if rng.random() < 0.5:
            m = Material("matte", albedo=tuple(float(x) for x in rng.uniform(0.2, 0.8, 3)))
        else:
            m = Material("conductor", roughness=float(rng.uniform(0.05, 0.6)),
                         f0=tuple(float(x) for x in rng.uniform(0.5, 1.0, 3)))
        groups.append(MeshGroup(sel, m))
    G = 60.0
    groups.append(MeshGroup(quad((-G, 0, -G), (-G, 0, G), (G, 0, G), (G, 0, -G)),
                            Material("matte", albedo=(0.5, 0.5, 0.5))))
    for _ in range(num_lights):
        x, z = rng.uniform(-4.0, 3.0, 2)
        w = float(rng.uniform(0.5, 1.5))
        y = float(rng.uniform(5.0, 7.0))
        radiance = float(rng.uniform(4.0, 12.0))
        groups.append(MeshGroup(quad((x, y, z), (x + w, y, z), (x + w, y, z + w), (x, y, z + w)), BLACK,
                                radiance=(radiance, radiance, radiance)))
    cam = centre + np.array([0.0, 1.0 * extent, -1.4 * extent])
    look = centre - cam
    return Scene(f"batch_{index}", res, res, spp, max_bounces, cam_pos=tuple(float(v) for v in cam),
                 cam_dir=tuple(float(v) for v in look / np.linalg.norm(look)), cam_up=(0.0, 1.0, 0.0),
                 fov_deg=50.0, groups=groups, estimator=estimator)


# ----------------------------------------------------------------------------------------------
# SDL serialisation


def _f(x: float) -> str:
    """Shortest text that round-trips to the same float32."""
    return str(np.float32(x))


def _v3(v) -> str:
    return f"{_f(v[0])} {_f(v[1])} {_f(v[2])}"


def _vec3_array(points: np.ndarray) -> str:
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    return "{" + " ".join('"%s %s %s"' % (str(a), str(b), str(c)) for a, b, c in pts) + "}"


def _zeros_array(n: int) -> str:
    return "{" + " ".join(['"0 0 0"'] * n) + "}"


def _material_sdl(name: str, m: Material, lines: List[str]) -> None:
    if m.kind == "matte":
        lines.append(f'image(constant) @{name}_albedo = [real-array values "{_v3(m.albedo)}"]'
                     f"[enum color-space LSRGB];")
        lines.append(f"material(matte-opaque) @{name} = [image albedo @{name}_albedo];")
    elif m.kind == "conductor":
        lines.append(f"material(abraded-opaque) @{name} = [enum microsurface ggx] "
                     f'[real roughness {_f(m.roughness)}] [spectrum f0 "{_v3(m.f0)}"];')
    elif m.kind == "dielectric":
        lines.append(f"material(abraded-translucent) @{name} = [enum microsurface ggx] "
                     f"[real roughness {_f(m.roughness)}] [real ior-outer {_f(m.ior_outer)}] "
                     f"[real ior-inner {_f(m.ior_inner)}];")
    else:
        raise ValueError(f"unknown material kind {m.kind}")


def to_sdl(scene: Scene, env_image_name: str = "env.pfm", mesh_format: str = "text") -> str:
    """The whole scene as SDL 1.1 command text. mesh_format "ply" refers every mesh group to a
    file g<i>.ply in the scene's directory (write them with write_meshes) instead of spelling its
    vertices out as vector3-array text."""
    lines = [
        "#version 1.1.0;",
        "option(single-frame-render-session) @session = "
        f'[vector2 frame-size "{scene.width} {scene.height}"] [string visualizer @visualizer] '
        "[string observer @observer] [string sample-source @sampler];",
        f"observer(single-lens) @observer = [real fov-degrees {_f(scene.fov_deg)}] "
        f'[vector3 pos "{_v3(scene.cam_pos)}"] [vector3 dir "{_v3(scene.cam_dir)}"] '
        f'[vector3 up-axis "{_v3(scene.cam_up)}"];',
        f"sample-source(stratified) @sampler = [integer samples {scene.spp}];",
        f"visualizer(path-tracing) @visualizer = [enum sample-filter {scene.sample_filter}] "
        f"[enum estimator {scene.estimator}];",
    ]
    for gi, g in enumerate(scene.groups):
        mname = f"m{gi}"
        _material_sdl(mname, g.material, lines)
        n = g.tris.shape[0] * 3
        if mesh_format == "ply":
            lines.append(f'geometry(ply) @g{gi} = [PRI ply-file ":g{gi}.ply"];')
        else:
            lines.append(f"geometry(triangle-mesh) @g{gi} = "
                         f"[vector3-array positions {_vec3_array(g.tris)}] "
                         f"[vector3-array texture-coordinates {_zeros_array(n)}] "
                         f"[vector3-array normals {_zeros_array(n)}];")
        if g.radiance is None:
            lines.append(f"actor(model) @a{gi} = [geometry geometry @g{gi}] [material material @{mname}];")
        else:
            lines.append(f'image(constant) @e{gi} = [real-array values "{_v3(g.radiance)}"]'
                         f"[enum color-space LSRGB];")
            lines.append(f"actor(model-light) @a{gi} = [geometry geometry @g{gi}] "
                         f"[material material @{mname}] [image emitted-energy @e{gi}];")
    if scene.has_env:
        lines.append(f'actor(image-dome) @dome = [PRI image-file ":{env_image_name}"];')
        if scene.env_rotation is not None:
            axis, degrees = scene.env_rotation
            lines.append(f'rotate(@dome) = [vector3 axis "{_v3(axis)}"] [real degrees {_f(degrees)}];')
    return "\n".join(lines) + "\n"


def write_ply(path: str, tris: np.ndarray, fmt: str = "binary_little_endian") -> None:
    """Triangles [n, 3, 3] as a PLY mesh: three float32 vertices per face (not shared), faces as
    `list uchar int vertex_indices`. fmt: binary_little_endian, binary_big_endian or ascii."""
    t = np.asarray(tris, np.float32).reshape(-1, 3)
    n = t.shape[0] // 3
    header = (f"ply\nformat {fmt} 1.0\ncomment photon-v2_b200 scenes.write_ply\n"
              f"element vertex {t.shape[0]}\nproperty float x\nproperty float y\nproperty float z\n"
              f"element face {n}\nproperty list uchar int vertex_indices\nend_header\n")
    idx = np.arange(3 * n, dtype=np.int64).reshape(n, 3)
    with open(path, "wb") as f:
        f.write(header.encode())
        if fmt == "ascii":
            f.write("".join(f"{a!r} {b!r} {c!r}\n" for a, b, c in t.tolist()).encode())
            f.write("".join(f"3 {a} {b} {c}\n" for a, b, c in idx.tolist()).encode())
            return
        order = "<" if fmt == "binary_little_endian" else ">"
        f.write(t.astype(order + "f4").tobytes())
        faces = np.zeros(n, dtype=[("k", "u1"), ("i", order + "i4", (3,))])
        faces["k"] = 3
        faces["i"] = idx
        f.write(faces.tobytes())


def write_meshes(scene: Scene, directory: str, fmt: str = "binary_little_endian") -> None:
    """The PLY files to_sdl(mesh_format="ply") refers to."""
    for gi, g in enumerate(scene.groups):
        write_ply(os.path.join(directory, f"g{gi}.ply"), g.tris, fmt)


def write_env(scene: Scene, directory: str, name: str = "env.pfm") -> None:
    """Writes the scene's dome image (or its 1 x 1 constant radiance) where to_sdl refers to it."""
    if scene.env_image is not None:
        write_pfm(os.path.join(directory, name), np.asarray(scene.env_image, np.float32))
    elif scene.env_radiance is not None:
        write_pfm(os.path.join(directory, name), np.array(scene.env_radiance, np.float32).reshape(1, 1, 3))


def sky_image(width: int = 64, height: int = 32, sun_uv: Tuple[float, float] = (0.3, 0.78),
              sun_radiance: float = 60.0, seed: int = 11) -> np.ndarray:
    """A lat-long sky [height, width, 3] (row 0 = top): a blue-to-white gradient above the
    horizon, a dim brown ground below, seeded per-texel variation, and a small bright sun disk
    centred at lat-long `sun_uv` (u = azimuth / 2 pi, v = 1 at the zenith)."""
    rng = np.random.default_rng(seed)
    v = 1.0 - (np.arange(height) + 0.5) / height          # row 0 = top = v near 1
    u = (np.arange(width) + 0.5) / width
    uu, vv = np.meshgrid(u, v)
    elev = (vv - 0.5) * np.pi                              # -pi/2 .. pi/2
    s = np.sin(np.clip(elev, 0, None))[..., None]          # 0 at the horizon, 1 at the zenith
    sky = (1 - s) * np.array([0.45, 0.5, 0.6]) + s * np.array([0.15, 0.3, 0.7])
    ground = np.stack([0.12 + 0 * uu, 0.09 + 0 * uu, 0.06 + 0 * uu], -1)
    img = np.where((elev >= 0)[..., None], sky, ground)
    img *= 1.0 + 0.15 * rng.random(img.shape[:2])[..., None]
    du = np.minimum(np.abs(uu - sun_uv[0]), 1 - np.abs(uu - sun_uv[0])) * width
    dv = np.abs(vv - sun_uv[1]) * height
    img[(du * du + dv * dv) <= 2.0 ** 2] = sun_radiance * np.array([1.0, 0.9, 0.75])
    return img.astype(np.float32)


def write_pfm(path: str, rgb: np.ndarray) -> None:
    """Little-endian colour PFM, rows stored bottom to top."""
    h, w, _ = rgb.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode())
        f.write(np.ascontiguousarray(rgb[::-1], dtype="<f4").tobytes())
