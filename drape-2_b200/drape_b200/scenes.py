"""Seeded synthetic scenes.

Regular-grid meshes stand in for the reference's hex-lattice + CDT mesher (libs/garment/src/sim_mesh_builder.cpp,
which needs CDT 1.4.5, absent here): each rectangular piece is a vertex grid split into triangles with alternating
diagonals, CCW in pattern space, with per-vertex areas of one third of the incident triangle rest areas (as
sim_mesh_builder.cpp:296-301). Bodies are analytic signed distances sampled onto CollisionField grids (the reference
bakes meshes, libs/avatar/src/collision_bake.cpp:98-208; defaults 4 mm cells, 5 cm padding, 2 cm band,
libs/avatar/include/drape/avatar/collision_bake.hpp:10-14).

Workloads:
  sheet_on_sphere()  square sheet 0.5 m, 40 x 40 vertices jittered +-1 mm from a seed, dropped from 0.3 m onto a
                     sphere r = 0.15 m (1600 particles, 3042 triangles).
  seamed_tube()      two 0.55 x 0.7 m panels sewn along both side edges into a sleeve around a capsule-union body
                     lying horizontally (torso r = 0.15 m, h = 0.6 m; arms r = 0.05 m at 45 degrees below
                     horizontal); 63 x 80 vertices per panel (10,080 particles, 128^3 field at 6 mm) or 154 x 195
                     (60,060 particles, 256^3 field at 3 mm).
  plus the reference's own test scenes restated on grids (strip, hanging sheet, sewn pair, patch on sphere, slope).
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np

from .scene import Fabric, Field, Garment, Scene, Settings, jersey_fabric


# ---------------------------------------------------------------------------------------------------------------
# Meshes.

def grid_piece(width: float, height: float, nx: int, ny: int):
    """Vertex grid nx x ny over [0, width] x [0, height]: rest (V, 2), triangles (T, 3), vertex areas, boundary."""
    xs = np.linspace(0.0, width, nx)
    ys = np.linspace(0.0, height, ny)
    gx, gy = np.meshgrid(xs, ys)  # row j = y index
    rest = np.stack([gx.reshape(-1), gy.reshape(-1)], axis=1)
    tris = []
    for j in range(ny - 1):
        for i in range(nx - 1):
            v00 = j * nx + i
            v10 = v00 + 1
            v01 = v00 + nx
            v11 = v01 + 1
            if (i + j) % 2 == 0:
                tris.append((v00, v10, v11))
                tris.append((v00, v11, v01))
            else:
                tris.append((v00, v10, v01))
                tris.append((v10, v11, v01))
    tris = np.asarray(tris, dtype=np.uint32)
    a = rest[tris[:, 1]] - rest[tris[:, 0]]
    b = rest[tris[:, 2]] - rest[tris[:, 0]]
    area = 0.5 * (a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0])
    assert np.all(area > 1e-12), "triangles must be CCW and non-degenerate"
    varea = np.zeros(rest.shape[0])
    for k in range(3):
        np.add.at(varea, tris[:, k], area / 3.0)
    boundary = np.zeros(rest.shape[0], dtype=np.uint8)
    jj, ii = np.divmod(np.arange(rest.shape[0]), nx)
    boundary[(ii == 0) | (ii == nx - 1) | (jj == 0) | (jj == ny - 1)] = 1
    return rest, tris, varea, boundary


def piece_garment(gid: str, width: float, height: float, nx: int, ny: int, fabric: Fabric,
                  grain=(0.0, 1.0)) -> Garment:
    rest, tris, varea, boundary = grid_piece(width, height, nx, ny)
    g = np.asarray(grain, dtype=np.float64)
    g = g / np.linalg.norm(g)
    return Garment(gid, rest, np.zeros(rest.shape[0], np.uint32), varea, tris, np.zeros(tris.shape[0], np.uint32),
                   g.reshape(1, 2), [fabric], np.zeros((0, 4), np.uint32), np.zeros((rest.shape[0], 3)), boundary)


def flat_garment(gid: str, width: float, height: float, h: float, fabric: Fabric, origin=(0.0, 0.0, 0.0),
                 grain=(0.0, 1.0)) -> Garment:
    """One rectangular piece meshed at spacing ~h, laid in the XZ plane: world = origin + (rest.x, 0, rest.y)
    (the reference's flatGarment, libs/sim/tests/sim_test_utils.hpp:14-25)."""
    nx = max(2, int(round(width / h)) + 1)
    ny = max(2, int(round(height / h)) + 1)
    g = piece_garment(gid, width, height, nx, ny, fabric, grain)
    o = np.asarray(origin, dtype=np.float64)
    g.initial_positions = np.stack([o[0] + g.rest[:, 0], np.full(g.vertex_count, o[1]), o[2] + g.rest[:, 1]], axis=1)
    return g


# ---------------------------------------------------------------------------------------------------------------
# Bodies.

def _grid_points(origin, cell, dims):
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return (origin[0] + x * cell, origin[1] + y * cell, origin[2] + z * cell)


def sampled_field(sdf, origin, cell: float, dims, band: float) -> Field:
    """Samples an analytic signed distance (negative inside) at origin + (i, j, k) * cell, x fastest, clamped to
    [-band, band] (collision_field.hpp:10)."""
    px, py, pz = _grid_points(np.asarray(origin, dtype=np.float64), cell, dims)
    vals = np.clip(sdf(px, py, pz), -band, band).astype(np.float32)
    return Field(np.asarray(origin, dtype=np.float64), float(cell), tuple(int(d) for d in dims), float(band), vals)


def sphere_sdf(center, radius):
    cx, cy, cz = center

    def f(x, y, z):
        return np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) - radius
    return f


def capsule_sdf(a, b, radius):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    ab = b - a
    L2 = float(ab @ ab)

    def f(x, y, z):
        px, py, pz = x - a[0], y - a[1], z - a[2]
        t = np.clip((px * ab[0] + py * ab[1] + pz * ab[2]) / L2, 0.0, 1.0)
        dx, dy, dz = px - t * ab[0], py - t * ab[1], pz - t * ab[2]
        return np.sqrt(dx * dx + dy * dy + dz * dz) - radius
    return f


def box_sdf(center, half, rotation):
    c = np.asarray(center, dtype=np.float64)
    R = np.asarray(rotation, dtype=np.float64)
    h = np.asarray(half, dtype=np.float64)

    def f(x, y, z):
        p = np.stack([x - c[0], y - c[1], z - c[2]], axis=-1) @ R  # world -> box frame (R^T p)
        q = np.abs(p) - h
        outside = np.linalg.norm(np.maximum(q, 0.0), axis=-1)
        inside = np.minimum(np.max(q, axis=-1), 0.0)
        return outside + inside
    return f


def union(*fs):
    def f(x, y, z):
        out = fs[0](x, y, z)
        for g in fs[1:]:
            out = np.minimum(out, g(x, y, z))
        return out
    return f


def sphere_field(radius=0.15, center=(0.0, 0.0, 0.0), cell=0.004, pad=0.05, band=0.02) -> Field:
    """A sphere baked the way the reference bakes its test sphere (cell 4 mm, pad 5 cm, band 2 cm)."""
    lo = np.asarray(center) - radius - pad
    span = 2 * (radius + pad)
    n = int(math.ceil(span / cell)) + 1
    return sampled_field(sphere_sdf(center, radius), lo, cell, (n, n, n), band)


TORSO_HALF = 0.3        # torso capsule: segment of 0.6 m along z, centred at the origin
TORSO_RADIUS = 0.15
ARM_RADIUS = 0.05
ARM_LENGTH = 0.45


def capsule_union_sdf(torso_radius=TORSO_RADIUS, arm_radius=ARM_RADIUS):
    """The capsule-union body, lying down: a torso capsule (r = 0.15 m, h = 0.6 m) along z through the origin, and two
    arm capsules (r = 0.05 m, 0.45 m long) leaving the torso's end points outward along +-z and 45 degrees below
    horizontal. A garment wrapped around the torso hangs from its top; the arms stand under the garment's open
    ends."""
    c, s = math.cos(math.radians(45.0)), math.sin(math.radians(45.0))
    parts = [capsule_sdf((0.0, 0.0, -TORSO_HALF), (0.0, 0.0, TORSO_HALF), torso_radius)]
    for sign in (1.0, -1.0):
        root = (0.0, 0.0, sign * TORSO_HALF)
        tip = (0.0, -ARM_LENGTH * s, sign * (TORSO_HALF + ARM_LENGTH * c))
        parts.append(capsule_sdf(root, tip, arm_radius))
    return union(*parts)


def capsule_union_field(n: int = 128, cell: float = 0.006, band: float = 0.02, torso_radius=TORSO_RADIUS,
                        arm_radius=ARM_RADIUS) -> Field:
    """The capsule union sampled on an n^3 grid centred on the torso (y shifted down by a quarter span, where the
    garment hangs). The grid must hold the 0.7 m garment: a 128^3 grid at the workload's nominal 4 mm spans only
    0.508 m, so the sample count is kept and the spacing widened (6 mm for 128^3, 3 mm for 256^3). Outside the grid
    the field is +band (no contact), as in collision_field.cpp:15."""
    span = (n - 1) * cell
    origin = (-0.5 * span, 0.16 - span, -0.5 * span)  # top of the grid 1 cm above the torso's top line
    return sampled_field(capsule_union_sdf(torso_radius, arm_radius), origin, cell, (n, n, n), band)


# ---------------------------------------------------------------------------------------------------------------
# Workloads.

def sheet_fabric() -> Fabric:
    """Sheet-on-sphere fabric: stretch 5e3 N/m warp and weft, bend 1e-5 N m, 0.15 kg/m^2, friction 0.3. The bias
    stiffness, strain limits, thickness and damping are not given by the workload; they take the jersey test fabric's
    ratios and values (bias = warp / 4, limits 0.5 / 0.8, 0.6 mm, damping 0.3)."""
    return Fabric(5e3, 5e3, 1.25e3, 0.5, 0.8, 1e-5, 1e-5, 0.15, 0.0006, 0.3, 0.3)


def sheet_on_sphere(n: int = 40, size: float = 0.5, height: float = 0.3, jitter: float = 1e-3, seed: int = 1,
                    cg_tolerance: float = 1e-6, max_cg: int = 200, field: Optional[Field] = None) -> Scene:
    g = piece_garment("sheet", size, size, n, n, sheet_fabric())
    rng = np.random.default_rng(seed)
    base = np.stack([g.rest[:, 0] - size / 2, np.full(g.vertex_count, height), g.rest[:, 1] - size / 2], axis=1)
    g.initial_positions = base + rng.uniform(-jitter, jitter, size=base.shape)
    s = Settings(cg_tolerance=cg_tolerance, max_cg_iterations=max_cg)
    return Scene([g], field if field is not None else sphere_field(), settings=s)


def tube_fabric(friction: float = 0.4) -> Fabric:
    """Tube fabric: the jersey test fabric with friction mu = 0.4."""
    f = jersey_fabric()
    f.friction = friction
    return f


def seamed_tube(nx: int = 63, ny: int = 80, width: float = 0.55, height: float = 0.7, radius: float = 0.20,
                friction: float = 0.4, field: Optional[Field] = None, field_n: int = 128,
                field_cell: float = 0.006, torso_radius=TORSO_RADIUS, arm_radius=ARM_RADIUS,
                settings: Optional[Settings] = None, gid: str = "tube") -> Scene:
    """Two panels (upper, lower) wrapped on a cylinder of the given radius around the torso's axis (z), sewn along
    both side edges (the 0.7 m edges, which run along the axis). The placement follows the reference's cylinder
    placement (libs/garment/src/placement.cpp:35-41): theta = centre + x / R, axial = y. At R = 0.2 m the open seams
    leave ~8 cm gaps at the sides; Assembling closes them into a 1.1 m-round sleeve, looser than the torso, which then
    hangs from the torso's top under gravity."""
    rest1, tris1, va1, b1 = grid_piece(width, height, nx, ny)
    V = rest1.shape[0]
    rest = np.concatenate([rest1, rest1])
    tris = np.concatenate([tris1, tris1 + V]).astype(np.uint32)
    tpiece = np.concatenate([np.zeros(len(tris1)), np.ones(len(tris1))]).astype(np.uint32)
    vpiece = np.concatenate([np.zeros(V), np.ones(V)]).astype(np.uint32)
    varea = np.concatenate([va1, va1])
    boundary = np.concatenate([b1, b1])
    jj, ii = np.divmod(np.arange(V), nx)
    left = np.where(ii == 0)[0]
    right = np.where(ii == nx - 1)[0]
    left = left[np.argsort(jj[left])]
    right = right[np.argsort(jj[right])]
    # seam 0: front right <-> back left; seam 1: back right <-> front left, each bottom to top.
    pairs = []
    for k in range(ny):
        pairs.append((right[k], V + left[k], 0, k))
    for k in range(ny):
        pairs.append((V + right[k], left[k], 1, k))
    pairs = np.asarray(pairs, dtype=np.uint32)
    x = np.zeros((2 * V, 3))
    for piece, centre in ((0, 0.0), (1, math.pi)):
        sl = slice(piece * V, (piece + 1) * V)
        theta = centre + (rest[sl, 0] - width / 2) / radius
        x[sl, 0] = radius * np.sin(theta)
        x[sl, 1] = radius * np.cos(theta)
        x[sl, 2] = rest[sl, 1] - height / 2
    fab = tube_fabric(friction)
    g = Garment(gid, rest, vpiece, varea, tris, tpiece, np.array([[0.0, 1.0], [0.0, 1.0]]), [fab, fab], pairs, x,
                boundary)
    if field is None:
        field = capsule_union_field(field_n, field_cell, torso_radius=torso_radius, arm_radius=arm_radius)
    return Scene([g], field, settings=settings or Settings())


def tube_10k(**kw) -> Scene:
    return seamed_tube(63, 80, field_n=128, field_cell=0.006, **kw)


def tube_60k(**kw) -> Scene:
    return seamed_tube(154, 195, field_n=256, field_cell=0.003, **kw)


def _tube_of_size(n_particles: int, w: float, h: float, tr: float, ar: float, field_n: int,
                  settings: Optional[Settings], gid: str, radius: Optional[float] = None) -> Scene:
    per_panel = n_particles / 2
    nx = max(4, int(round(math.sqrt(per_panel * w / h))))
    ny = max(4, int(round(per_panel / nx)))
    radius = tr + 0.05 if radius is None else radius
    cell = 0.762 / (field_n - 1)
    return seamed_tube(nx, ny, width=w, height=h, radius=radius, field_n=field_n, field_cell=cell, torso_radius=tr,
                       arm_radius=ar, settings=settings, gid=gid)


def tube_variant(seed: int, n_particles: int, field_n: int = 128, settings: Optional[Settings] = None) -> Scene:
    """A seeded tube variant: panel sizes +-20 %, torso and arm radii +-15 %, about n_particles particles."""
    rng = np.random.default_rng(seed)
    w = 0.55 * rng.uniform(0.8, 1.2)
    h = 0.7 * rng.uniform(0.8, 1.2)
    tr = TORSO_RADIUS * rng.uniform(0.85, 1.15)
    ar = ARM_RADIUS * rng.uniform(0.85, 1.15)
    return _tube_of_size(n_particles, w, h, tr, ar, field_n, settings, f"tube{seed}")


def body_tube(seed: int, n_particles: int, field_n: int = 128) -> Scene:
    """The seamed tube of the tube workloads (two 0.55 x 0.7 m panels on a 0.2 m cylinder) at about n_particles
    particles, on its own seeded capsule-union body: torso radius 0.15 m +-5 %, arm radius 0.05 m +-10 %, so every
    sleeve is as loose on its torso as the workloads' tube (its circumference 1.17 x the torso's, +-5 %)."""
    rng = np.random.default_rng(seed)
    tr = TORSO_RADIUS * rng.uniform(0.95, 1.05)
    ar = ARM_RADIUS * rng.uniform(0.9, 1.1)
    return _tube_of_size(n_particles, 0.55, 0.7, tr, ar, field_n, None, f"body{seed}", radius=0.2)


def batch_tubes(count: int = 64, seed: int = 5, n_min: int = 2000, n_max: int = 40000):
    """Uneven batch of seeded tubes (body_tube): particle counts log-uniform in [n_min, n_max], each tube on its own
    seeded capsule-union body whose field resolution grows with the garment, from 32^3 samples at n_min to 128^3 at
    n_max (log-linear). Returns the scenes in order."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), count))
    scenes = []
    for k, n in enumerate(ns):
        t = math.log(n / n_min) / math.log(n_max / n_min) if n_max > n_min else 0.0
        field_n = int(round(32 * 4 ** t))
        scenes.append(body_tube(seed * 1000 + k, int(round(n)), field_n=field_n))
    return scenes


# ---------------------------------------------------------------------------------------------------------------
# The reference's test scenes, restated on grid meshes.

def strip_scene(grain=(1.0, 0.0), fabric: Optional[Fabric] = None, h: float = 0.005) -> Scene:
    """Strip 0.2 x 0.05 m pinned at x = 0 and pulled along +x with 0.5 N in total at x = 0.2, no gravity
    (libs/sim/tests/test_cpu_solver.cpp:30-53)."""
    if fabric is None:
        fabric = jersey_fabric()
        fabric.damping = 1.0
    g = flat_garment("strip", 0.2, 0.05, h, fabric, grain=grain)
    scene = Scene([g], settings=Settings(gravity=(0.0, 0.0, 0.0)))
    r = g.rest
    for v in np.where(r[:, 0] <= 1e-9)[0]:
        scene.pins.append((int(v), tuple(g.initial_positions[v])))
    loaded = np.where(r[:, 0] >= 0.2 - 1e-9)[0]
    loaded = loaded[np.argsort(r[loaded, 1])]
    for i, v in enumerate(loaded):
        lo = r[v, 1] if i == 0 else 0.5 * (r[v, 1] + r[loaded[i - 1], 1])
        hi = r[v, 1] if i + 1 == len(loaded) else 0.5 * (r[v, 1] + r[loaded[i + 1], 1])
        scene.forces.append((int(v), (0.5 * (hi - lo) / 0.05, 0.0, 0.0)))
    return scene


def measured_strain(x: np.ndarray, rest: np.ndarray) -> float:
    """Least-squares slope of world x over rest x for rest x in [0.04, 0.16], minus one (test_cpu_solver.cpp:55-70)."""
    r = rest[:, 0]
    sel = (r >= 0.04) & (r <= 0.16)
    rr, xx = r[sel], x[sel, 0]
    n = len(rr)
    slope = (n * np.sum(rr * xx) - np.sum(rr) * np.sum(xx)) / (n * np.sum(rr * rr) - np.sum(rr) ** 2)
    return float(slope - 1.0)


def hanging_sheet() -> Scene:
    """0.5 x 0.5 m jersey sheet (h = 1 cm) in the XY plane pinned at its two top corners
    (libs/sim/tests/sim_test_utils.hpp:52-80)."""
    g = piece_garment("sheet", 0.5, 0.5, 51, 51, jersey_fabric())
    g.initial_positions = np.stack([g.rest[:, 0], 0.5 + g.rest[:, 1], np.zeros(g.vertex_count)], axis=1)
    scene = Scene([g])
    for corner in ((0.0, 0.5), (0.5, 0.5)):
        v = int(np.argmin(np.linalg.norm(g.rest - np.asarray(corner), axis=1)))
        scene.pins.append((v, tuple(g.initial_positions[v])))
    return scene


def centred_sheet(size: float, h: float, height: float, fabric: Optional[Fabric] = None) -> Garment:
    """libs/sim/tests/sphere_scene.hpp:24-27."""
    return flat_garment("sheet", size, size, h, fabric or jersey_fabric(), (-size / 2, height, -size / 2))


K_CONTACT = 0.003 + 0.0006 / 2  # collision offset + half the jersey thickness (sphere_scene.hpp:21)


def sewn_pair(w=0.05, hgt=0.05, gap=0.1, h=0.01, fabric: Optional[Fabric] = None) -> Garment:
    """Two w x hgt squares in the XZ plane, the second shifted by gap beyond the first's right edge, sewn
    first.right <-> second.left (libs/sim/tests/test_seams.cpp:12-29)."""
    fabric = fabric or jersey_fabric()
    nx = int(round(w / h)) + 1
    ny = int(round(hgt / h)) + 1
    rest1, tris1, va1, b1 = grid_piece(w, hgt, nx, ny)
    V = rest1.shape[0]
    jj, ii = np.divmod(np.arange(V), nx)
    right = np.where(ii == nx - 1)[0]
    left = np.where(ii == 0)[0]
    right = right[np.argsort(jj[right])]
    left = left[np.argsort(jj[left])]
    pairs = np.asarray([(right[k], V + left[k], 0, k) for k in range(ny)], dtype=np.uint32)
    rest = np.concatenate([rest1, rest1])
    x = np.zeros((2 * V, 3))
    x[:V, 0] = rest1[:, 0]
    x[:V, 2] = rest1[:, 1]
    x[V:, 0] = rest1[:, 0] + w + gap
    x[V:, 2] = rest1[:, 1]
    return Garment("pair", rest, np.concatenate([np.zeros(V), np.ones(V)]).astype(np.uint32),
                   np.concatenate([va1, va1]), np.concatenate([tris1, tris1 + V]).astype(np.uint32),
                   np.concatenate([np.zeros(len(tris1)), np.ones(len(tris1))]).astype(np.uint32),
                   np.array([[0.0, 1.0], [0.0, 1.0]]), [fabric, fabric], pairs, x)


def slope_scene(friction: float, angle_deg: float = 20.0):
    """A 2 x 2 cm jersey patch resting 4 mm above a box tilted by angle_deg about z
    (libs/sim/tests/test_body_collision.cpp:139-169). Returns the scene and the uphill direction."""
    a = math.radians(angle_deg)
    R = np.array([[math.cos(a), -math.sin(a), 0.0], [math.sin(a), math.cos(a), 0.0], [0.0, 0.0, 1.0]])
    up = R @ np.array([0.0, 1.0, 0.0])
    uphill = R @ np.array([1.0, 0.0, 0.0])
    sdf = box_sdf(-0.05 * up, (0.5, 0.05, 0.5), R)
    cell, pad = 0.004, 0.05
    # Bake only around the patch: the box is large, the patch small.
    lo = np.array([-0.1, -0.1, -0.1])
    n = int(math.ceil(0.2 / cell)) + 1
    field = sampled_field(sdf, lo, cell, (n, n, n), 0.02)
    f = jersey_fabric()
    f.friction = friction
    g = flat_garment("patch", 0.02, 0.02, 0.01, f)
    r = g.rest - 0.01
    local = np.stack([r[:, 0], np.zeros(len(r)), r[:, 1]], axis=1)
    g.initial_positions = local @ R.T + 0.004 * up
    return Scene([g], field), uphill
