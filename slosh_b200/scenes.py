"""Seeded synthetic scenes with the shapes, sizes and materials of the
benchmark configurations (no datasets are involved: every scene is
generated from a lattice with seeded jitter).

* ``dam_break_2d``     2D weakly-compressible fluid column, sticky walls
* ``elastic_drop_3d``  two fixed-corotated cubes falling on a slip floor
* ``sand_column_3d``   Drucker-Prager sand cylinder + a rigid cuboid
* ``random_scene_3d``  a box-shaped blob of one material on a floor (the
                       batched / served scenes)
* ``two_way_impact``   an elastic box hitting a free ball coupled two-way
                       (no gravity: total momentum is conserved)

The cell width is a parameter so tests can build the same scenes at small
particle counts.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .pipeline import (
    GpuBoundaryCondition,
    ParticleModel,
    RigidBody,
    SimulationParams,
    make_particles,
    quat_from_axis_angle,
)


@dataclass
class Scene:
    name: str
    dim: int
    cell_width: float
    params: SimulationParams
    particles: np.ndarray
    bodies: list = field(default_factory=list)
    substeps: int = 100
    grid_capacity: int = 1024

    @property
    def n(self) -> int:
        return len(self.particles)


def _lattice(lo, hi, spacing):
    """Cell-centred lattice points of spacing `spacing` inside [lo, hi)."""
    axes = []
    for a, b in zip(lo, hi):
        cnt = int(math.floor((b - a) / spacing + 1e-9))
        axes.append(a + (np.arange(cnt) + 0.5) * spacing)
    grids = np.meshgrid(*axes[::-1], indexing="ij")  # last axis fastest -> x fastest
    pts = np.stack([g.ravel() for g in grids[::-1]], axis=1)
    return pts


def _jitter(pts, amp, rng):
    return pts + rng.uniform(-amp, amp, size=pts.shape)


def _grid_capacity(n_particles: int, ppc: int, dim: int, margin: float = 4.0) -> int:
    cells_per_block = 64
    blocks = n_particles / max(ppc, 1) / cells_per_block
    cap = int(blocks * margin) + 4096
    p = 1
    while p < cap:
        p <<= 1
    return p


def _walls_2d(h: float, bc: GpuBoundaryCondition) -> list:
    """Four cuboid walls of half-thickness 4h whose inner faces are the unit
    box [0, 1]^2."""
    t = 4.0 * h
    return [
        RigidBody(("cuboid", (t, 1.0 + 2 * t)), translation=(-t, 0.5), rotation=0.0, boundary_condition=bc),
        RigidBody(("cuboid", (t, 1.0 + 2 * t)), translation=(1.0 + t, 0.5), rotation=0.0, boundary_condition=bc),
        RigidBody(("cuboid", (1.0 + 2 * t, t)), translation=(0.5, -t), rotation=0.0, boundary_condition=bc),
        RigidBody(("cuboid", (1.0 + 2 * t, t)), translation=(0.5, 1.0 + t), rotation=0.0, boundary_condition=bc),
    ]


def dam_break_2d(h: float = 1.0 / 256.0, seed: int = 1, substeps: int = 1000) -> Scene:
    """Unit box, weakly compressible fluid (rest density 1000, K = 1e4,
    gamma = 7); a 0.4 x 0.6 column in the lower-left corner at 2x2 jittered
    particles per cell; dt = 1e-4; sticky walls."""
    rng = np.random.default_rng(seed)
    lo = (3 * h, 3 * h)
    pts = _lattice(lo, (lo[0] + 0.4, lo[1] + 0.6), h / 2)
    pts = _jitter(pts, h / 4, rng)
    model = ParticleModel.fluid_tait(1000.0, 1.0e4, 7.0)
    parts = make_particles(pts, h / 4, 1000.0, model, dim=2)
    return Scene(
        "dam_break_2d",
        2,
        h,
        SimulationParams((0.0, -9.81), 1.0e-4),
        parts,
        _walls_2d(h, GpuBoundaryCondition.stick()),
        substeps,
        _grid_capacity(len(parts), 4, 2),
    )


def _cube_points(center, side, h, rng, rot_z_deg=0.0):
    half = side / 2
    pts = _lattice((-half,) * 3, (half,) * 3, h / 2)
    pts = _jitter(pts, h / 4, rng)
    if rot_z_deg:
        a = math.radians(rot_z_deg)
        c, s = math.cos(a), math.sin(a)
        x, y = pts[:, 0].copy(), pts[:, 1].copy()
        pts[:, 0] = c * x - s * y
        pts[:, 1] = s * x + c * y
    return pts + np.asarray(center)


def elastic_drop_3d(h: float = 1.0 / 128.0, seed: int = 2, substeps: int = 2000) -> Scene:
    """Two fixed-corotated cubes of side 0.25 (E = 1e5, nu = 0.3, density
    1000) at 2x2x2 jittered particles per cell, the second rotated 30 degrees
    about z, falling onto a slip floor whose top face is at y = 0.05."""
    rng = np.random.default_rng(seed)
    a = _cube_points((0.35, 0.40, 0.50), 0.25, h, rng)
    b = _cube_points((0.65, 0.75, 0.50), 0.25, h, rng, rot_z_deg=30.0)
    pts = np.concatenate([a, b])
    model = ParticleModel.elastic(1.0e5, 0.3)
    parts = make_particles(pts, h / 4, 1000.0, model, dim=3)
    t = 4.0 * h
    floor = RigidBody(("cuboid", (2.0, t, 2.0)), translation=(0.5, 0.05 - t, 0.5), boundary_condition=GpuBoundaryCondition.slip())
    return Scene(
        "elastic_drop_3d",
        3,
        h,
        SimulationParams((0.0, -9.81, 0.0), 5.0e-5),
        parts,
        [floor],
        substeps,
        _grid_capacity(len(parts), 8, 3),
    )


def sand_column_3d(
    h: float = 1.0 / 256.0, seed: int = 3, substeps: int = 500, cube_coupling: str = "one_way", radius: float = 0.15
) -> Scene:
    """Drucker-Prager sand (friction angle 30 deg, E = 3.5e5, nu = 0.3,
    density 2200): a cylinder of radius 0.15 (``radius``) and height 0.5 standing on a
    Separate(1.0) floor at y = 0.05, axis through (0.5, ., 0.5), 8 jittered
    particles per cell, plus a 0.1^3 rigid cuboid (density 500) resting 2h
    above the column, coupled as a collider (one-way; ``cube_coupling``
    "two_way" makes it a dynamic body the sand pushes).  dt = 2e-5."""
    rng = np.random.default_rng(seed)
    r, height, base = radius, 0.5, 0.05
    sp = h / 2
    pts = _lattice((0.5 - r, base, 0.5 - r), (0.5 + r, base + height, 0.5 + r), sp)
    inside = (pts[:, 0] - 0.5) ** 2 + (pts[:, 2] - 0.5) ** 2 <= r * r
    pts = _jitter(pts[inside], h / 4, rng)
    model = ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0)
    parts = make_particles(pts, h / 4, 2200.0, model, dim=3)
    t = 4.0 * h
    floor = RigidBody(("cuboid", (2.0, t, 2.0)), translation=(0.5, base - t, 0.5))
    cube_half = 0.05
    cube_shape = ("cuboid", (cube_half, cube_half, cube_half))
    cube_pos = (0.5, base + height + 2 * h + cube_half, 0.5)
    if cube_coupling == "two_way":
        cube = RigidBody.two_way(cube_shape, 500.0, 3, translation=cube_pos)
    else:
        cube = RigidBody(cube_shape, translation=cube_pos)
    return Scene(
        "sand_column_3d",
        3,
        h,
        SimulationParams((0.0, -9.81, 0.0), 2.0e-5),
        parts,
        [floor, cube],
        substeps,
        _grid_capacity(len(parts), 8, 3),
    )


def random_scene_3d(
    n_target: int,
    material: str,
    h: float,
    seed: int,
    substeps: int = 1000,
) -> Scene:
    """A box-shaped blob of about `n_target` particles (8 per cell) of one
    material, dropped from rest onto a Separate(1.0) floor at y = 0.05."""
    rng = np.random.default_rng(seed)
    side = (n_target / 8.0) ** (1.0 / 3.0) * h
    side = max(side, 4 * h)
    lo = np.array([0.5 - side / 2, 0.1, 0.5 - side / 2])
    pts = _lattice(tuple(lo), tuple(lo + side), h / 2)
    pts = _jitter(pts, h / 4, rng)
    if material == "fluid":
        model, density = ParticleModel.fluid_tait(1000.0, 1.0e4, 7.0), 1000.0
    elif material == "elastic":
        model, density = ParticleModel.elastic(1.0e5, 0.3), 1000.0
    elif material == "sand":
        model, density = ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0), 2200.0
    else:
        raise ValueError(material)
    parts = make_particles(pts, h / 4, density, model, dim=3)
    t = 4.0 * h
    floor = RigidBody(("cuboid", (4.0, t, 4.0)), translation=(0.5, 0.05 - t, 0.5))
    dt = 1.0e-4 if h >= 1.0 / 64 else 5.0e-5
    return Scene(
        f"blob_{material}_{len(parts)}",
        3,
        h,
        SimulationParams((0.0, -9.81, 0.0), dt),
        parts,
        [floor],
        substeps,
        _grid_capacity(len(parts), 8, 3),
    )


def two_way_impact(dim: int = 3, h: float = 1.0 / 32.0, seed: int = 6, substeps: int = 100) -> Scene:
    """A box of fixed-corotated material (E = 1e4, nu = 0.3, density 1000),
    side 0.12, moving at 1 m/s along +x into a free ball of radius 0.06
    (density 1000) at (0.5, 0.5[, 0.5]) coupled two-way, its surface 0.02
    from the box.  No gravity and no other collider, so the total momentum of
    particles and ball is conserved.  2^D jittered particles per cell,
    dt = 1e-4."""
    rng = np.random.default_rng(seed)
    lo = (0.30,) + (0.44,) * (dim - 1)
    hi = (0.42,) + (0.56,) * (dim - 1)
    pts = _jitter(_lattice(lo, hi, h / 2), h / 4, rng)
    parts = make_particles(pts, h / 4, 1000.0, ParticleModel.elastic(1.0e4, 0.3), dim=dim)
    parts["velocity"][:, 0] = 1.0
    centre = (0.5,) * dim
    ball = RigidBody.two_way(("ball", 0.06), 1000.0, dim, translation=centre, rotation=(0.0, 0.0, 0.0, 1.0) if dim == 3 else 0.0)
    return Scene(
        f"two_way_impact_{dim}d",
        dim,
        h,
        SimulationParams((0.0,) * dim, 1.0e-4),
        parts,
        [ball],
        substeps,
        _grid_capacity(len(parts), 2**dim, dim),
    )


def build_mpm_data(scene: Scene, device: int = 0, max_particles: int | None = None):
    from .pipeline import MpmData

    return MpmData(
        scene.params,
        scene.particles,
        scene.bodies,
        cell_width=scene.cell_width,
        grid_capacity=scene.grid_capacity,
        dim=scene.dim,
        device=device,
        max_particles=max_particles,
    )


__all__ = [
    "Scene",
    "dam_break_2d",
    "elastic_drop_3d",
    "sand_column_3d",
    "random_scene_3d",
    "two_way_impact",
    "build_mpm_data",
    "quat_from_axis_angle",
]
