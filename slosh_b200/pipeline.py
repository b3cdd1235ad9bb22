"""Host-side mirror of slosh's pipeline API over the C ABI.

Names and argument meaning follow dimforge/slosh:

* ``SimulationParams``            src/solver/params.rs:13-21
* ``ElasticCoefficients``          src/models/mod.rs:52-59
* ``DruckerPrager``                src/models/drucker_prager.rs:12-68
* ``ParticleModel``                src/solver/particle_model.rs:9-80
* ``Particle`` / ``ParticleDynamics``  src/solver/particle.rs:23-100, 226-233
* ``GpuBoundaryCondition``         src/solver/boundary_condition.rs:8-65
* ``MpmData``                      src/pipeline.rs:311-430
* ``MpmPipeline.launch_step``      src/pipeline.rs:562-770

Rigid bodies are given directly (shape, pose, velocity, mass properties and
boundary condition) instead of through rapier's body/collider sets; the
one-way coupling of ``MpmData::new`` (zero mass properties) is the default.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np

from . import _lib
from ._lib import (
    BODY_DTYPE,
    PARTICLE_DTYPE,
    SloshConfig,
    SloshError,
    SloshGridDump,
    SloshParams,
    ptr,
)


@dataclass
class SimulationParams:
    gravity: Sequence[float] = (0.0, -9.81, 0.0)
    dt: float = 1.0 / 60.0


def lame_lambda_mu(young_modulus: float, poisson_ratio: float) -> tuple[float, float]:
    """src/models/mod.rs:17-27, in float32 like the reference."""
    e = np.float32(young_modulus)
    nu = np.float32(poisson_ratio)
    one = np.float32(1.0)
    two = np.float32(2.0)
    lam = e * nu / ((one + nu) * (one - two * nu))
    mu = e / (two * (one + nu))
    return float(np.float32(lam)), float(np.float32(mu))


@dataclass
class ElasticCoefficients:
    lam: float
    mu: float
    cfl_coeff: float = 0.5

    @staticmethod
    def from_young_modulus(young_modulus: float, poisson_ratio: float) -> "ElasticCoefficients":
        lam, mu = lame_lambda_mu(young_modulus, poisson_ratio)
        return ElasticCoefficients(lam, mu, 0.5)


@dataclass
class DruckerPrager:
    h0: float
    h1: float
    h2: float
    h3: float
    lam: float
    mu: float

    @staticmethod
    def new(young_modulus: float, poisson_ratio: float) -> "DruckerPrager":
        if young_modulus > 0.0:
            lam, mu = lame_lambda_mu(young_modulus, poisson_ratio)
        else:
            lam, mu = -1.0, -1.0
        return DruckerPrager.from_lame(lam, mu)

    @staticmethod
    def from_lame(lam: float, mu: float) -> "DruckerPrager":
        return DruckerPrager(math.radians(35.0), math.radians(9.0), 0.2, math.radians(10.0), lam, mu)


@dataclass
class ParticleModel:
    """A GpuParticleModel record: tag + 12 payload words."""

    tag: int
    data: tuple

    @staticmethod
    def elastic(young_modulus: float, poisson_ratio: float) -> "ParticleModel":
        c = ElasticCoefficients.from_young_modulus(young_modulus, poisson_ratio)
        return ParticleModel(_lib.MODEL_ELASTIC_LINEAR, (c.lam, c.mu, c.cfl_coeff) + (0.0,) * 9)

    @staticmethod
    def elastic_neo_hookean(young_modulus: float, poisson_ratio: float) -> "ParticleModel":
        c = ElasticCoefficients.from_young_modulus(young_modulus, poisson_ratio)
        return ParticleModel(_lib.MODEL_ELASTIC_NEO_HOOKEAN, (c.lam, c.mu, c.cfl_coeff) + (0.0,) * 9)

    @staticmethod
    def _sand(tag: int, young_modulus: float, poisson_ratio: float, friction_angle_deg: float | None):
        plastic = DruckerPrager.new(young_modulus, poisson_ratio)
        if friction_angle_deg is not None:
            plastic.h0 = math.radians(friction_angle_deg)
        c = ElasticCoefficients.from_young_modulus(young_modulus, poisson_ratio)
        state = (1.0, 1.0, 0.0)  # DruckerPragerPlasticState::default
        return ParticleModel(
            tag,
            state
            + (plastic.h0, plastic.h1, plastic.h2, plastic.h3, plastic.lam, plastic.mu)
            + (c.lam, c.mu, c.cfl_coeff),
        )

    @staticmethod
    def sand(young_modulus: float, poisson_ratio: float, friction_angle_deg: float | None = None) -> "ParticleModel":
        return ParticleModel._sand(_lib.MODEL_SAND_LINEAR, young_modulus, poisson_ratio, friction_angle_deg)

    @staticmethod
    def sand_neo_hookean(
        young_modulus: float, poisson_ratio: float, friction_angle_deg: float | None = None
    ) -> "ParticleModel":
        return ParticleModel._sand(_lib.MODEL_SAND_NEO_HOOKEAN, young_modulus, poisson_ratio, friction_angle_deg)

    @staticmethod
    def fluid_tait(rest_density: float, bulk_modulus: float, gamma: float) -> "ParticleModel":
        return ParticleModel(_lib.MODEL_FLUID_TAIT, (rest_density, bulk_modulus, gamma) + (0.0,) * 9)


def make_particles(
    positions: np.ndarray,
    radius: float,
    density: float,
    model: ParticleModel,
    dim: int = 3,
    velocities: np.ndarray | None = None,
) -> np.ndarray:
    """Vectorised ``Particle::new(position, radius, density, model)``
    (src/solver/particle.rs:66-84, 236-246): V0 = (2r)^dim, mass = V0 density,
    F = I, C = 0, enabled, not fixed."""
    pos = np.asarray(positions, dtype=np.float32)
    n = pos.shape[0]
    rec = np.zeros(n, dtype=PARTICLE_DTYPE)
    rec["position"][:, : pos.shape[1]] = pos
    if velocities is not None:
        v = np.asarray(velocities, dtype=np.float32)
        rec["velocity"][:, : v.shape[1]] = v
    ident = np.zeros(9, np.float32)
    ident[0] = ident[4] = 1.0
    if dim == 3:
        ident[8] = 1.0
    rec["def_grad"][:] = ident
    d2 = np.float32(np.float32(radius) * np.float32(2.0))
    vol = d2 * d2 * d2 if dim == 3 else d2 * d2  # f32 powi, repeated products
    rec["init_volume"] = vol
    rec["init_radius"] = radius
    rec["mass"] = np.float32(vol) * np.float32(density)
    rec["phase"] = 1.0
    rec["enabled"] = 1
    rec["model_tag"] = model.tag
    rec["model"][:] = np.asarray(model.data, dtype=np.float32)
    return rec


class GpuBoundaryCondition:
    """Boundary condition of a collider (src/solver/boundary_condition.rs)."""

    def __init__(self, ty: int, friction: float = 0.0):
        self.ty = ty
        self.friction = friction

    @staticmethod
    def stick():
        return GpuBoundaryCondition(_lib.BC_STICK, 0.0)

    @staticmethod
    def slip():
        return GpuBoundaryCondition(_lib.BC_SLIP, 0.0)

    @staticmethod
    def separate(friction: float):
        return GpuBoundaryCondition(_lib.BC_SEPARATE, friction)

    @staticmethod
    def friction_z_up(friction: float):
        return GpuBoundaryCondition(_lib.BC_FRICTION_Z_UP, friction)

    @staticmethod
    def disabled():
        return GpuBoundaryCondition(_lib.BC_DISABLED, 0.0)

    @staticmethod
    def default():
        return GpuBoundaryCondition.separate(1.0)


@dataclass
class RigidBody:
    """One body with its collider (a GpuBodySet entry).  ``shape`` is
    ("cuboid", half_extents), ("ball", radius), ("capsule", (a, b, radius))
    with a, b the segment end points, or in 3D ("cylinder", (half_height,
    radius)) or ("cone", (half_height, radius)) around the local y axis
    (GpuShape layouts, shaders/slosh/rbd/shapes/shape.slang:37-80), or in 3D
    ("trimesh", (vertices, triangles)) with vertices an (n, 3) array and
    triangles an (m, 3) array of vertex indices, counter-clockwise seen from
    outside (``box_mesh``, ``heightfield_mesh``).  Rotation
    is a unit quaternion (i, j, k, w) in 3D or an angle in radians in 2D.
    ``coupling`` is "one_way" (slosh's GPU behaviour: the particles never
    push the body) or "two_way" (the grid's contact impulses move it; see
    :meth:`two_way`).  ``inv_inertia`` is the world-space inverse inertia at
    this pose: a 3x3 matrix in 3D, a scalar in 2D."""

    shape: tuple
    translation: Sequence[float] = (0.0, 0.0, 0.0)
    rotation: Sequence[float] | float = (0.0, 0.0, 0.0, 1.0)
    linvel: Sequence[float] = (0.0, 0.0, 0.0)
    angvel: Sequence[float] = (0.0, 0.0, 0.0)
    inv_mass: Sequence[float] = (0.0, 0.0, 0.0)
    local_com: Sequence[float] = (0.0, 0.0, 0.0)
    boundary_condition: GpuBoundaryCondition = field(default_factory=GpuBoundaryCondition.default)
    scale: float = 1.0
    inv_inertia: object = None
    coupling: str = "one_way"

    @classmethod
    def two_way(cls, shape: tuple, density: float, dim: int, **kw) -> "RigidBody":
        """A dynamic body coupled two-way, with the mass properties of its
        shape (cuboid or ball, scaled by ``scale``) at ``density``, centre of
        mass at the shape's origin."""
        body = cls(shape, coupling="two_way", **kw)
        m, inertia = shape_mass_properties(shape, density, dim, body.scale)
        body.inv_mass = (1.0 / m,) * 3 if dim == 3 else (1.0 / m, 1.0 / m, 0.0)
        if dim == 3:
            rot = quat_to_matrix(body.rotation)
            body.inv_inertia = rot @ np.diag(1.0 / np.asarray(inertia)) @ rot.T
        else:
            body.inv_inertia = 1.0 / float(inertia)
        return body

    def record(self, dim: int) -> np.ndarray:
        r = np.zeros((), dtype=BODY_DTYPE)
        kind, param = self.shape
        if kind == "cuboid":
            he = list(param) + [0.0] * (3 - len(param))
            r["shape_a"][:3] = he[:3]
            r["shape_a"].view(np.uint32)[3] = _lib.SHAPE_CUBOID
        elif kind == "ball":
            r["shape_a"][0] = float(param)
            r["shape_a"].view(np.uint32)[3] = _lib.SHAPE_BALL
        elif kind == "capsule":
            a, b, radius = param
            a = list(a) + [0.0] * (3 - len(a))
            b = list(b) + [0.0] * (3 - len(b))
            r["shape_a"][:3] = a[:3]
            r["shape_a"].view(np.uint32)[3] = _lib.SHAPE_CAPSULE
            r["shape_b"][:3] = b[:3]
            r["shape_b"][3] = float(radius)
        elif kind in ("cylinder", "cone") and dim == 3:
            hh, radius = param
            r["shape_a"][0] = float(hh)
            r["shape_a"][1] = float(radius)
            r["shape_a"].view(np.uint32)[3] = _lib.SHAPE_CYLINDER if kind == "cylinder" else _lib.SHAPE_CONE
        elif kind == "trimesh" and dim == 3:
            # the mesh offsets are filled in by the context the mesh is added to
            r["shape_a"].view(np.uint32)[3] = _lib.SHAPE_TRIMESH
        else:
            raise ValueError(f"unsupported shape {kind!r}")
        if dim == 3:
            r["rotation"][:] = np.asarray(self.rotation, np.float32)
        else:
            ang = float(self.rotation) if np.isscalar(self.rotation) else 0.0
            r["rotation"][:2] = (math.cos(ang), math.sin(ang))
        t = list(self.translation) + [0.0] * (3 - len(self.translation))
        r["translation"][:3] = t[:3]
        r["translation"][3] = self.scale
        for name in ("linvel", "angvel", "inv_mass", "local_com"):
            v = list(getattr(self, name))
            v = v + [0.0] * (3 - len(v))
            r[name][:3] = v[:3]
        r["bc_type"] = self.boundary_condition.ty
        r["bc_friction"] = self.boundary_condition.friction
        if self.inv_inertia is not None:
            if dim == 3:
                m = np.asarray(self.inv_inertia, np.float64).reshape(3, 3)
                for c in range(3):
                    r["inv_inertia"][4 * c : 4 * c + 3] = m[:, c]
            else:
                r["inv_inertia"][0] = float(self.inv_inertia)
        modes = {"one_way": _lib.COUPLING_ONE_WAY, "two_way": _lib.COUPLING_TWO_WAY}
        if self.coupling not in modes:
            raise ValueError(f"unknown coupling {self.coupling!r}")
        r["coupling"] = modes[self.coupling]
        return r


def shape_mass_properties(shape: tuple, density: float, dim: int, scale: float = 1.0):
    """Mass and principal inertia (3D: the three moments; 2D: the scalar)
    of a uniform cuboid or ball about its centre."""
    kind, param = shape
    if kind == "cuboid":
        he = [float(v) * scale for v in list(param)[:dim]]
        if dim == 3:
            m = density * 8.0 * he[0] * he[1] * he[2]
            return m, (m / 3.0 * (he[1] ** 2 + he[2] ** 2), m / 3.0 * (he[0] ** 2 + he[2] ** 2),
                       m / 3.0 * (he[0] ** 2 + he[1] ** 2))
        m = density * 4.0 * he[0] * he[1]
        return m, m / 3.0 * (he[0] ** 2 + he[1] ** 2)
    if kind == "ball":
        r = float(param) * scale
        if dim == 3:
            m = density * 4.0 / 3.0 * math.pi * r**3
            return m, (0.4 * m * r * r,) * 3
        m = density * math.pi * r * r
        return m, 0.5 * m * r * r
    raise ValueError(f"mass properties of {kind!r} are not implemented")


def mesh_arrays(shape: tuple) -> tuple[np.ndarray, np.ndarray]:
    """The (vertices, triangles) of a ("trimesh", ...) shape as contiguous
    float32 (n, 3) and uint32 (m, 3) arrays."""
    v, t = shape[1]
    return np.ascontiguousarray(v, np.float32).reshape(-1, 3), np.ascontiguousarray(t, np.uint32).reshape(-1, 3)


def box_mesh(half_extents: Sequence[float]) -> tuple[np.ndarray, np.ndarray]:
    """A closed box of 12 triangles, outward counter-clockwise."""
    hx, hy, hz = (float(x) for x in half_extents)
    v = np.array([[sx * hx, sy * hy, sz * hz] for sz in (-1, 1) for sy in (-1, 1) for sx in (-1, 1)], np.float32)
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    t = []
    for a, b, c, d in quads:
        t += [(a, b, c), (a, c, d)]
    return v, np.array(t, np.uint32)


def heightfield_mesh(heights: np.ndarray, extent: Sequence[float]) -> tuple[np.ndarray, np.ndarray]:
    """The triangle mesh of a heightfield (rows along z, columns along x)
    over [-ex/2, ex/2] x [-ez/2, ez/2], up = +y, as slosh turns heightfields
    into meshes (src/rbd/shapes.rs:241-269)."""
    h = np.asarray(heights, np.float32)
    nz, nx = h.shape
    ex, ez = float(extent[0]), float(extent[1])
    xs = np.linspace(-ex / 2, ex / 2, nx, dtype=np.float32)
    zs = np.linspace(-ez / 2, ez / 2, nz, dtype=np.float32)
    v = np.stack([np.tile(xs, nz), h.ravel(), np.repeat(zs, nx)], axis=1).astype(np.float32)
    t = []
    for iz in range(nz - 1):
        for ix in range(nx - 1):
            a, b = iz * nx + ix, iz * nx + ix + 1
            c, d = a + nx, b + nx
            t += [(a, c, b), (b, c, d)]
    return v, np.array(t, np.uint32)


def quat_to_matrix(q: Sequence[float]) -> np.ndarray:
    """Rotation matrix of the unit quaternion (i, j, k, w)."""
    x, y, z, w = (float(v) for v in q)
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ]
    )


def quat_from_axis_angle(axis: Sequence[float], angle: float) -> tuple:
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s = math.sin(angle / 2.0)
    return (float(a[0] * s), float(a[1] * s), float(a[2] * s), math.cos(angle / 2.0))


def _check(lib, ctx, code: int):
    if code != 0:
        buf = ctypes.create_string_buffer(512)
        if ctx:
            lib.slosh_last_error(ctx, buf, 512)
        raise SloshError(code, buf.value.decode(errors="replace"))


class MpmData:
    """GPU-resident state of one scene: particles, sparse grid, bodies.

    Mirrors ``MpmData::new(backend, params, particles, bodies, colliders,
    materials, cell_width, grid_capacity)`` (src/pipeline.rs:311)."""

    def __init__(
        self,
        params: SimulationParams,
        particles: np.ndarray,
        bodies: Iterable[RigidBody] = (),
        cell_width: float = 1.0,
        grid_capacity: int = 30_000,
        dim: int = 3,
        device: int = 0,
        max_particles: int | None = None,
    ):
        self._lib = _lib.load()
        self.dim = dim
        self.cell_width = float(cell_width)
        self.params = params
        cfg = SloshConfig(dim, float(cell_width), int(grid_capacity), int(max_particles or max(len(particles), 1)), device, 0)
        ctx = ctypes.c_void_p()
        code = self._lib.slosh_ctx_create(ctypes.byref(cfg), ctypes.byref(ctx))
        if code != 0:
            raise SloshError(code, "slosh_ctx_create failed")
        self._ctx = ctx
        self.set_params(params)
        self.set_bodies(list(bodies))
        self.upload(particles)

    @staticmethod
    def new(params, particles, bodies=(), cell_width=1.0, grid_capacity=30_000, dim=3, device=0) -> "MpmData":
        return MpmData(params, particles, bodies, cell_width, grid_capacity, dim, device)

    # -- state -----------------------------------------------------------------
    def set_params(self, params: SimulationParams):
        g = list(params.gravity) + [0.0] * (3 - len(params.gravity))
        p = SloshParams((ctypes.c_float * 3)(*g[:3]), float(params.dt))
        _check(self._lib, self._ctx, self._lib.slosh_set_params(self._ctx, ctypes.byref(p)))
        self.params = params

    def set_bodies(self, bodies: list):
        self.bodies = bodies
        recs = np.zeros(len(bodies), dtype=BODY_DTYPE)
        if not hasattr(self, "_meshes"):
            self._meshes = {}  # id of a trimesh shape's vertex array -> its (shape_a, shape_b)
        for i, b in enumerate(bodies):
            recs[i] = b.record(self.dim)
            if b.shape[0] == "trimesh":
                key = id(b.shape[1][0])
                if key not in self._meshes:
                    v, t = mesh_arrays(b.shape)
                    tmp = np.zeros(1, dtype=BODY_DTYPE)
                    _check(self._lib, self._ctx,
                           self._lib.slosh_add_trimesh(self._ctx, ptr(v), len(v), ptr(t), len(t), ptr(tmp)))
                    self._meshes[key] = (tmp["shape_a"][0].copy(), tmp["shape_b"][0].copy(), b.shape[1])
                recs[i]["shape_a"], recs[i]["shape_b"] = self._meshes[key][0], self._meshes[key][1]
        self.n_bodies = len(bodies)
        _check(self._lib, self._ctx, self._lib.slosh_set_bodies(self._ctx, ptr(recs) if len(bodies) else None, len(bodies)))

    def upload(self, particles: np.ndarray, stream=None):
        particles = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self.n = len(particles)
        _check(
            self._lib,
            self._ctx,
            self._lib.slosh_upload_particles(self._ctx, ptr(particles), self.n, stream),
        )

    def append(self, particles: np.ndarray, stream=None):
        """``GpuParticles::append`` (src/solver/particle.rs:536-572)."""
        particles = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        _check(self._lib, self._ctx, self._lib.slosh_append_particles(self._ctx, ptr(particles), len(particles), stream))
        self.n += len(particles)

    def shift_remove(self, start: int, end: int, stream=None) -> int:
        """``GpuParticles::shift_remove`` of the insertion-order range
        [start, end) (src/solver/particle.rs:505-534); returns the number
        removed."""
        removed = ctypes.c_uint32(0)
        count = max(int(end) - int(start), 0)
        _check(
            self._lib,
            self._ctx,
            self._lib.slosh_remove_particles(self._ctx, int(start), count, ctypes.byref(removed), stream),
        )
        self.n -= removed.value
        return removed.value

    def download_particles(self, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.n, dtype=PARTICLE_DTYPE)
        _check(self._lib, self._ctx, self._lib.slosh_download_particles(self._ctx, ptr(out), self.n, stream))
        return out

    def positions(self, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        if out is None:
            out = np.zeros((self.n, 4), dtype=np.float32)
        _check(self._lib, self._ctx, self._lib.slosh_download_positions(self._ctx, ptr(out), self.n, stream))
        return out

    def get_bodies(self) -> np.ndarray:
        out = np.zeros(self.n_bodies, dtype=BODY_DTYPE)
        if self.n_bodies:
            _check(self._lib, self._ctx, self._lib.slosh_get_bodies(self._ctx, ptr(out), self.n_bodies))
        return out

    def sync(self, stream=None):
        _check(self._lib, self._ctx, self._lib.slosh_sync(self._ctx, stream))

    def timestep_bound(self, stream=None) -> float:
        """Largest stable dt of the current particles (seconds), as
        ``WgTimestepBounds::compute_bounds`` (src/solver/timestep_bound.rs:58-81)."""
        dt = ctypes.c_float()
        _check(self._lib, self._ctx, self._lib.slosh_timestep_bound(self._ctx, ctypes.byref(dt), stream))
        return float(dt.value)

    @property
    def kernels_per_substep(self) -> int:
        return int(self._lib.slosh_kernels_per_substep(self._ctx))

    def stats(self) -> dict:
        raw = np.zeros(8, np.uint32)
        _check(self._lib, self._ctx, self._lib.slosh_get_stats(self._ctx, ptr(raw)))
        keys = ("n_particles", "n_blocks", "n_primary_blocks", "n_materials", "n_svd_fp64", "n_grid_rebuilds",
                "n_grid_reuses", "conditional_graphs")
        return {k: int(raw[i]) for i, k in enumerate(keys)}

    def profile_substeps(self, n_substeps: int, stream=None) -> dict:
        """Per-kernel device milliseconds summed over `n_substeps` substeps
        (CUDA events around every launch; advances the simulation)."""
        ms = np.zeros(32, np.float32)
        nk = ctypes.c_uint32(0)
        _check(
            self._lib,
            self._ctx,
            self._lib.slosh_profile_substeps(self._ctx, int(n_substeps), stream, ptr(ms), 32, ctypes.byref(nk)),
        )
        out = {}
        buf = ctypes.create_string_buffer(64)
        for k in range(nk.value):
            self._lib.slosh_kernel_name(k, buf, 64)
            out[buf.value.decode()] = float(ms[k])
        return out

    # -- debug views -------------------------------------------------------------
    def grid_debug(self) -> dict:
        d = SloshGridDump()
        _check(self._lib, self._ctx, self._lib.slosh_grid_debug(self._ctx, ctypes.byref(d), 0, 0))
        nb, ns, NB, NN = d.n_blocks, d.n_sorted, d.nb_buckets, d.n_neighbors
        out = {
            "keys": np.zeros(nb, np.uint32),
            "first_particle": np.zeros(nb, np.uint32),
            "num_particles": np.zeros(nb, np.uint32),
            "num_particles_with_extras": np.zeros(nb, np.uint32),
            "bucket_counts": np.zeros(nb * NB, np.uint32),
            "sorted_ids": np.zeros(ns, np.uint32),
            "primary_first": np.zeros(nb, np.uint32),
            "primary_perm": np.zeros(self.n, np.uint32),
            "neighbors": np.zeros(nb * NN, np.uint32),
        }
        d2 = SloshGridDump()
        for name, arr in out.items():
            setattr(d2, name, arr.ctypes.data if arr.size else None)
        _check(self._lib, self._ctx, self._lib.slosh_grid_debug(self._ctx, ctypes.byref(d2), nb, ns))
        out["bucket_counts"] = out["bucket_counts"].reshape(nb, NB)
        out["neighbors"] = out["neighbors"].reshape(nb, NN)
        return out

    def debug_nodes(self, stage: int) -> np.ndarray:
        nb = ctypes.c_uint32(0)
        _check(self._lib, self._ctx, self._lib.slosh_debug_nodes(self._ctx, stage, None, 0, ctypes.byref(nb)))
        out = np.zeros((nb.value * 64, 4), np.float32)
        _check(self._lib, self._ctx, self._lib.slosh_debug_nodes(self._ctx, stage, ptr(out), nb.value, ctypes.byref(nb)))
        return out

    def device_view(self) -> "_lib.SloshDeviceView":
        """The device buffers of the substep a stage hook runs in (only
        inside a hook)."""
        v = _lib.SloshDeviceView()
        _check(self._lib, self._ctx, self._lib.slosh_device_view_get(self._ctx, ctypes.byref(v)))
        return v

    def enqueue_builtin(self, point: int, stream) -> None:
        """The built-in stage a run hook replaces (only inside that hook)."""
        _check(self._lib, self._ctx, self._lib.slosh_enqueue_builtin(self._ctx, int(point), stream))

    def prefix_sum(self, values: np.ndarray) -> np.ndarray:
        v = np.ascontiguousarray(values, dtype=np.uint32)
        out = np.zeros_like(v)
        _check(self._lib, self._ctx, self._lib.slosh_prefix_sum(self._ctx, ptr(v), ptr(out), len(v)))
        return out

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.slosh_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MpmPipelineHooks:
    """``MpmPipelineHooks`` (src/pipeline.rs:146-238): override the stages
    to hook.  Each method gets the scene, the CUDA stream of the substep (an
    int handle; work enqueued on it runs in order with the substep) and the
    caller's state object.  ``run_p2g`` / ``run_g2p`` return True when they
    replaced the built-in stage (``data.enqueue_builtin`` runs it from inside
    the hook); the ``after_*`` methods return None.  ``data.device_view()``
    gives the substep's device buffers inside a hook."""

    def after_particle_sort(self, data, stream, state):
        return None

    def run_p2g(self, data, stream, state) -> bool:
        return False

    def after_p2g(self, data, stream, state):
        return None

    def after_grid_update(self, data, stream, state):
        return None

    def run_g2p(self, data, stream, state) -> bool:
        return False

    def after_g2p(self, data, stream, state):
        return None

    def after_particles_update(self, data, stream, state):
        return None


class MpmPipeline:
    """``MpmPipeline::launch_step``: enqueues substeps on the GPU.

    Without hooks the whole substep is one CUDA graph; no host round trip
    happens inside ``launch_step``.  Device-side errors (block capacity
    overflow) surface at the next ``MpmData.sync()`` or download.  With
    hooks (an ``MpmPipelineHooks`` whose methods are overridden), the
    substep's kernels are launched one by one and each overridden method is
    called at its point of every substep."""

    def __init__(self):
        self._lib = _lib.load()

    def launch_step(self, data: MpmData, n_substeps: int = 1, stream=None, hooks=None, hooks_state=None):
        if hooks is None:
            _check(self._lib, data._ctx, self._lib.slosh_step(data._ctx, int(n_substeps), stream))
            return
        callbacks, errors = [], []
        base = MpmPipelineHooks
        for point, name in enumerate(_lib.HOOK_NAMES):
            method = getattr(type(hooks), name, None)
            if method is None or method is getattr(base, name):
                continue

            def call(ctx, pt, st, user, _name=name):
                try:
                    r = getattr(hooks, _name)(data, st or 0, hooks_state)
                    return 1 if r is True else 0
                except Exception as e:  # reported after slosh_step returns
                    errors.append(e)
                    return _lib.SLOSH_E_STATE

            cb = _lib.HOOK_FN(call)
            callbacks.append(cb)
            _check(self._lib, data._ctx, self._lib.slosh_set_hook(data._ctx, point, cb, None))
        try:
            code = self._lib.slosh_step(data._ctx, int(n_substeps), stream)
        finally:
            for point in range(len(_lib.HOOK_NAMES)):
                self._lib.slosh_set_hook(data._ctx, point, _lib.HOOK_FN(), None)
        if errors:
            raise errors[0]
        _check(self._lib, data._ctx, code)

    def compute_timestep_bound(self, data: MpmData, stream=None) -> float:
        """``pipeline.timestep_bounds.compute_bounds`` (src/solver/timestep_bound.rs:58-81)."""
        return data.timestep_bound(stream)


def adaptive_substeps(base_dt: float, bound: float, min_substeps: int, max_substeps: int) -> int:
    """Number of substeps per frame of the testbed's adaptive stepping
    (src_testbed/step.rs:104-134): ceil(base_dt / bound) clamped to
    [min_substeps, max_substeps]; each substep then uses base_dt / n."""
    est = math.ceil(base_dt / bound) if bound > 0 else max_substeps
    return int(min(max(est, min_substeps), max_substeps))
