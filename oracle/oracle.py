"""TEST INFRASTRUCTURE — ctypes wrapper of the oracle (``liboracle.so``).

The oracle is the CPU restatement of slosh's MPM substep used as the parity
checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.  It
is never part of the product path.  Its record layouts are the C structs of
include/slosh_b200.h.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import LIB, build_oracle

PARTICLE_DTYPE = np.dtype(
    [
        ("position", "<f4", 3),
        ("velocity", "<f4", 3),
        ("def_grad", "<f4", 9),
        ("affine", "<f4", 9),
        ("force_dt", "<f4", 3),
        ("vel_grad_det", "<f4"),
        ("init_volume", "<f4"),
        ("init_radius", "<f4"),
        ("mass", "<f4"),
        ("damping", "<f4"),
        ("phase", "<f4"),
        ("enabled", "<u4"),
        ("fixed", "<u4"),
        ("model_tag", "<u4"),
        ("model", "<f4", 12),
    ]
)
BODY_ITEMSIZE = 192

_lib = None
_P = ctypes.c_void_p


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build_oracle()
        lib = ctypes.CDLL(LIB)
        sigs = {
            "orc_create": (_P, [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_uint32]),
            "orc_destroy": (None, [_P]),
            "orc_set_params": (None, [_P, _P, ctypes.c_float]),
            "orc_set_particles": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
            "orc_get_particles": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
            "orc_set_bodies": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
            "orc_get_bodies": (ctypes.c_int, [_P, _P, ctypes.c_uint32]),
            "orc_step": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_int]),
            "orc_stages": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int]),
            "orc_num_blocks": (ctypes.c_uint32, [_P]),
            "orc_num_sorted": (ctypes.c_uint32, [_P]),
            "orc_grid_get": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
            "orc_nodes_get": (ctypes.c_int, [_P, _P]),
            "orc_totals": (None, [_P, _P]),
            "orc_node_totals": (None, [_P, _P]),
            "orc_prefix_sum": (None, [_P, ctypes.c_uint32]),
            "orc_svd": (None, [ctypes.c_uint32, _P, _P, _P, _P]),
            "orc_model_stress": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P]),
            "orc_timestep_bound": (ctypes.c_uint32, [_P]),
            "orc_project": (ctypes.c_int, [ctypes.c_uint32, _P, _P, _P, _P]),
            "orc_add_trimesh": (ctypes.c_int, [_P, _P, ctypes.c_uint32, _P, ctypes.c_uint32]),
            "orc_project_trimesh": (
                ctypes.c_int,
                [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P, ctypes.c_float, _P, _P],
            ),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else None


def project_on_boundary(dim: int, body_record, point) -> tuple[np.ndarray, bool] | None:
    """Shape::project_point_on_boundary of one body record (FP32); None
    when the shape is not supported in `dim`."""
    lib = load()
    rec = np.ascontiguousarray(np.asarray(body_record).reshape(1))
    pt = np.zeros(3, np.float32)
    pt[:dim] = np.asarray(point, np.float32)[:dim]
    out = np.zeros(3, np.float32)
    inside = ctypes.c_int(0)
    ok = lib.orc_project(dim, _p(rec), _p(pt), _p(out), ctypes.byref(inside))
    return (out[:dim].copy(), bool(inside.value)) if ok else None


def project_on_trimesh(vertices, triangles, body_record, point, cap: float):
    """Closest point on a posed triangle mesh within `cap` and the inside
    flag (FP64 scan of all triangles), or None."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
    rec = np.ascontiguousarray(body_record)
    pt = np.zeros(3, np.float32)
    pt[: len(point)] = point
    out = np.zeros(3, np.float32)
    inside = ctypes.c_int(0)
    ok = load().orc_project_trimesh(_p(v), len(v), _p(t), len(t), _p(rec), _p(pt), float(cap), _p(out), ctypes.byref(inside))
    return (out, bool(inside.value)) if ok else None


def prefix_sum(values) -> np.ndarray:
    """WgPrefixSum::eval_cpu restated (src/grid/prefix_sum.rs:97-110)."""
    v = np.array(values, dtype=np.uint32, copy=True)
    load().orc_prefix_sum(_p(v), len(v))
    return v


def svd(F: np.ndarray):
    F = np.ascontiguousarray(F, dtype=np.float64)
    d = F.shape[0]
    U = np.zeros((d, d))
    V = np.zeros((d, d))
    S = np.zeros(d)
    load().orc_svd(d, _p(F), _p(U), _p(S), _p(V))
    return U, S, V


def model_stress(tag: int, model: np.ndarray, F: np.ndarray):
    """Kirchhoff stress of one 3D model in FP64 (returns tau, F', model')."""
    m = np.array(model, dtype=np.float64, copy=True)
    f = np.array(F, dtype=np.float64, copy=True).reshape(9)
    tau = np.zeros(9)
    code = load().orc_model_stress(3, tag, _p(m), _p(f), _p(tau))
    assert code == 0
    return tau.reshape(3, 3), f.reshape(3, 3), m


class Oracle:
    """One oracle scene (FP32 or FP64)."""

    def __init__(self, dim: int, cell_width: float, grid_capacity: int, double: bool = False, threads: int = 0):
        self.lib = load()
        self.dim = dim
        self.ctx = self.lib.orc_create(dim, 1 if double else 0, cell_width, grid_capacity)
        self.threads = threads or (os.cpu_count() or 1)
        self.n = 0

    def set_params(self, gravity, dt):
        g = np.zeros(3, np.float32)
        g[: len(gravity)] = gravity
        self.lib.orc_set_params(self.ctx, _p(g), float(dt))

    def set_particles(self, recs: np.ndarray):
        recs = np.ascontiguousarray(recs)
        assert recs.dtype.itemsize == 192
        self.n = len(recs)
        assert self.lib.orc_set_particles(self.ctx, _p(recs), self.n) == 0

    def set_bodies(self, recs: np.ndarray, bodies=None):
        """`bodies`: the RigidBody objects of the records, whose triangle
        meshes are added here (each record then names its mesh by ordinal)."""
        recs = np.array(recs, copy=True)
        if bodies is not None:
            if not hasattr(self, "_meshes"):
                self._meshes = {}
            for i, b in enumerate(bodies):
                if b.shape[0] != "trimesh":
                    continue
                key = id(b.shape[1][0])
                if key not in self._meshes:
                    v = np.ascontiguousarray(b.shape[1][0], np.float32).reshape(-1, 3)
                    t = np.ascontiguousarray(b.shape[1][1], np.uint32).reshape(-1, 3)
                    ordinal = self.lib.orc_add_trimesh(self.ctx, _p(v), len(v), _p(t), len(t))
                    assert ordinal >= 0
                    self._meshes[key] = (ordinal, b.shape[1])
                recs[i]["shape_b"].view(np.uint32)[2] = self._meshes[key][0]
        recs = np.ascontiguousarray(recs)
        assert recs.dtype.itemsize == BODY_ITEMSIZE
        assert self.lib.orc_set_bodies(self.ctx, _p(recs) if len(recs) else None, len(recs)) == 0
        self.body_dtype = recs.dtype
        self.n_bodies = len(recs)

    def get_particles(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=PARTICLE_DTYPE)
        self.lib.orc_get_particles(self.ctx, _p(out), self.n)
        return out

    def get_bodies(self) -> np.ndarray:
        out = np.zeros(self.n_bodies, dtype=self.body_dtype)
        if self.n_bodies:
            self.lib.orc_get_bodies(self.ctx, _p(out), self.n_bodies)
        return out

    def step(self, n: int = 1):
        code = self.lib.orc_step(self.ctx, n, self.threads)
        if code != 0:
            raise RuntimeError(f"oracle step failed: {code}")

    def stages(self, last: int):
        code = self.lib.orc_stages(self.ctx, last, self.threads)
        if code != 0:
            raise RuntimeError(f"oracle stages failed: {code}")

    def grid(self) -> dict:
        """Grid of the last `stages()` call in slosh's layout."""
        self.stages(0)
        nb = self.lib.orc_num_blocks(self.ctx)
        ns = self.lib.orc_num_sorted(self.ctx)
        NB = 10 if self.dim == 3 else 18
        out = {
            "keys": np.zeros(nb, np.uint32),
            "first_particle": np.zeros(nb, np.uint32),
            "num_particles": np.zeros(nb, np.uint32),
            "num_particles_with_extras": np.zeros(nb, np.uint32),
            "bucket_counts": np.zeros(nb * NB, np.uint32),
            "sorted_ids": np.zeros(ns, np.uint32),
        }
        self.lib.orc_grid_get(
            self.ctx,
            _p(out["keys"]),
            _p(out["first_particle"]),
            _p(out["num_particles"]),
            _p(out["num_particles_with_extras"]),
            _p(out["bucket_counts"]),
            _p(out["sorted_ids"]),
        )
        out["bucket_counts"] = out["bucket_counts"].reshape(nb, NB)
        return out

    def nodes(self, stage: int) -> np.ndarray:
        self.stages(stage)
        nb = self.lib.orc_num_blocks(self.ctx)
        out = np.zeros((nb * 64, 4), np.float32)
        self.lib.orc_nodes_get(self.ctx, _p(out))
        return out

    def node_totals(self, stage: int) -> np.ndarray:
        """Sums (momentum xyz, mass) over the nodes after `stage`, in double."""
        self.stages(stage)
        out = np.zeros(4)
        self.lib.orc_node_totals(self.ctx, _p(out))
        return out

    def totals(self) -> np.ndarray:
        out = np.zeros(4)
        self.lib.orc_totals(self.ctx, _p(out))
        return out

    def timestep_bound(self) -> tuple[int, float]:
        """(picosecond count, seconds as f32) of estimate_timestep_bound
        (shaders/slosh/solver/timestep_bound.slang:37-91)."""
        u = int(self.lib.orc_timestep_bound(self.ctx))
        return u, float(np.float32(u) / np.float32(1.0e12))

    def close(self):
        if self.ctx:
            self.lib.orc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def from_scene(scene, double: bool = False, threads: int = 0) -> Oracle:
    o = Oracle(scene.dim, scene.cell_width, scene.grid_capacity, double=double, threads=threads)
    o.set_params(scene.params.gravity, scene.params.dt)
    from slosh_b200._lib import BODY_DTYPE

    recs = np.zeros(len(scene.bodies), dtype=BODY_DTYPE)
    for i, b in enumerate(scene.bodies):
        recs[i] = b.record(scene.dim)
    o.set_bodies(recs, scene.bodies)
    o.set_particles(scene.particles)
    return o
