"""Multi-scene batches: many independent scenes advanced by one set of
kernel launches per substep (``slosh_batch_*`` in include/slosh_b200.h).

Stepping a batch by k substeps is equivalent to calling
``MpmPipeline::launch_step`` (src/pipeline.rs:562-770) k times on each
scene's own ``MpmData``; each scene keeps its own cell width, dt, gravity and
colliders.  A scene's results do not depend on the other scenes of the batch
(bit for bit), so scenes can join and leave between steps (continuous
batching).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (
    BODY_DTYPE,
    PARTICLE_DTYPE,
    SloshBatchConfig,
    SloshBatchStats,
    SloshError,
    SloshParams,
    SloshSceneDesc,
    SloshTuning,
    ptr,
)


def _check(lib, b, code: int):
    if code != 0:
        buf = ctypes.create_string_buffer(512)
        if b:
            lib.slosh_batch_last_error(b, buf, 512)
        raise SloshError(code, buf.value.decode(errors="replace"))


class MpmBatch:
    def __init__(
        self,
        dim: int = 3,
        max_particles: int = 1 << 22,
        grid_capacity: int = 1 << 16,
        max_scenes: int = 1024,
        max_bodies: int = 4096,
        device: int = 0,
    ):
        self._lib = _lib.load()
        self.dim = dim
        cfg = SloshBatchConfig(dim, int(max_particles), int(grid_capacity), int(max_scenes), int(max_bodies), device, 0)
        h = ctypes.c_void_p()
        code = self._lib.slosh_batch_create(ctypes.byref(cfg), ctypes.byref(h))
        if code != 0:
            raise SloshError(code, "slosh_batch_create failed")
        self._b = h
        self.sizes: dict[int, int] = {}
        self.n_bodies: dict[int, int] = {}

    # -- scenes ------------------------------------------------------------------
    def add_scene(self, particles: np.ndarray, cell_width: float, params, bodies=(), stream=None) -> int:
        """Adds a scene (records as for MpmData.upload) and returns its slot."""
        particles = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        bodies = list(bodies)
        recs = np.zeros(len(bodies), dtype=BODY_DTYPE)
        for i, b in enumerate(bodies):
            recs[i] = b.record(self.dim)
        g = list(params.gravity) + [0.0] * (3 - len(params.gravity))
        desc = SloshSceneDesc(float(cell_width), SloshParams((ctypes.c_float * 3)(*g[:3]), float(params.dt)))
        slot = ctypes.c_uint32()
        _check(
            self._lib,
            self._b,
            self._lib.slosh_batch_add_scene(
                self._b,
                ctypes.byref(desc),
                ptr(particles),
                len(particles),
                ptr(recs) if len(bodies) else None,
                len(bodies),
                ctypes.byref(slot),
                stream,
            ),
        )
        self.sizes[slot.value] = len(particles)
        self.n_bodies[slot.value] = len(bodies)
        return slot.value

    def add(self, scene, stream=None) -> int:
        """Adds a :class:`slosh_b200.scenes.Scene`."""
        return self.add_scene(scene.particles, scene.cell_width, scene.params, scene.bodies, stream)

    def remove_scene(self, slot: int):
        _check(self._lib, self._b, self._lib.slosh_batch_remove_scene(self._b, slot))
        self.sizes.pop(slot, None)
        self.n_bodies.pop(slot, None)

    # -- stepping ----------------------------------------------------------------
    def step(self, n_substeps: int, stream=None):
        _check(self._lib, self._b, self._lib.slosh_batch_step(self._b, int(n_substeps), stream))

    def sync(self, stream=None):
        _check(self._lib, self._b, self._lib.slosh_batch_sync(self._b, stream))

    # -- results -----------------------------------------------------------------
    def positions(self, slot: int, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        n = self.sizes[slot]
        if out is None:
            out = np.empty((n, 4), np.float32)
        _check(self._lib, self._b, self._lib.slosh_batch_download_positions(self._b, slot, ptr(out), n, stream))
        return out

    def download_particles(self, slot: int, stream=None) -> np.ndarray:
        n = self.sizes[slot]
        out = np.empty(n, PARTICLE_DTYPE)
        _check(self._lib, self._b, self._lib.slosh_batch_download_particles(self._b, slot, ptr(out), n, stream))
        return out

    def get_bodies(self, slot: int) -> np.ndarray:
        n = self.n_bodies[slot]
        out = np.zeros(n, BODY_DTYPE)
        _check(self._lib, self._b, self._lib.slosh_batch_get_bodies(self._b, slot, ptr(out) if n else None, n))
        return out

    def timestep_bound(self, slot: int, stream=None) -> float:
        """Largest stable dt of one scene (as MpmData.timestep_bound)."""
        dt = ctypes.c_float()
        _check(self._lib, self._b, self._lib.slosh_batch_timestep_bound(self._b, slot, ctypes.byref(dt), stream))
        return float(dt.value)

    def stats(self) -> dict:
        st = SloshBatchStats()
        _check(self._lib, self._b, self._lib.slosh_batch_get_stats(self._b, ctypes.byref(st)))
        return {
            "live_scenes": st.live_scenes,
            "n_particles": st.n_particles,
            "n_blocks": st.n_blocks,
            "n_materials": st.n_materials,
            "n_svd_fp64": st.n_svd_fp64,
            "n_bodies": st.n_bodies,
            "fused_graph": st.fused_graph,
            "g2p_launches": st.g2p_launches,
            "tuning": {
                "p2g_ctas_per_sm": st.tuning.p2g_ctas_per_sm,
                "g2p_threads": st.tuning.g2p_threads,
                "g2p_ctas_per_sm": st.tuning.g2p_ctas_per_sm,
                "p2g_stages": st.tuning.p2g_stages,
                "fused": st.tuning.fused,
            },
        }

    # -- launch shape --------------------------------------------------------------
    def autotune(self, substeps: int = 2, stream=None) -> dict:
        _check(self._lib, self._b, self._lib.slosh_batch_autotune(self._b, int(substeps), stream))
        return self.stats()["tuning"]

    def set_tuning(self, p2g_ctas_per_sm: int, g2p_threads: int, g2p_ctas_per_sm: int, p2g_stages: int = 3,
                   fused: int = 0):
        """Launch shape of the batched substep; ``fused=1`` runs each substep
        as one persistent cooperative kernel (the shape fields are then
        unused).  Results do not depend on the choice."""
        t = SloshTuning(p2g_ctas_per_sm, g2p_threads, g2p_ctas_per_sm, p2g_stages, fused)
        _check(self._lib, self._b, self._lib.slosh_batch_set_tuning(self._b, ctypes.byref(t)))

    def close(self):
        if self._b:
            self._lib.slosh_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
