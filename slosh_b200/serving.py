"""Serving loop (``slosh_server_*`` in include/slosh_b200.h): requests of
(scene, substeps) admitted by device footprint, advanced together by a
worker thread with continuous batching, retired with their final positions.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (
    BODY_DTYPE,
    PARTICLE_DTYPE,
    SloshCompletion,
    SloshError,
    SloshParams,
    SloshRequest,
    SloshSceneDesc,
    SloshServerConfig,
    SloshServerStats,
)


def _check(lib, s, code: int):
    if code != 0:
        buf = ctypes.create_string_buffer(512)
        if s:
            lib.slosh_server_last_error(s, buf, 512)
        raise SloshError(code, buf.value.decode(errors="replace"))


class MpmServer:
    def __init__(
        self,
        hbm_budget_bytes: int,
        dim: int = 3,
        max_scenes: int = 1024,
        max_bodies: int = 4096,
        tick_substeps: int = 100,
        max_in_flight: int = 0,
        autotune: bool = True,
        device: int = 0,
    ):
        self._lib = _lib.load()
        self.dim = dim
        cfg = SloshServerConfig(
            dim, device, int(hbm_budget_bytes), max_scenes, max_bodies, tick_substeps, max_in_flight, int(autotune), 0
        )
        h = ctypes.c_void_p()
        code = self._lib.slosh_server_create(ctypes.byref(cfg), ctypes.byref(h))
        if code != 0:
            raise SloshError(code, "slosh_server_create failed")
        self._s = h
        self._keep: dict[int, tuple] = {}  # arrays the worker reads or writes until completion

    def submit(self, particles: np.ndarray, cell_width: float, params, bodies=(), substeps: int = 1):
        """Queues a scene; returns (request id, positions array filled at completion)."""
        particles = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        bodies = list(bodies)
        recs = np.zeros(len(bodies), dtype=BODY_DTYPE)
        for i, b in enumerate(bodies):
            recs[i] = b.record(self.dim)
        out = np.zeros((len(particles), 4), np.float32)
        g = list(params.gravity) + [0.0] * (3 - len(params.gravity))
        desc = SloshSceneDesc(float(cell_width), SloshParams((ctypes.c_float * 3)(*g[:3]), float(params.dt)))
        req = SloshRequest(
            desc,
            len(particles),
            len(bodies),
            int(substeps),
            0,
            particles.ctypes.data,
            recs.ctypes.data if len(bodies) else None,
            out.ctypes.data,
        )
        rid = ctypes.c_uint64()
        _check(self._lib, self._s, self._lib.slosh_server_submit(self._s, ctypes.byref(req), ctypes.byref(rid)))
        self._keep[rid.value] = (particles, recs, out)
        return rid.value, out

    def submit_scene(self, scene, substeps: int | None = None):
        return self.submit(scene.particles, scene.cell_width, scene.params, scene.bodies, substeps or scene.substeps)

    def poll(self, cap: int = 1024) -> list[dict]:
        buf = (SloshCompletion * cap)()
        n = ctypes.c_uint32()
        _check(self._lib, self._s, self._lib.slosh_server_poll(self._s, buf, cap, ctypes.byref(n)))
        res = []
        for k in range(n.value):
            c = buf[k]
            keep = self._keep.pop(c.id, None)
            res.append(
                {
                    "id": c.id,
                    "status": c.status,
                    "n": c.n,
                    "substeps": c.substeps,
                    "submit_s": c.submit_s,
                    "admit_s": c.admit_s,
                    "done_s": c.done_s,
                    "positions": keep[2] if keep else None,
                }
            )
        return res

    def wait_idle(self, timeout_s: float = 600.0):
        _check(self._lib, self._s, self._lib.slosh_server_wait_idle(self._s, float(timeout_s)))

    def stats(self) -> dict:
        st = SloshServerStats()
        _check(self._lib, self._s, self._lib.slosh_server_get_stats(self._s, ctypes.byref(st)))
        out = {k: getattr(st, k) for k, _ in SloshServerStats._fields_ if k not in ("pad", "tuning")}
        out["tuning"] = {k: getattr(st.tuning, k) for k, _ in st.tuning._fields_}
        return out

    def close(self):
        if self._s:
            self._lib.slosh_server_destroy(self._s)
            self._s = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
