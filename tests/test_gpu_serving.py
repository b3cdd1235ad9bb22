"""The serving loop (slosh_server_* C ABI) on the GPU: every request gets
exactly its own substep count, and its result is bit-identical to the same
scene advanced alone, whatever else is in flight."""
import time

import numpy as np
import pytest

from slosh_b200 import scenes
from slosh_b200._lib import SLOSH_E_CAPACITY, SloshError
from slosh_b200.batch import MpmBatch
from slosh_b200.serving import MpmServer

pytestmark = pytest.mark.gpu


def alone(sc, substeps):
    b = MpmBatch(3, max_particles=1 << 16, grid_capacity=1 << 12, max_scenes=4, max_bodies=16)
    s = b.add(sc)
    b.step(substeps)
    out = b.positions(s)
    b.close()
    return out


def test_served_results_equal_alone(cuda_lib):
    reqs = [
        (scenes.random_scene_3d(5000, "sand", 1 / 64, seed=41), 37),
        (scenes.random_scene_3d(9000, "elastic", 1 / 128, seed=42), 15),
        (scenes.random_scene_3d(3000, "fluid", 1 / 64, seed=43), 52),
        (scenes.random_scene_3d(7000, "sand", 1 / 128, seed=44), 23),
        (scenes.random_scene_3d(4000, "fluid", 1 / 128, seed=45), 9),
    ]
    srv = MpmServer(2 << 30, max_scenes=8, tick_substeps=10)
    outs = {}
    for k, (sc, sub) in enumerate(reqs):
        rid, out = srv.submit(sc.particles, sc.cell_width, sc.params, sc.bodies, sub)
        outs[rid] = (k, out)
        time.sleep(0.01 * k)  # staggered arrivals: requests join a running batch
    srv.wait_idle(120)
    done = srv.poll()
    st = srv.stats()
    srv.close()
    assert len(done) == len(reqs) and all(d["status"] == 0 for d in done)
    assert st["completed"] == len(reqs)
    assert st["particle_substeps"] == sum(sc.n * s for sc, s in reqs)
    for d in done:
        k, out = outs[d["id"]]
        sc, sub = reqs[k]
        assert d["substeps"] == sub and d["submit_s"] <= d["admit_s"] <= d["done_s"]
        assert np.array_equal(out, alone(sc, sub)), f"request {k}"


def test_server_rejects_oversized_request(cuda_lib):
    srv = MpmServer(256 << 20, max_scenes=4)
    big = scenes.random_scene_3d(800000, "fluid", 1 / 128, seed=46)
    with pytest.raises(SloshError) as e:
        srv.submit_scene(big, 10)
    assert e.value.code == SLOSH_E_CAPACITY
    srv.close()
