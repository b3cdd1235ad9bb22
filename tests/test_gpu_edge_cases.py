"""Edge cases of the substep on the GPU, against the oracle.

- one particle alone (one primary block, its +1 neighbours);
- many particles in one cell (more than a warp: the canonical order of a
  crowded cell is fixed by the one-lane insertion sort, and P2G's cell loop
  runs long);
- disabled particles mixed with enabled ones (mass 0, kept in storage);
- far-apart clusters at negative coordinates (blocks with no neighbours in
  common, keys on both sides of the packed-key origin).

Grid layout bit-exact at upload and after the substeps; particle state
within the FP32 tolerance of the single-scene parity tests.
"""
import numpy as np
import pytest

from oracle import oracle as O
from slosh_b200 import scenes
from slosh_b200.pipeline import MpmPipeline, ParticleModel, RigidBody, SimulationParams, make_particles

pytestmark = pytest.mark.gpu

H = 1.0 / 64.0
DT = 1.0e-4


def close(name, got, exp, atol, rtol):
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    err = np.abs(got - exp).max() if got.size else 0.0
    bound = atol + rtol * (np.abs(exp).max() if exp.size else 0.0)
    print(f"{name}: max err {err:.3e} bound {bound:.3e}")
    assert err <= bound, f"{name}: max err {err:.3e} > {bound:.3e}"


def grid_equal(gpu, orc):
    for k in ("keys", "first_particle", "num_particles", "num_particles_with_extras", "sorted_ids"):
        assert np.array_equal(gpu[k], orc[k]), k
    assert np.array_equal(gpu["bucket_counts"], orc["bucket_counts"])


def scene(name, pts, model, density=1000.0, vel=None, floor=True):
    parts = make_particles(pts, H / 4, density, model, dim=3, velocities=vel)
    bodies = []
    if floor:
        t = 4.0 * H
        bodies = [RigidBody(("cuboid", (4.0, t, 4.0)), translation=(0.5, 0.05 - t, 0.5))]
    return scenes.Scene(name, 3, H, SimulationParams(dt=DT), parts, bodies, 10, 1 << 12)


def run(sc, steps, loose=1.0):
    data = scenes.build_mpm_data(sc)
    orc = O.from_scene(sc, threads=8)
    grid_equal(data.grid_debug(), orc.grid())
    MpmPipeline().launch_step(data, steps)
    orc.step(steps)
    g, o = data.download_particles(), orc.get_particles()
    assert np.array_equal(g["enabled"], o["enabled"])
    close(f"{sc.name} position", g["position"], o["position"], 2e-6 * loose, 0)
    close(f"{sc.name} velocity", g["velocity"], o["velocity"], 1e-6 * loose, 1e-4 * loose)
    close(f"{sc.name} def_grad", g["def_grad"], o["def_grad"], 2e-6 * loose, 2e-6 * loose)
    close(f"{sc.name} mass", g["mass"], o["mass"], 0, 0)
    orc.set_particles(g)
    grid_equal(data.grid_debug(), orc.grid())
    data.close()
    return g


def test_single_particle(cuda_lib):
    sc = scene("one", np.array([[0.5, 0.3, 0.5]]), ParticleModel.elastic(1.0e5, 0.3))
    g = run(sc, 5)
    # free fall: v_y = -g t (the particle never meets the floor)
    assert abs(float(g["velocity"][0, 1]) + 9.81 * 5 * DT) <= 1e-5


@pytest.mark.parametrize("model", ["sand", "fluid"])
def test_crowded_cell(cuda_lib, model):
    """300 particles inside one cell, beside an ordinary lattice blob."""
    rng = np.random.default_rng(7)
    c = np.array([0.5 + 0.5 * H, 0.2 + 0.5 * H, 0.5 + 0.5 * H])  # a cell centre
    crowd = c + rng.uniform(-0.45 * H, 0.45 * H, (300, 3))
    blob = np.stack(np.meshgrid(*[np.arange(0.4, 0.45, H / 2)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pts = np.concatenate([blob, crowd])
    m = ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0) if model == "sand" else ParticleModel.fluid_tait(
        1000.0, 1.0e4, 7.0)
    run(scene(f"crowd_{model}", pts, m, 2200.0 if model == "sand" else 1000.0), 5, loose=5.0)


def test_disabled_particles_mixed(cuda_lib):
    sc = scenes.random_scene_3d(6000, "elastic", H, seed=31, substeps=10)
    parts = sc.particles.copy()
    parts["enabled"][::4] = 0
    sc.particles = parts
    g = run(sc, 6, loose=3.0)
    assert np.all(g["enabled"][::4] == 0)


def test_far_clusters_negative_coordinates(cuda_lib):
    """Three clusters far apart, one at negative coordinates, no floor."""
    rng = np.random.default_rng(11)
    centres = [(-3.0, -2.0, -4.0), (0.5, 0.5, 0.5), (5.0, 1.0, -1.0)]
    pts = np.concatenate([np.asarray(c) + rng.uniform(-4 * H, 4 * H, (400, 3)) for c in centres])
    vel = rng.normal(0.0, 0.2, pts.shape)
    run(scene("far", pts, ParticleModel.elastic(1.0e5, 0.3), vel=vel, floor=False), 5, loose=3.0)
