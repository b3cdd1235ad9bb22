"""Multi-scene batches (slosh_batch_* C ABI) on the GPU.

- a batch holding one scene reproduces the single-scene context;
- a scene's results are bit-identical alone and in a mix, also while other
  scenes join and leave (continuous batching);
- every scene of a mix matches the oracle within the FP32 tolerance of the
  single-scene parity tests;
- every launch shape the autotuner tries gives identical bits, the fused
  persistent substep (one cooperative kernel) included, in 3D and 2D and
  while scenes join and leave;
- capacity, state and unsupported-input errors are reported, not faulted,
  and so is a fused-kernel grid barrier that gives up waiting.
"""
import numpy as np
import pytest

from oracle import oracle as O
from slosh_b200 import scenes
from slosh_b200._lib import SLOSH_E_CAPACITY, SLOSH_E_INVALID, SLOSH_E_STATE, SLOSH_E_TIMEOUT, SloshError
from slosh_b200.batch import MpmBatch
from slosh_b200.pipeline import MpmPipeline

pytestmark = pytest.mark.gpu


def close(name, got, exp, atol, rtol):
    got = np.asarray(got, np.float64)
    exp = np.asarray(exp, np.float64)
    err = np.abs(got - exp).max() if got.size else 0.0
    bound = atol + rtol * (np.abs(exp).max() if exp.size else 0.0)
    print(f"{name}: max err {err:.3e} bound {bound:.3e}")
    assert err <= bound, f"{name}: max err {err:.3e} > {bound:.3e}"


def mix_scenes():
    return [
        scenes.random_scene_3d(6000, "sand", 1 / 64, seed=11),
        scenes.random_scene_3d(9000, "elastic", 1 / 128, seed=12),
        scenes.random_scene_3d(4000, "fluid", 1 / 64, seed=13),
        scenes.random_scene_3d(12000, "sand", 1 / 128, seed=14),
    ]


def new_batch(**kw):
    args = dict(max_particles=1 << 17, grid_capacity=1 << 13, max_scenes=64, max_bodies=256)
    args.update(kw)
    return MpmBatch(3, **args)


def fields(p):
    return {k: p[k] for k in ("position", "velocity", "def_grad", "affine", "mass", "model")}


def test_batch_of_one_matches_single_context(cuda_lib):
    """A scene alone in a batch advances like its own context, to FP32
    summation order: a context this small has its P2G blocks shared by a
    CTA's warps (a different, fixed order of the node sums), which a batch
    never does so that a scene's bits do not depend on its batch."""
    sc = scenes.sand_column_3d(h=1 / 32, substeps=10)
    data = scenes.build_mpm_data(sc)
    MpmPipeline().launch_step(data, 10)
    single = data.download_particles()
    data.close()
    b = new_batch()
    slot = b.add(sc)
    b.step(10)
    got = b.download_particles(slot)
    b.close()
    for k, v in fields(single).items():
        close(f"batch of one vs context {k}", got[k], v, 1e-6, 1e-5)
    assert np.array_equal(got["init_radius"], single["init_radius"])


def test_alone_vs_mix_bit_identical(cuda_lib):
    target = scenes.random_scene_3d(8000, "sand", 1 / 64, seed=21)
    alone = new_batch()
    s0 = alone.add(target)
    alone.step(30)
    ref = alone.download_particles(s0)
    alone.close()

    others = mix_scenes()
    mix = new_batch()
    mix.add(others[0])
    a = mix.add(others[1])
    st = mix.add(target)
    mix.step(10)
    mix.remove_scene(a)  # leaves at the next substep
    mix.add(others[2])
    mix.step(10)
    mix.add(others[3])
    mix.step(10)
    got = mix.download_particles(st)
    mix.close()
    assert got.tobytes() == ref.tobytes()


def test_mix_matches_oracle(cuda_lib):
    scs = mix_scenes()
    b = new_batch()
    slots = [b.add(sc) for sc in scs]
    b.step(5)
    loose = 5.0  # the single-scene parity tests' factor for multi-substep runs
    for sc, sl in zip(scs, slots):
        orc = O.from_scene(sc, threads=8)
        orc.step(5)
        o = orc.get_particles()
        g = b.download_particles(sl)
        tag = sc.name
        close(f"{tag} position", g["position"], o["position"], 1e-6 * loose, 0)
        close(f"{tag} velocity", g["velocity"], o["velocity"], 1e-6 * loose, 1e-4 * loose)
        close(f"{tag} def_grad", g["def_grad"], o["def_grad"], 2e-6 * loose, 2e-6 * loose)
        close(f"{tag} mass", g["mass"], o["mass"], 0, 0)
    b.close()


def test_launch_shapes_give_identical_bits(cuda_lib):
    scs = mix_scenes()
    results = []
    for shape in [(8, 128, 8, 3), (4, 64, 8, 2), (16, 256, 4, 4), (5, 64, 8, 3, 1)]:
        b = new_batch()
        slots = [b.add(sc) for sc in scs]
        b.set_tuning(*shape)
        b.step(8)
        results.append([b.download_particles(s).tobytes() for s in slots])
        b.close()
    assert results[0] == results[1] == results[2] == results[3]
    b = new_batch()
    for sc in scs:
        b.add(sc)
    tuned = b.autotune(1)
    assert tuned["g2p_threads"] in (64, 128, 256)
    b.step(2)
    b.sync()
    b.close()


def run_mix(dim, scs, fused, steps=(6, 6, 6)):
    """Scenes 0-1 from the start, scene 1 leaving and scene 2 joining after
    steps[0] substeps, scene 3 joining after steps[1] more; all results."""
    b = MpmBatch(dim, max_particles=1 << 17, grid_capacity=1 << 13, max_scenes=16, max_bodies=64)
    b.set_tuning(5, 64, 8, 3, fused)
    s0, s1 = b.add(scs[0]), b.add(scs[1])
    b.step(steps[0])
    gone = b.download_particles(s1).tobytes()
    b.remove_scene(s1)
    s2 = b.add(scs[2])
    b.step(steps[1])
    s3 = b.add(scs[3])
    b.step(steps[2])
    st = b.stats()
    assert st["tuning"]["fused"] == fused
    print(f"fused={fused}: fused kernel inside the substep graph: {bool(st['fused_graph'])}")
    out = [gone] + [b.download_particles(s).tobytes() for s in (s0, s2, s3)]
    b.sync()
    b.close()
    return out


def test_fused_substep_bit_identical_to_graph(cuda_lib):
    """The persistent cooperative substep gives the 13-kernel graph's bits,
    3D (sand, elastic, fluid; two cell widths) and 2D, with scenes joining
    and leaving between substeps."""
    scs3 = mix_scenes()
    assert run_mix(3, scs3, 1) == run_mix(3, scs3, 0)
    scs2 = [scenes.dam_break_2d(h=1 / 64, substeps=10), scenes.dam_break_2d(h=1 / 128, substeps=10),
            scenes.dam_break_2d(h=1 / 64, substeps=10), scenes.dam_break_2d(h=1 / 128, substeps=10)]
    assert run_mix(2, scs2, 1) == run_mix(2, scs2, 0)


def test_fused_barrier_timeout_reported(cuda_lib, monkeypatch):
    """The fused kernel's grid barriers wait with a time limit.  Made to wait
    for CTAs that never arrive (SLOSH_FUSED_BARRIER_TEST: 4 extra arrivals,
    a 1 ms limit), the substep ends and the host reports SLOSH_E_TIMEOUT;
    the device stays usable, and a new batch then runs normally."""
    scs = mix_scenes()
    monkeypatch.setenv("SLOSH_FUSED_BARRIER_TEST", "4:1000000")
    b = new_batch()
    for sc in scs[:2]:
        b.add(sc)
    b.set_tuning(5, 64, 8, 3, 1)
    with pytest.raises(SloshError) as e:
        b.step(1)
        b.sync()
    assert e.value.code == SLOSH_E_TIMEOUT
    b.close()
    monkeypatch.delenv("SLOSH_FUSED_BARRIER_TEST")
    got = run_mix(3, scs, 1)
    assert got == run_mix(3, scs, 0)


def mixed_model_scene():
    """A scene mixing every model (it goes to the G2P launch compiled for all
    models; one-model scenes go to launches compiled for their model)."""
    from slosh_b200.pipeline import ParticleModel, RigidBody, SimulationParams, make_particles

    h = 1 / 64
    rng = np.random.default_rng(23)
    models = [
        ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0),
        ParticleModel.elastic(1e5, 0.3),
        ParticleModel.elastic_neo_hookean(1e5, 0.3),
        ParticleModel.sand_neo_hookean(3.5e5, 0.3, friction_angle_deg=30.0),
        ParticleModel.fluid_tait(1000.0, 1e4, 7.0),
    ]
    parts = []
    for k, model in enumerate(models):
        lo = np.array([0.2 + 0.12 * k, 0.12, 0.45])
        parts.append(make_particles(lo + rng.uniform(0.0, 0.08, size=(600, 3)), h / 4, 1000.0, model, dim=3))
    parts = np.concatenate(parts)
    parts["velocity"][:, :3] = rng.normal(scale=0.3, size=(len(parts), 3)).astype(np.float32)
    floor = RigidBody(("cuboid", (4.0, 4 * h, 4.0)), translation=(0.5, 0.05 - 4 * h, 0.5))
    return scenes.Scene("mixed_models", 3, h, SimulationParams((0.0, -9.81, 0.0), 1e-4), parts, [floor], 10, 4096)


def test_mixed_model_scene_in_batch(cuda_lib):
    """A mixed-model scene beside one-model scenes (four G2P launches side
    by side): its bits equal the same scene alone in a batch, and it agrees
    with its own single-scene context to FP32 summation order."""
    mixed = mixed_model_scene()
    alone = new_batch()
    s0 = alone.add(mixed)
    alone.step(8)
    assert alone.stats()["g2p_launches"] == 1  # the launch compiled for every model
    ref = alone.download_particles(s0)
    alone.close()
    mix = new_batch()
    others = mix_scenes()
    mix.add(others[0])
    sm = mix.add(mixed)
    mix.add(others[1])
    mix.add(others[2])
    mix.step(8)
    assert mix.stats()["g2p_launches"] == 4  # sand, linear elastic, fluid, every model
    got = mix.download_particles(sm)
    mix.close()
    assert got.tobytes() == ref.tobytes()
    data = scenes.build_mpm_data(mixed)
    MpmPipeline().launch_step(data, 8)
    single = data.download_particles()
    data.close()
    # the context sums each P2G block in a different (fixed) grouping; over
    # 8 substeps of five models the velocities drift to the single-substep
    # parity bound (1e-4 of the scale, plus 2e-6), the other fields stay within
    # the batch-of-one bound
    for k, v in fields(single).items():
        loose = k in ("velocity", "affine")
        close(f"mixed-model batch vs context {k}", got[k], v, 2e-6 if loose else 1e-6, 1e-4 if loose else 1e-5)


def test_batch_errors_reported(cuda_lib):
    b = new_batch(max_particles=5000, max_scenes=2)
    sc = scenes.random_scene_3d(4000, "fluid", 1 / 64, seed=31)
    s0 = b.add(sc)
    with pytest.raises(SloshError) as e:
        b.add(sc)  # pool of 5000 particles
    assert e.value.code == SLOSH_E_CAPACITY
    forced = sc.particles.copy()[:100]
    forced["force_dt"][:, 0] = 1.0
    with pytest.raises(SloshError) as e:
        b.add_scene(forced, sc.cell_width, sc.params, sc.bodies)
    assert e.value.code == SLOSH_E_INVALID
    b.remove_scene(s0)
    with pytest.raises(SloshError) as e:
        b.remove_scene(s0)
    assert e.value.code == SLOSH_E_STATE
    b.step(1)  # the removed scene leaves storage
    assert b.stats()["n_particles"] == 0
    s1 = b.add(sc)  # the pool and the slot are free again
    b.step(2)
    assert b.stats()["live_scenes"] == 1 and b.stats()["n_particles"] == sc.n
    b.positions(s1)
    b.close()


def test_batch_timestep_bound_per_scene(cuda_lib):
    """Each scene's bound in a batch equals the single-scene context's."""
    scs = mix_scenes()
    b = new_batch()
    slots = [b.add(sc) for sc in scs]
    for sc, sl in zip(scs, slots):
        data = scenes.build_mpm_data(sc)
        assert b.timestep_bound(sl) == data.timestep_bound()
        data.close()
    b.close()


def test_batch_2d_alone_vs_mix_and_context(cuda_lib):
    """2D batches: a dam break alone in a batch equals the single-scene
    context, and stays bit-identical next to other 2D scenes of different
    cell widths."""
    a = scenes.dam_break_2d(h=1 / 64, substeps=10)
    b_sc = scenes.dam_break_2d(h=1 / 128, substeps=10)
    data = scenes.build_mpm_data(a)
    MpmPipeline().launch_step(data, 12)
    single = data.download_particles()
    data.close()
    alone = MpmBatch(2, max_particles=1 << 17, grid_capacity=1 << 12, max_scenes=8, max_bodies=64)
    s0 = alone.add(a)
    alone.step(12)
    ref = alone.download_particles(s0)
    alone.close()
    for k, v in fields(single).items():
        close(f"2D batch of one vs context {k}", ref[k], v, 1e-7, 1e-6)
    mix = MpmBatch(2, max_particles=1 << 17, grid_capacity=1 << 12, max_scenes=8, max_bodies=64)
    mix.add(b_sc)
    s1 = mix.add(a)
    mix.step(5)
    mix.add(b_sc)
    mix.step(7)
    got = mix.download_particles(s1)
    mix.close()
    assert got.tobytes() == ref.tobytes()


def test_two_way_scene_in_batch_matches_context(cuda_lib):
    """A scene with a two-way coupled ball advances in a batch next to other
    scenes as it does in its own context (ball and particles)."""
    sc = scenes.two_way_impact(3, h=1 / 64)
    data = scenes.build_mpm_data(sc)
    MpmPipeline().launch_step(data, 20)
    single, single_body = data.download_particles(), data.get_bodies()[0]
    data.close()
    b = new_batch()
    b.add(scenes.random_scene_3d(6000, "sand", 1 / 64, seed=11))
    slot = b.add(sc)
    b.step(20)
    got, body = b.download_particles(slot), b.get_bodies(slot)[0]
    b.close()
    assert body["linvel"][0] > 1e-3
    for k in ("linvel", "angvel", "translation", "rotation"):
        close(f"batched ball {k}", body[k][:3], single_body[k][:3], 1e-7, 1e-5)
    for k, v in fields(single).items():
        close(f"batched two-way scene {k}", got[k], v, 1e-7, 1e-6)


def test_cell_width_not_power_of_two_joins_batch(cuda_lib):
    """A scene whose cell width is not a power of two may join a batch of
    power-of-two scenes (the batch then stops using the multiply-only
    G2P): the earlier scene keeps its bits, and the new scene advances as in
    its own batch."""
    target = scenes.random_scene_3d(8000, "sand", 1 / 64, seed=21)
    odd = scenes.random_scene_3d(6000, "elastic", 1 / 48, seed=22)
    alone = new_batch()
    s0 = alone.add(target)
    alone.step(12)
    ref = alone.download_particles(s0)
    alone.close()
    odd_alone = new_batch()
    s1 = odd_alone.add(odd)
    odd_alone.step(6)
    ref_odd = odd_alone.download_particles(s1)
    odd_alone.close()
    mix = new_batch()
    st = mix.add(target)
    mix.step(6)
    so = mix.add(odd)
    mix.step(6)
    got, got_odd = mix.download_particles(st), mix.download_particles(so)
    mix.close()
    assert got.tobytes() == ref.tobytes()
    assert got_odd.tobytes() == ref_odd.tobytes()
