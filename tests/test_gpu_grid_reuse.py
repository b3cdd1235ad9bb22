"""Grid reuse between substeps, on the GPU, through the C ABI.

A substep keeps the previous substep's grid (blocks, ranks, hash map) when
no particle left the set of blocks holding particles, and only re-counts
the cells particles entered or left; otherwise it runs the full build.  The
kept layout must be the one the full build gives from the same positions:
the same canonical permutation, so the same P2G summation order and the
same bits.  Each scene runs twice, with reuse and with every substep a full
build (SLOSH_GRID_REUSE=0 at context creation), and the particle records
are compared byte for byte.
"""
import numpy as np
import pytest

from slosh_b200 import scenes
from slosh_b200.pipeline import MpmPipeline

pytestmark = pytest.mark.gpu


def run(sc, substeps, monkeypatch, reuse, between=None):
    monkeypatch.setenv("SLOSH_GRID_REUSE", "1" if reuse else "0")
    data = scenes.build_mpm_data(sc)
    pipe = MpmPipeline()
    done = 0
    for k in substeps:
        pipe.launch_step(data, k - done)
        done = k
        if between is not None:
            between(data, k)
    out = data.download_particles()
    st = data.stats()
    data.close()
    return out, st


@pytest.mark.parametrize(
    "name",
    ["sand3d", "fluid2d", "elastic3d", "sand3d_two_way"],
)
def test_reuse_matches_full_build_bit_for_bit(cuda_lib, monkeypatch, name):
    sc = {
        "sand3d": lambda: scenes.sand_column_3d(h=1 / 64),
        "fluid2d": lambda: scenes.dam_break_2d(h=1 / 128),
        "elastic3d": lambda: scenes.elastic_drop_3d(h=1 / 64),
        "sand3d_two_way": lambda: scenes.sand_column_3d(h=1 / 48, cube_coupling="two_way"),
    }[name]()
    steps = [60]
    full, st_full = run(sc, steps, monkeypatch, reuse=False)
    kept, st_kept = run(sc, steps, monkeypatch, reuse=True)
    print(f"{name}: {sc.n} particles, reuse {st_kept['n_grid_reuses']} of 60 substeps, "
          f"rebuilds {st_kept['n_grid_rebuilds']}, conditional graphs {st_kept['conditional_graphs']}")
    assert st_full["n_grid_reuses"] == 0
    assert st_kept["n_grid_reuses"] + st_kept["n_grid_rebuilds"] == 60
    assert kept.tobytes() == full.tobytes()


def test_reuse_with_uploads_and_debug_builds(cuda_lib, monkeypatch):
    """An upload, an append, a removal and the debug grid build between
    substeps each make the next substep rebuild; results stay identical to
    the full build's."""
    sc = scenes.sand_column_3d(h=1 / 48)
    extra = scenes.sand_column_3d(h=1 / 48, radius=0.05).particles.copy()
    extra["position"][:, 0] += 0.3

    def between(data, k):
        if k == 10:
            data.grid_debug()
        elif k == 20:
            p = data.download_particles()
            p["velocity"][:, 1] -= 0.5
            data.upload(p)
        elif k == 30:
            data.append(extra)
        elif k == 40:
            data.shift_remove(100, 400)
        elif k == 50:
            data.debug_nodes(2)

    def go(reuse):
        monkeypatch.setenv("SLOSH_GRID_REUSE", "1" if reuse else "0")
        data = scenes.build_mpm_data(sc, max_particles=sc.n + len(extra))
        pipe = MpmPipeline()
        done = 0
        for k in (10, 20, 30, 40, 50, 60):
            pipe.launch_step(data, k - done)
            done = k
            between(data, k)
        out, st = data.download_particles(), data.stats()
        data.close()
        return out, st

    full, _ = go(False)
    kept, st = go(True)
    print(f"reuse {st['n_grid_reuses']}, rebuilds {st['n_grid_rebuilds']}")
    assert st["n_grid_reuses"] > 0
    assert kept.tobytes() == full.tobytes()


def test_reuse_full_size_sand_column(cuda_lib, monkeypatch):
    """The 4.74 M-particle sand column: 40 substeps with reuse equal the full
    build's bits."""
    sc = scenes.sand_column_3d()
    full, _ = run(sc, [40], monkeypatch, reuse=False)
    kept, st = run(sc, [40], monkeypatch, reuse=True)
    print(f"4.74M: reuse {st['n_grid_reuses']} of 40, rebuilds {st['n_grid_rebuilds']}")
    assert st["n_grid_reuses"] > 0
    assert kept.tobytes() == full.tobytes()


def test_reuse_with_forces_damping_fixed(cuda_lib, monkeypatch):
    """Pending forces (a substep launched kernel by kernel), damping and
    fixed particles under grid reuse: the same bits as full builds."""
    sc = scenes.elastic_drop_3d(h=1 / 48)
    parts = sc.particles.copy()
    parts["force_dt"][::3] = (0.0, 2e-3, -1e-3)
    parts["damping"][::5] = 3.0
    parts["fixed"][::11] = 1
    sc.particles = parts
    full, _ = run(sc, [30], monkeypatch, reuse=False)
    kept, st = run(sc, [30], monkeypatch, reuse=True)
    print(f"forces/damping/fixed: reuse {st['n_grid_reuses']} of 30")
    assert st["n_grid_reuses"] > 0
    assert kept.tobytes() == full.tobytes()
