"""Stage hooks (slosh's MpmPipelineHooks, src/pipeline.rs:146-238) on the GPU.

A hook is called at its point of every substep and may enqueue device work
on the substep's stream.  Checked here: every point is called once a
substep in launch_step's order, no-op hooks leave the results bit-identical,
a hook's change to the grid nodes after P2G reaches the particles, run
hooks that wrap the built-in stage give the built-in bits, and a failing
hook drops its substep without corrupting the scene.
"""
import ctypes
import glob
import os

import numpy as np
import pytest

from slosh_b200 import _lib, scenes
from slosh_b200.pipeline import MpmPipeline, MpmPipelineHooks

pytestmark = pytest.mark.gpu


def cudart():
    paths = glob.glob(os.path.join(os.path.dirname(np.__file__), "..", "nvidia", "cuda_runtime", "lib", "libcudart.so*"))
    paths += ["/usr/local/cuda/lib64/libcudart.so.12", "libcudart.so.12"]
    for p in paths:
        try:
            lib = ctypes.CDLL(p)
        except OSError:
            continue
        lib.cudaMemcpyAsync.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p]
        lib.cudaStreamSynchronize.argtypes = [ctypes.c_void_p]
        return lib
    raise RuntimeError("no CUDA runtime library to copy device buffers with")


D2H, H2D = 2, 1


def read_nodes(rt, data, stream):
    """The substep's grid nodes (n_blocks x 64 float4) copied to the host."""
    v = data.device_view()
    nb = np.zeros(1, np.uint32)
    assert rt.cudaMemcpyAsync(nb.ctypes.data, v.n_blocks, 4, D2H, stream) == 0
    assert rt.cudaStreamSynchronize(stream) == 0
    nodes = np.zeros((int(nb[0]) * 64, 4), np.float32)
    assert rt.cudaMemcpyAsync(nodes.ctypes.data, v.nodes, nodes.nbytes, D2H, stream) == 0
    assert rt.cudaStreamSynchronize(stream) == 0
    return nodes


def scene():
    return scenes.sand_column_3d(h=1 / 48)


def plain(sc, n):
    data = scenes.build_mpm_data(sc)
    MpmPipeline().launch_step(data, n)
    out = data.download_particles()
    data.close()
    return out


class Recorder(MpmPipelineHooks):
    def __init__(self):
        self.calls = []

    def after_particle_sort(self, data, stream, state):
        self.calls.append("after_particle_sort")

    def run_p2g(self, data, stream, state):
        self.calls.append("run_p2g")
        return False

    def after_p2g(self, data, stream, state):
        self.calls.append("after_p2g")

    def after_grid_update(self, data, stream, state):
        self.calls.append("after_grid_update")

    def run_g2p(self, data, stream, state):
        self.calls.append("run_g2p")
        return False

    def after_g2p(self, data, stream, state):
        self.calls.append("after_g2p")

    def after_particles_update(self, data, stream, state):
        self.calls.append("after_particles_update")


def test_noop_hooks_called_in_order_and_bit_identical(cuda_lib, monkeypatch):
    monkeypatch.setenv("SLOSH_GRID_REUSE", "1")
    sc = scene()
    ref = plain(sc, 12)
    data = scenes.build_mpm_data(sc)
    rec = Recorder()
    MpmPipeline().launch_step(data, 12, hooks=rec)
    got = data.download_particles()
    data.close()
    assert rec.calls == list(_lib.HOOK_NAMES) * 12
    assert got.tobytes() == ref.tobytes()


def test_after_p2g_sees_and_changes_the_nodes(cuda_lib):
    """The nodes after P2G carry the particles' mass; zeroing their momentum
    leaves each particle with the velocity gravity gives a grid at rest."""
    rt = cudart()
    sc = scene()
    mass = float(sc.particles["mass"].astype(np.float64).sum())

    class ZeroMomentum(MpmPipelineHooks):
        def __init__(self):
            self.masses = []

        def after_p2g(self, data, stream, state):
            nodes = read_nodes(rt, data, stream)
            self.masses.append(float(nodes[:, 3].astype(np.float64).sum()))
            nodes[:, :3] = 0.0
            v = data.device_view()
            assert rt.cudaMemcpyAsync(v.nodes, nodes.ctypes.data, nodes.nbytes, H2D, stream) == 0
            assert rt.cudaStreamSynchronize(stream) == 0

        def after_grid_update(self, data, stream, state):
            nodes = read_nodes(rt, data, stream)
            state.append(np.abs(nodes[:, :3]).max())

    data = scenes.build_mpm_data(sc)
    hk, seen = ZeroMomentum(), []
    MpmPipeline().launch_step(data, 1, hooks=hk, hooks_state=seen)
    got = data.download_particles()
    data.close()
    assert abs(hk.masses[0] - mass) <= 1e-6 * mass
    g_dt = 9.81 * sc.params.dt
    assert seen[0] <= g_dt * (1 + 1e-5)  # node velocities: gravity only (or 0 at the floor)
    vy = got["velocity"][:, 1][got["enabled"] == 1]
    print(f"particle vy: min {vy.min():.6e} max {vy.max():.6e}, -g dt = {-g_dt:.6e}")
    assert np.abs(got["velocity"][:, [0, 2]]).max() <= 1e-6
    assert vy.max() <= 1e-9 and vy.min() >= -g_dt * (1 + 1e-5)


def test_run_hooks_wrapping_the_builtin_are_bit_identical(cuda_lib, monkeypatch):
    monkeypatch.setenv("SLOSH_GRID_REUSE", "1")  # a replaced G2P must turn grid reuse off for a substep
    sc = scene()
    ref = plain(sc, 10)

    class Wrap(MpmPipelineHooks):
        def run_p2g(self, data, stream, state):
            data.enqueue_builtin(_lib.HOOK_RUN_P2G, stream)
            return True

        def run_g2p(self, data, stream, state):
            data.enqueue_builtin(_lib.HOOK_RUN_G2P, stream)
            return True

    data = scenes.build_mpm_data(sc)
    MpmPipeline().launch_step(data, 10, hooks=Wrap())
    got = data.download_particles()
    st = data.stats()
    data.close()
    assert got.tobytes() == ref.tobytes()
    # a replaced G2P records no cell changes, so every substep rebuilt its grid
    assert st["n_grid_reuses"] == 0


def test_failing_hook_drops_its_substep(cuda_lib, monkeypatch):
    monkeypatch.setenv("SLOSH_GRID_REUSE", "1")  # the dropped substep also resets the kept grid
    sc = scene()
    ref = plain(sc, 8)

    class Boom(MpmPipelineHooks):
        def after_g2p(self, data, stream, state):
            raise ValueError("hook failure")

    data = scenes.build_mpm_data(sc)
    pipe = MpmPipeline()
    pipe.launch_step(data, 5)
    with pytest.raises(ValueError):
        pipe.launch_step(data, 1, hooks=Boom())
    pipe.launch_step(data, 3)
    got = data.download_particles()
    data.close()
    assert got.tobytes() == ref.tobytes()


def test_view_and_builtin_only_inside_hooks(cuda_lib):
    sc = scene()
    data = scenes.build_mpm_data(sc)
    with pytest.raises(_lib.SloshError) as ei:
        data.device_view()
    assert ei.value.code == _lib.SLOSH_E_STATE
    with pytest.raises(_lib.SloshError):
        data.enqueue_builtin(_lib.HOOK_RUN_P2G, None)
    data.close()
