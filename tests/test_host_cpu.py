"""CPU checks of the host side: the C ABI library loads and exports every
declared symbol, record layouts match the C structs, model constructors and
scene generators follow the reference's definitions."""
import math
import os
import re
import subprocess
import textwrap

import numpy as np
import pytest

from slosh_b200 import _lib, scenes
from slosh_b200.pipeline import ParticleModel, lame_lambda_mu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "slosh_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|uint32_t)\s+\*?\s*(slosh_\w+)\s*\(", src, re.M)))


@pytest.fixture(scope="module")
def built_lib():
    from slosh_b200.build import build_library

    return build_library()


def test_library_exports_every_declared_symbol(built_lib):
    names = declared_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the ctypes binding covers exactly those symbols
    assert sorted(_lib.SIGNATURES) == names


def test_library_loads_without_gpu(built_lib):
    lib = _lib.load()
    for name in declared_functions():
        assert getattr(lib, name) is not None


def test_record_layouts_match_c_structs(tmp_path):
    prog = textwrap.dedent(
        """
        #include <stdio.h>
        #include <stddef.h>
        #include "slosh_b200.h"
        int main(void) {
          printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(slosh_particle), offsetof(slosh_particle, model),
                 offsetof(slosh_particle, enabled), sizeof(slosh_body), offsetof(slosh_body, bc_type),
                 sizeof(slosh_model));
          printf("%zu %zu\\n", sizeof(slosh_grid_dump), offsetof(slosh_grid_dump, neighbors));
          printf("%zu %zu %zu %zu %zu\\n", sizeof(slosh_batch_config), sizeof(slosh_scene_desc),
                 sizeof(slosh_tuning), sizeof(slosh_batch_stats), offsetof(slosh_batch_stats, tuning));
          printf("%zu %zu %zu %zu %zu\\n", sizeof(slosh_server_config), sizeof(slosh_request),
                 offsetof(slosh_request, particles), sizeof(slosh_completion), sizeof(slosh_server_stats));
          printf("%zu\\n", offsetof(slosh_body, coupling));
          return 0;
        }
        """
    )
    c = tmp_path / "layout.c"
    c.write_text(prog)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    vals = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    P, B = _lib.PARTICLE_DTYPE, _lib.BODY_DTYPE
    assert vals[0] == P.itemsize
    assert vals[1] == P.fields["model_tag"][1]
    assert vals[2] == P.fields["enabled"][1]
    assert vals[3] == B.itemsize
    assert vals[4] == B.fields["bc_type"][1]
    assert vals[5] == 52
    assert vals[-1] == B.fields["coupling"][1]
    import ctypes

    assert vals[6] == ctypes.sizeof(_lib.SloshGridDump)
    assert vals[7] == _lib.SloshGridDump.neighbors.offset
    assert vals[8:13] == [
        ctypes.sizeof(_lib.SloshBatchConfig),
        ctypes.sizeof(_lib.SloshSceneDesc),
        ctypes.sizeof(_lib.SloshTuning),
        ctypes.sizeof(_lib.SloshBatchStats),
        _lib.SloshBatchStats.tuning.offset,
    ]
    assert vals[13:18] == [
        ctypes.sizeof(_lib.SloshServerConfig),
        ctypes.sizeof(_lib.SloshRequest),
        _lib.SloshRequest.particles.offset,
        ctypes.sizeof(_lib.SloshCompletion),
        ctypes.sizeof(_lib.SloshServerStats),
    ]


def test_lame_parameters():
    """Config values quoted for the configs (src/models/mod.rs:17-27)."""
    lam, mu = lame_lambda_mu(3.5e5, 0.3)
    assert round(lam) == 201923 and round(mu) == 134615
    lam, mu = lame_lambda_mu(1e5, 0.3)
    assert round(lam) == 57692 and round(mu) == 38462


def test_sand_model_record():
    m = ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0)
    assert m.tag == _lib.MODEL_SAND_LINEAR and len(m.data) == 12
    assert m.data[:3] == (1.0, 1.0, 0.0)  # DruckerPragerPlasticState::default
    assert math.isclose(m.data[3], math.radians(30.0))
    assert math.isclose(m.data[4], math.radians(9.0)) and m.data[5] == 0.2
    assert math.isclose(m.data[6], math.radians(10.0))


def test_scene_sizes():
    d = scenes.dam_break_2d()
    assert d.n == 204 * 307
    e = scenes.elastic_drop_3d(h=1 / 64)
    assert e.n == 2 * 32**3
    # full-size sand column: count lattice points inside the cylinder only
    h = 1 / 256
    sp = h / 2
    n_axis = int(math.floor(0.3 / sp + 1e-9))
    c = 0.5 - 0.15 + (np.arange(n_axis) + 0.5) * sp
    inside = ((c[:, None] - 0.5) ** 2 + (c[None, :] - 0.5) ** 2 <= 0.15**2).sum()
    n_full = int(inside) * int(math.floor(0.5 / sp + 1e-9))
    assert 4.6e6 < n_full < 4.8e6


def test_scene_determinism():
    a = scenes.sand_column_3d(h=1 / 32).particles
    b = scenes.sand_column_3d(h=1 / 32).particles
    assert np.array_equal(a, b)


def _c_structs(src):
    """typedef struct name { fields } name; -> {name: [(field, type, count)]}."""
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\} \1;", src, re.S):
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            ty, rest = decl.split(None, 1) if not decl.startswith("const ") else ("const " + decl.split()[1], decl.split(None, 2)[2])
            for item in rest.split(","):
                m = re.fullmatch(r"\s*\*?\s*(\w+)\s*(?:\[(\d+)\])?\s*", item)
                assert m, (name, decl)
                fields.append((m.group(1), ty, int(m.group(2) or 1)))
        out[name] = fields
    return out


def _rust_structs(md):
    """#[repr(C)] structs of INTEGRATION.md's Rust blocks."""
    block = "\n".join(b.split("```", 1)[0] for b in md.split("```rust")[1:])
    block = re.sub(r"//[^\n]*", "", block)
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\][^{]*?pub struct (\w+)\s*\{(.*?)\}", block, re.S):
        assert name not in out, name
        fields = []
        for m in re.finditer(r"(?:pub\s+)?(\w+)\s*:\s*(\[\s*\w+\s*;\s*\d+\s*\]|\w+)", body):
            ty = m.group(2).replace(" ", "")
            arr = re.fullmatch(r"\[(\w+);(\d+)\]", ty)
            fields.append((m.group(1), arr.group(1), int(arr.group(2))) if arr else (m.group(1), ty, 1))
        out[name] = fields
    return out


def test_integration_rust_records_match_header():
    """The #[repr(C)] records of the documented Rust binding have the
    header's fields, types and order, so a maintainer who copies them gets
    the library's exact layouts."""
    c = _c_structs(open(HEADER).read())
    rust = _rust_structs(open(os.path.join(ROOT, "INTEGRATION.md")).read())
    c_to_rust = {"float": "f32", "double": "f64", "uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64",
                 "slosh_model": "SloshModel", "slosh_params": "SloshParams", "slosh_tuning": "SloshTuning"}
    pairs = {"SloshModel": "slosh_model", "SloshParticle": "slosh_particle", "SloshBody": "slosh_body",
             "SloshConfig": "slosh_config", "SloshParams": "slosh_params", "SloshBatchConfig": "slosh_batch_config",
             "SloshSceneDesc": "slosh_scene_desc", "SloshTuning": "slosh_tuning", "SloshBatchStats": "slosh_batch_stats",
             "SloshServerConfig": "slosh_server_config", "SloshCompletion": "slosh_completion",
             "SloshServerStats": "slosh_server_stats", "SloshStats": "slosh_stats"}
    assert set(pairs) <= set(rust), sorted(rust)
    for rname, cname in pairs.items():
        want = [(f, c_to_rust[t], k) for f, t, k in c[cname]]
        assert rust[rname] == want, (rname, rust[rname], want)


def test_environment_settings_documented():
    """Every SLOSH_* setting the library reads from the environment is listed
    in INTEGRATION.md's table of settings."""
    src = os.path.join(ROOT, "slosh_b200", "csrc")
    names = set()
    for f in os.listdir(src):
        if f.endswith((".cu", ".cuh")):
            names |= set(re.findall(r'getenv\("(SLOSH_[A-Z0-9_]+)"\)', open(os.path.join(src, f)).read()))
    assert names, "no settings found"
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = sorted(n for n in names if f"`{n}" not in doc)
    assert not missing, missing


def test_bench_l2_note():
    """bench.py states, per line, whether the particle storage its timed
    substeps touch outgrows the L2 (no flush runs between substeps)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.l2_note(62628 * bench.STORAGE_BYTES).startswith("inputs smaller than L2")  # dam break
    assert bench.l2_note(4741888 * bench.STORAGE_BYTES).startswith("inputs larger than L2")  # sand column
    assert "4.9 GB" in bench.l2_note(17607256 * bench.STORAGE_BYTES)  # 256-scene batch
    cfg = bench.workload_config(scenes.sand_column_3d(h=1.0 / 64.0))
    assert cfg["l2"].startswith("inputs smaller than L2")  # a reduced column: about 20 MB


def test_integration_rust_declares_every_export():
    """INTEGRATION.md's Rust blocks declare every function the header
    declares, each with the header's number of parameters."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    c_args = {}
    for name, params in re.findall(r"^\s*(?:int|void|uint32_t)\s+\*?\s*(slosh_\w+)\s*\(([^)]*)\)\s*;", src, re.M):
        params = params.strip()
        c_args[name] = 0 if params in ("", "void") else params.count(",") + 1
    assert set(c_args) == set(declared_functions())
    md = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    rust = "\n".join(b.split("```", 1)[0] for b in md.split("```rust")[1:])
    rust = re.sub(r"//[^\n]*", "", rust)
    r_args = {}
    for name, params in re.findall(r"pub fn (slosh_\w+)\s*\(([^)]*)\)", rust, re.S):
        params = params.strip()
        r_args[name] = 0 if not params else params.count(",") + 1
    missing = sorted(set(c_args) - set(r_args))
    assert not missing, missing
    wrong = sorted(n for n in c_args if r_args[n] != c_args[n])
    assert not wrong, [(n, c_args[n], r_args[n]) for n in wrong]


def test_bench_launch_accounting():
    """bench.py counts a kept-grid substep 7 kernels below a full-build one
    (the 9 build kernels replaced by the 2 reuse kernels) when the graphs
    are conditional, and every substep at the library's count otherwise."""
    import importlib.util
    from types import SimpleNamespace

    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    st0 = {"n_grid_reuses": 10, "n_grid_rebuilds": 3, "conditional_graphs": 1}
    st1 = {"n_grid_reuses": 27, "n_grid_rebuilds": 6, "conditional_graphs": 1}
    launches, reuse = bench.timed_launches(SimpleNamespace(kernels_per_substep=14), st0, st1, 20)
    assert launches == 14 * 3 + 7 * 17 and reuse["reused_substeps"] == 17 and reuse["rebuilt_substeps"] == 3
    st1 = {"n_grid_reuses": 0, "n_grid_rebuilds": 0, "conditional_graphs": 0}
    launches, _ = bench.timed_launches(SimpleNamespace(kernels_per_substep=13), st1, st1, 1000)
    assert launches == 13000
