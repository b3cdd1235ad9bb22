"""The GPU SVD and its FP64 fallback, through the constitutive models.

The models' 3x3 SVD runs in FP32 and is recomputed in FP64 when F is nearly
singular or inverted (s2 <= 1e-3 s0), when the FP32 QR step leaves
off-diagonal mass above 1e-5 s0 (nearly repeated singular values), or when
all three singular values lie within 1e-5 s0 of each other away from a
rotation (nearly isotropic stretch, where Drucker-Prager's exact
zero-deviator test is discontinuous).  Here
particles at rest (v = 0, C = 0, no gravity, no collider) carry chosen
deformation gradients: the grid then holds zero velocity, the substep leaves
F unchanged up to the model, and the model's output is read back exactly:
  - F' (Drucker-Prager projects F) from the def_grad record,
  - the Kirchhoff stress from C = grad v m - tau V0 (4 / h^2) dt = -tau coef.
Both are compared with the FP64 oracle's model (`orc_model_stress`) on the
same FP32 inputs.  Reference formulas: shaders/slosh/models/
linear_elasticity.slang:69-82 and drucker_prager.slang:144-200.

Tolerance.  The input F is FP32, so the stress carries a noise floor of a
few FP32 ulps of F times the stiffness: |tau_gpu - tau_64| <= 2e-6 (lambda +
2 mu) + 1e-5 max |tau_64| for each family of inputs, and |F'_gpu - F'_64| <=
1e-6 + 1e-5 max |F'_64|.  Inverted F is not physical: both sides disable the
particle.
"""
import numpy as np
import pytest

from oracle import oracle as O
from slosh_b200.pipeline import MpmData, MpmPipeline, ParticleModel, SimulationParams, make_particles

pytestmark = pytest.mark.gpu

H = 1.0 / 64.0
DT = 2.0e-5


def _rotation(rng):
    q, r = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def _families(rng, per):
    """F = U diag(sigma) V^T for each family (FP32 entries)."""
    sig = {
        "repeated": [(1.0, 1.0 + 1e-7, 1.0 - 1e-7), (1.1, 1.1 * (1.0 + 3e-7), 0.97)],
        # all three nearly equal, away from a rotation: Drucker-Prager's exact
        # zero-deviator test is discontinuous there
        "isotropic": [(0.95, 0.95, 0.95 * (1 + 2e-7)), (1.08, 1.08 * (1 - 1e-7), 1.08), (0.9, 0.9 * (1 + 3e-7), 0.9 * (1 - 2e-7))],
        "near_singular": [(1.0, 0.6, 1e-5), (1.2, 2e-4, 1e-5), (0.9, 0.9, 5e-4)],
        "rotated_diagonal": [(1.05, 0.98, 0.93), (1.01, 1.0, 0.99), (0.97, 0.96, 0.9)],
        "inverted": [(1.0, 0.9, -0.8), (1.0, 1.0, -1e-4)],
    }
    out = {}
    for name, rows in sig.items():
        fs = []
        for k in range(per):
            s = np.diag(rows[k % len(rows)])
            U = _rotation(rng)
            V = U.T if name == "rotated_diagonal" and k % 2 == 0 else _rotation(rng).T
            fs.append(U @ s @ V)
        out[name] = np.asarray(fs, np.float32)
    return out


def _scene(model, fs):
    n = len(fs)
    side = int(np.ceil(n ** (1 / 3)))
    idx = np.arange(n)
    pts = 0.25 + H * np.stack([idx % side, (idx // side) % side, idx // (side * side)], axis=1) + 0.5 * H
    recs = make_particles(pts, H / 4, 1000.0, model, dim=3)
    for r in range(3):
        for c in range(3):
            recs["def_grad"][:, c * 3 + r] = fs[:, r, c]
    return recs


@pytest.mark.parametrize(
    "model",
    [ParticleModel.elastic(1.0e5, 0.3), ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0)],
    ids=["fixed_corotated", "drucker_prager"],
)
def test_svd_fp64_fallback_against_fp64_oracle(cuda_lib, model):
    rng = np.random.default_rng(31)
    fams = _families(rng, 60)
    names = list(fams)
    fs = np.concatenate([fams[k] for k in names])
    fam_of = np.concatenate([[k] * len(fams[k]) for k in names])
    recs = _scene(model, fs)
    data = MpmData(SimulationParams((0.0, 0.0, 0.0), DT), recs, [], cell_width=H, grid_capacity=1 << 12, dim=3)
    MpmPipeline().launch_step(data, 1)
    got = data.download_particles()
    n64 = data.stats()["n_svd_fp64"]
    data.close()

    v0 = np.float32(recs["init_volume"][0])
    coef = np.float64(v0 * np.float32(4.0 / (H * H)) * np.float32(DT))
    lam, mu = (model.data[9], model.data[10]) if model.tag == 2 else (model.data[0], model.data[1])
    stiff = lam + 2.0 * mu
    tau_gpu = np.empty((len(fs), 3, 3))
    f_gpu = np.empty((len(fs), 3, 3))
    for r in range(3):
        for c in range(3):
            tau_gpu[:, r, c] = -got["affine"][:, c * 3 + r].astype(np.float64) / coef
            f_gpu[:, r, c] = got["def_grad"][:, c * 3 + r]
    tau64 = np.empty_like(tau_gpu)
    f64 = np.empty_like(f_gpu)
    st64 = np.empty((len(fs), 3))
    for i in range(len(fs)):
        t, f, m = O.model_stress(model.tag, np.asarray(model.data, np.float64), fs[i].astype(np.float64))
        tau64[i], f64[i], st64[i] = t, f, m[:3]
    ok64 = np.isfinite(f64).all(axis=(1, 2)) & (np.linalg.det(np.nan_to_num(f64)) > 0)
    assert np.array_equal(got["enabled"].astype(bool), ok64), "disabled particles differ from the FP64 oracle"
    assert not ok64[fam_of == "inverted"].any()
    for name in names:
        sel = (fam_of == name) & ok64
        if not sel.any():
            continue
        et = np.abs(tau_gpu[sel] - tau64[sel]).max()
        bt = 2e-6 * stiff + 1e-5 * np.abs(tau64[sel]).max()
        ef = np.abs(f_gpu[sel] - f64[sel]).max()
        bf = 1e-6 + 1e-5 * np.abs(f64[sel]).max()
        print(f"{name}: tau err {et:.3e} (bound {bt:.3e}), F' err {ef:.3e} (bound {bf:.3e})")
        assert et <= bt, name
        assert ef <= bf, name
        if model.tag == 2:  # plastic state: det, hardening, log volume gain
            es = np.abs(got["model"][sel, :3].astype(np.float64) - st64[sel]).max(axis=0)
            print(f"{name}: plastic state err {es}")
            assert (es <= 1e-5 * np.maximum(1.0, np.abs(st64[sel]).max(axis=0))).all(), name
    must = int(((fam_of == "near_singular") | (fam_of == "inverted") | (fam_of == "isotropic")).sum())
    print(f"FP64 SVD fallbacks: {n64} (at least {must} expected)")
    assert n64 >= must
