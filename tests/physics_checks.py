"""Physics checks shared by the oracle tests and the GPU tests."""
import math


def dam_front_checks(advance, front_x, a, taus, tol):
    """Advances a 2D dam break to each dimensionless time tau = sqrt(2 g / a) t
    and compares the surge front (the largest x; the wall is at x = 0) with
    the criterion of slosh's own validation scenario
    (validation_tests/src/scenarios/dam_break.rs:55-70, after Martin & Moyce
    1952): x / a = 1 + tau^2 / 4 for tau < 2, about tau after."""
    k = math.sqrt(2.0 * 9.81 / a)
    t = 0.0
    for tau in taus:
        n = int(round((tau / k - t) / 1e-4))
        advance(n)
        t += n * 1e-4
        front = front_x() / a
        model = 1.0 + (k * t) ** 2 / 4.0 if k * t < 2.0 else k * t
        print(f"tau {k * t:.2f}: front {front:.3f} a, criterion {model:.3f} a")
        assert abs(front / model - 1.0) <= tol, (k * t, front, model)



def cantilever_scene(h=1.0 / 64.0, young=9.2e6, dim=2, neo_hookean=False):
    """A 2D cantilever after slosh's elastic-beam validation scenario
    (validation_tests/src/scenarios/elastic_beam.rs:58-63): a fixed-corotated
    beam (Poisson ratio 0, so plane strain and plane stress agree) of length
    L = 0.5 and height H = 0.1, clamped by embedding its first 4 cells in a
    sticky wall, loaded by gravity from rest (`neo_hookean`: the Neo-Hookean
    model, which agrees with it at these small strains).  Returns the scene, the mask of
    the particles within a cell of the tip, the analytic static tip
    deflection q L^4 / (8 E I) and the first bending period in substeps.
    In 3D the beam's cross-section is H x H (I = H^4 / 12, q = rho g H^2:
    the same deflection and period)."""
    import numpy as np

    from slosh_b200 import scenes
    from slosh_b200.pipeline import GpuBoundaryCondition, ParticleModel, RigidBody, SimulationParams, make_particles

    rho, g, length, height, x0, dt = 1000.0, 9.81, 0.5, 0.1, 0.2, 5e-5
    xs = np.arange(x0 - 4 * h + h / 4, x0 + length, h / 2)
    ys = np.arange(0.5 - height / 2 + h / 4, 0.5 + height / 2, h / 2)
    axes = (xs, ys) if dim == 2 else (xs, ys, ys)
    pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, dim)
    model = ParticleModel.elastic_neo_hookean(young, 0.0) if neo_hookean else ParticleModel.elastic(young, 0.0)
    parts = make_particles(pts, h / 4, rho, model, dim=dim)
    if dim == 2:
        wall = RigidBody(("cuboid", (0.1, 0.2)), translation=(x0 - 0.1, 0.5), rotation=0.0,
                         boundary_condition=GpuBoundaryCondition.stick())
        gravity = (0.0, -g)
    else:
        wall = RigidBody(("cuboid", (0.1, 0.2, 0.2)), translation=(x0 - 0.1, 0.5, 0.5),
                         boundary_condition=GpuBoundaryCondition.stick())
        gravity = (0.0, -g, 0.0)
    sc = scenes.Scene(f"cantilever_{dim}d", dim, h, SimulationParams(gravity, dt), parts, [wall], 10,
                      4096 if dim == 2 else 8192)
    inertia = height**3 / 12.0
    delta = rho * g * height * length**4 / (8.0 * young * inertia)
    omega = 1.875**2 * math.sqrt(young * inertia / (rho * height * length**4))
    return sc, pts[:, 0] > x0 + length - h, delta, int(2.0 * math.pi / omega / dt)


def cantilever_checks(advance, tip_y, tip, delta, period, tol):
    """Samples the tip's mean deflection 40 times over two bending periods.
    Released from rest under a suddenly applied load, the undamped beam
    swings between 0 and twice the static deflection, so the samples'
    mean is the static deflection (within `tol` of the analytic one) and
    their largest is about twice it."""
    import numpy as np

    y0 = float(tip_y()[tip].mean())
    d = []
    for _ in range(40):
        advance(period // 20)
        d.append(y0 - float(tip_y()[tip].mean()))
    d = np.asarray(d)
    print(f"tip deflection: mean {d.mean():.5f}, peak {d.max():.5f}; analytic static {delta:.5f}")
    assert abs(d.mean() / delta - 1.0) <= tol, (d.mean(), delta)
    assert 1.8 <= d.max() / delta <= 2.2, (d.max(), delta)


def tank_scene(h=1.0 / 64.0, depth=0.2):
    """A 2D layer of the Tait fluid (rest density 1000, K = 1e4, gamma = 7)
    filling the unit box's width to `depth`, released at rest with J = 1
    (no initial pressure), sticky walls."""
    import numpy as np

    from slosh_b200 import scenes
    from slosh_b200.pipeline import GpuBoundaryCondition, ParticleModel, SimulationParams, make_particles

    xs = np.arange(h / 4, 1.0, h / 2)
    ys = np.arange(h / 4, depth, h / 2)
    pts = np.stack(np.meshgrid(xs, ys, indexing="ij"), -1).reshape(-1, 2)
    parts = make_particles(pts, h / 4, 1000.0, ParticleModel.fluid_tait(1000.0, 1.0e4, 7.0), dim=2)
    return scenes.Scene("tank_2d", 2, h, SimulationParams((0.0, -9.81), 1e-4), parts,
                        scenes._walls_2d(h, GpuBoundaryCondition.stick()), 10, 8192)


def hydrostatic_check(advance, particles, depth, tol):
    """Lets the layer settle for 0.5 s, then averages the particles' Tait
    pressure p = (K / gamma) (J^-gamma - 1) (J = F00, the fluid's volume
    ratio) in ten depth bins over the next second.  Between the bottom's
    boundary layer (the first two bins) and the free surface (the last) the
    profile is hydrostatic: its slope is rho0 g within `tol`."""
    import numpy as np

    advance(5000)
    bins = np.linspace(0.0, depth, 11)
    prof = np.zeros(10)
    for _ in range(20):
        advance(500)
        p = particles()
        J = p["def_grad"][:, 0]
        pr = (1.0e4 / 7.0) * (J**-7.0 - 1.0)
        idx = np.digitize(p["position"][:, 1], bins) - 1
        prof += np.array([pr[idx == i].mean() for i in range(10)]) / 20.0
    mid = 0.5 * (bins[1:] + bins[:-1])
    slope = -np.polyfit(mid[2:9], prof[2:9], 1)[0]
    print("pressure by depth bin:", np.round(prof, 1), f"slope {slope:.0f} (rho0 g = 9810)")
    assert abs(slope / 9810.0 - 1.0) <= tol, slope


def sand_layer_check(h=1.0 / 64.0, depth=0.2, tol=0.10, oracle=None):
    """A 2D layer of Drucker-Prager sand (the benchmark's material: friction
    angle 30 deg, E = 3.5e5, nu = 0.3, density 2200) filling the unit box's
    width to `depth` between frictionless (slip) walls settles for 0.5 s;
    averaged over the next second, the Cauchy stress sigma_yy of its
    fixed-corotated elasticity, tau = 2 mu (F - R) F^T + lambda (J - 1) J I
    over J, grows with depth at rho g within `tol` between the bottom's
    boundary layer and the surface: the layer carries its own weight."""
    import numpy as np

    from slosh_b200 import scenes
    from slosh_b200.pipeline import GpuBoundaryCondition, ParticleModel, SimulationParams, make_particles

    rho, g = 2200.0, 9.81
    xs = np.arange(h / 4, 1.0, h / 2)
    ys = np.arange(h / 4, depth, h / 2)
    pts = np.stack(np.meshgrid(xs, ys, indexing="ij"), -1).reshape(-1, 2)
    parts = make_particles(pts, h / 4, rho, ParticleModel.sand(3.5e5, 0.3, friction_angle_deg=30.0), dim=2)
    lam, mu = float(parts["model"][0][9]), float(parts["model"][0][10])
    sc = scenes.Scene("sand_layer_2d", 2, h, SimulationParams((0.0, -g), 1e-4), parts,
                      scenes._walls_2d(h, GpuBoundaryCondition.slip()), 10, 8192)
    o = oracle.from_scene(sc)
    o.step(5000)
    bins = np.linspace(0.0, depth, 11)
    prof = np.zeros(10)
    for _ in range(20):
        o.step(500)
        p = o.get_particles()
        f = p["def_grad"].astype(np.float64)
        F = np.stack([np.stack([f[:, 0], f[:, 3]], -1), np.stack([f[:, 1], f[:, 4]], -1)], 1)  # column-major
        u, _, vt = np.linalg.svd(F)
        J = np.linalg.det(F)
        tau = 2.0 * mu * (F - u @ vt) @ np.transpose(F, (0, 2, 1)) + (lam * (J - 1.0) * J)[:, None, None] * np.eye(2)
        syy = tau[:, 1, 1] / J
        idx = np.digitize(p["position"][:, 1], bins) - 1
        prof += np.array([syy[idx == i].mean() for i in range(10)]) / 20.0
    mid = 0.5 * (bins[1:] + bins[:-1])
    slope = np.polyfit(mid[2:9], prof[2:9], 1)[0]
    print("sigma_yy by depth bin:", np.round(prof, 0), f"slope {slope:.0f} (rho g = {rho * g:.0f})")
    assert abs(slope / (rho * g) - 1.0) <= tol, slope
