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

