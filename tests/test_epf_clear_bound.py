"""The displacement-first clear-hold bound of the staged explicit step (the step configurations with flag 8).

A bond whose relative displacement e = u_j - u_i satisfies |e|^2 < e2_hold, e2_hold = (s_c (1 - 1e-6) - 1e-12)^2
r_min^2 with r_min the mesh's shortest bond, is taken as holding without its positions being read: its stretch
s = (|xi + e| - |xi|) / |xi| is at most |e| / |xi| <= |e| / r_min < s_c. This checks that the argument survives
rounding: the bond stretch in the reference's FP64 arithmetic (ExplicitPDDOFracElement.cpp:239-266, restated in
oracle/pddo_oracle.c orc_epf_rate: s = (sqrt(y.y) - r) / r, y = xi + e, every operation rounded) never breaks a
bond the bound clears, for tension-only and two-sided criteria, critical stretches from 1e-6 to 0.5, bonds from
r_min to 3 r_min, lattice and random directions, and displacements placed at the bound along and against the bond
(the worst case) as well as in random directions. Host arithmetic only (numpy rounds every operation)."""
import numpy as np


def _clear_bound(sc, r2min):
    """e2_hold as the set-up computes it (capi.cpp epf_args)."""
    s = sc * (1.0 - 1.0e-6) - 1.0e-12
    return s * s * r2min if s > 0.0 else 0.0


def _ref_stretch(xi, e):
    """The reference's stretch of bond vectors xi (k x 3) under relative displacements e, op by op."""
    r = np.sqrt((xi[:, 0] * xi[:, 0] + xi[:, 1] * xi[:, 1]) + xi[:, 2] * xi[:, 2])
    y = xi + e
    return (np.sqrt((y[:, 0] * y[:, 0] + y[:, 1] * y[:, 1]) + y[:, 2] * y[:, 2]) - r) / r


def _kernel_e2(e):
    """|e|^2 with every operation rounded; the kernel's fused multiply-add for the last term differs from this by
    at most an ulp, far inside the bound's 1e-6 relative margin."""
    return e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1] + e[:, 2] * e[:, 2]


def _bonds(rng, h, k):
    """k bond vectors from a lattice point x_i to x_j, |xi| in [h, 3h]: lattice offsets and random directions, with
    the coordinates' own rounding (x_j - x_i of points in a 0.12 m box)."""
    offs = np.array([(a, b, c) for a in range(-3, 4) for b in range(-3, 4) for c in range(-3, 4)
                     if 0 < a * a + b * b + c * c <= 9], np.float64)
    lat = offs[rng.integers(0, len(offs), k // 2)] * h
    d = rng.standard_normal((k - k // 2, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    rnd = d * rng.uniform(h, 3 * h, (k - k // 2, 1))
    xi_ideal = np.vstack([lat, rnd])
    xi0 = rng.uniform(0.0, 0.12, (k, 3))
    xj0 = xi0 + xi_ideal
    return xj0 - xi0  # rounded as the kernels form it


def test_clear_bound_never_clears_a_breaking_bond():
    rng = np.random.default_rng(2025)
    h = 1.0e-3
    k = 200_000
    cleared_total = 0
    for sc in (1.0e-6, 1.0e-4, 4.0e-3, 5.0e-2, 0.5):
        xi = _bonds(rng, h, k)
        r2 = (xi[:, 0] * xi[:, 0] + xi[:, 1] * xi[:, 1]) + xi[:, 2] * xi[:, 2]
        r2min = float(r2.min())
        hold2 = _clear_bound(sc, r2min)
        lim = np.sqrt(hold2)
        # displacements at the bound: along the bond (pure tension), against it (pure compression), random
        unit = xi / np.sqrt(r2)[:, None]
        d = rng.standard_normal((k, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        scale = lim * (1.0 - rng.uniform(0.0, 1.0e-12, (k, 1)))
        for e_ideal in (unit * scale, -unit * scale, d * scale):
            ui = rng.uniform(-1.0e-3, 1.0e-3, (k, 3))
            e = (ui + e_ideal) - ui  # e = u_j - u_i with the state's rounding
            cleared = _kernel_e2(e) < hold2
            s = _ref_stretch(xi, e)
            assert not np.any(cleared & (s > sc)), "tension-only: a cleared bond breaks"
            assert not np.any(cleared & (np.abs(s) > sc)), "two-sided: a cleared bond breaks"
            cleared_total += int(cleared.sum())
    assert cleared_total > 2_000_000  # the bound was exercised, not vacuous


def test_clear_bound_is_tight_to_the_stated_margin():
    """Just past the bound (shortest bond, displacement along it) the reference stretch reaches s_c (1 - 1e-6)
    within rounding: the bound gives away no more than its stated margin."""
    h = 1.0e-3
    xi = np.array([[h, 0.0, 0.0]])
    for sc in (1.0e-4, 4.0e-3, 0.5):
        lim = np.sqrt(_clear_bound(sc, h * h))
        s = _ref_stretch(xi, np.array([[lim, 0.0, 0.0]]))[0]
        assert abs(s - (sc * (1.0 - 1.0e-6) - 1.0e-12)) <= 1e-12 * max(1.0, sc)
        assert s < sc
