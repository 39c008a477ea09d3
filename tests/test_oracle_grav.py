"""The oracle's gravity (P2) against the reference's known answers and analytic oracles
(crates/sr-physics/src/reference/grav.rs, crates/sr-engine/tests/gpu/grav.rs:22-215, 318-440)."""
import math

import numpy as np

import oracle as O
from sandbox_reactions_b200.abi import Config

SELF_CELL = 3.525494348078172


def square_potential_by_quadrature():
    """∫∫ over [-½, ½]² of dA / r by Simpson on the polar form (tests/gpu/grav.rs:22-38)."""
    n = 4096
    a, b = 0.0, math.pi / 4
    hh = (b - a) / n
    s = 0.5 / math.cos(a) + 0.5 / math.cos(b)
    for k in range(1, n):
        s += (0.5 / math.cos(a + k * hh)) * (4.0 if k % 2 else 2.0)
    return 8.0 * s * hh / 3.0


def test_self_cell_is_the_closed_form_and_the_quadrature():
    assert abs(SELF_CELL - 4.0 * math.log(1.0 + math.sqrt(2.0))) < 1e-15
    assert abs(SELF_CELL - square_potential_by_quadrature()) < 1e-12
    cfg = Config()
    t = O.kernel_table(cfg, 32, 32)
    assert t[0, 0] == -SELF_CELL
    for i, j, r in ((1, 0, 1.0), (0, 1, 1.0), (3, 4, 5.0), (-5, 12, 13.0), (8, -15, 17.0)):
        assert abs(t[j % 32, i % 32] + 1.0 / r) < 1e-15
    soft = O.kernel_table(cfg.replace(kernel="softened", softening=1.0), 32, 32)
    assert abs(soft[0, 0] + 1.0) < 1e-15 and abs(soft[4, 3] + 1.0 / math.sqrt(26.0)) < 1e-15


def test_a_unit_source_makes_the_kernel_through_the_convolution():
    w = h = 33
    sigma = np.zeros((h, w))
    sigma[16, 16] = 1.0
    phi, _, _ = O.grav_field(Config(), sigma)
    assert abs(phi[16, 16] + SELF_CELL) < 1e-12
    assert abs(phi[16, 19] + 1.0 / 3.0) < 1e-12 and abs(phi[20, 19] + 1.0 / 5.0) < 1e-12


def test_vacuum_is_no_source():
    sigma = np.zeros((32, 32))
    sigma[5, 5] = 9e-7
    phi, gx, gy = O.grav_field(Config(), sigma)
    assert np.all(phi == 0.0)
    sigma[5, 5] = 1e-6
    phi, _, _ = O.grav_field(Config(), sigma)
    assert phi[5, 5] < 0.0


def disk(a, sc, cx, cy, w, h):
    j, i = np.mgrid[0:h, 0:w]
    r2 = ((i - cx) ** 2 + (j - cy) ** 2) / (a * a)
    return np.where(r2 < 1.0, sc * np.sqrt(np.clip(1.0 - r2, 0.0, None)), 0.0)


def worst_error(a, centre=(0.0, 0.0)):
    """Largest |Δg|/|g| for 0 < r ≤ 0.75a against the Maclaurin disk's g = -(π²GΣc/2a) r (tests/gpu/grav.rs:60-97)."""
    side = int(math.ceil(2 * a)) + 17
    o = (side - 1) / 2.0
    ox, oy = o + centre[0], o + centre[1]
    sigma = disk(a, 1.0, ox, oy, side, side)
    cfg = Config(sigma_vac=0.0)
    _, gx, gy = O.grav_field(cfg, sigma)
    k = math.pi ** 2 / (2.0 * a)
    j, i = np.mgrid[0:side, 0:side]
    dx, dy = i - ox, j - oy
    r = np.hypot(dx, dy)
    m = (r > 0) & (r <= 0.75 * a)
    err = np.sqrt((gx + k * dx) ** 2 + (gy + k * dy) ** 2)[m] / (k * r[m])
    return err.max(), int(m.sum())


def test_maclaurin_disk_a40_force_is_within_2_percent():
    worst, count = worst_error(40.0)
    assert count > 2700
    assert worst <= 0.02


def test_force_error_halves_when_the_disk_doubles():
    e40, _ = worst_error(40.0)
    e20, _ = worst_error(20.0)
    assert 1.6 <= e20 / e40 <= 2.4


def test_maclaurin_disk_centred_on_a_cell_corner_holds_too():
    worst, _ = worst_error(40.0, (0.5, 0.5))
    assert worst <= 0.02


def test_random_asymmetric_masses_have_no_net_self_force():
    """Σ m·g cancels by the kernel's symmetry (tests/gpu/grav.rs:339-372), also with matter on the outer ring."""
    rng = np.random.default_rng(7)
    for rim in (3, 0):
        w, h = 50, 37
        sigma = np.zeros((h, w))
        inner = rng.random((h - 2 * rim, w - 2 * rim)) < 0.4
        sigma[rim:h - rim, rim:w - rim] = np.where(inner, 0.01 + 2.0 * rng.random(inner.shape) ** 2, 0.0)
        _, gx, gy = O.grav_field(Config(), sigma)
        net = np.array([(sigma * gx).sum(), (sigma * gy).sum()])
        scale = (sigma * np.hypot(gx, gy)).sum()
        assert np.hypot(*net) / scale < 1e-12


def test_potential_matches_the_direct_sum_for_both_kernels():
    rng = np.random.default_rng(3)
    sigma = np.where(rng.random((40, 48)) < 0.5, rng.random((40, 48)), 0.0)
    ty, tx = np.mgrid[0:40:3, 0:48:5]
    for cfg in (Config(), Config(kernel="softened", softening=1.0)):
        phi, _, _ = O.grav_field(cfg, sigma)
        d = O.direct_potential(cfg, sigma, tx.ravel(), ty.ravel())
        assert np.abs(phi[ty.ravel(), tx.ravel()] - d).max() / np.abs(d).max() < 1e-10
