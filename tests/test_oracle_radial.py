"""The oracle's radial (QDHT) restatement: transform checks and the reference's own
radial pin, bulk consistency (test/test_coordinate_systems.jl:60-81: at a uniform
profile dF/drho at the first grid point equals mu_res to 1e-5)."""
import numpy as np
import pytest

import _systems as S
from oracle import functional as fn
from oracle import pcsaft_bulk as pb
from oracle import radial as rd


@pytest.mark.parametrize("n", [1, 2])
def test_qdht_convolution_of_gaussians_is_exact(n):
    """A Gaussian convolved with a Gaussian kernel (multiplier exp(-k^2 s2^2 / 2)) in D = n + 1
    dimensions is the Gaussian of variance s1^2 + s2^2 scaled by (s1^2/(s1^2+s2^2))^(D/2)."""
    Q = rd.QDHT(n, 2.0, 151)
    s1, s2 = 0.2, 0.15
    f = np.exp(-Q.r ** 2 / (2 * s1 ** 2))
    g = Q.conv_matrix(np.exp(-Q.k ** 2 * s2 ** 2 / 2)) @ f
    D = n + 1
    ref = (s1 ** 2 / (s1 ** 2 + s2 ** 2)) ** (D / 2) * np.exp(-Q.r ** 2 / (2 * (s1 ** 2 + s2 ** 2)))
    assert np.max(np.abs(g - ref)) < 1e-13


def test_qdht_spherical_grid_is_the_sine_grid():
    """Order 1/2: zeros j_m = m pi, so r_m = m R / (N + 1) and T is the orthogonal DST-I."""
    Q = rd.QDHT(2, 3.0, 50)
    np.testing.assert_allclose(Q.r, 3.0 * np.arange(1, 51) / 51, rtol=1e-15)
    np.testing.assert_allclose(Q.T @ Q.T, np.eye(50), atol=1e-13)


@pytest.mark.parametrize("coord,ub_L,N", [("sphr", 10.0, 151), ("cyl", 20.0, 101)])
def test_bulk_consistency_radial(coord, ub_L, N):
    """The reference's configuration: PC-SAFT methane, 150 K, 10 MPa liquid."""
    _, om = S.models(["methane"])
    T, p = 150.0, 1e7
    rb = pb.density(om, p, T, [1.0])
    L = om.length_scale()
    so = rd.RadialDFTSystem(om, rd.RadialStructure((p, T), [rb], ub_L * L, N, coord))
    d = so.dFdrho(so.initialize_profiles())
    mu = pb.mu_res(om, [rb], T)[0]
    assert abs(d[0, 0] - mu) < 1e-5


def test_product_radial_grid_matches_oracle():
    import cdft_b200 as cd
    L = 3.7039e-10
    for coord, make in [("sphr", cd.Uniform1DSphr), ("cyl", cd.Uniform1DCyl)]:
        st = make((1e7, 150.0), [3e4], [0.0, 10 * L], 101)
        ost = rd.RadialStructure((1e7, 150.0), [3e4], 10 * L, 101, coord)
        np.testing.assert_allclose(st.coords(0), ost.coords(0), rtol=1e-14)
        ang = 4 * np.pi if coord == "sphr" else 2 * np.pi
        np.testing.assert_allclose(st.weights, ang * ost.qdht.w, rtol=1e-13)


@pytest.mark.parametrize("coord", ["sphr", "cyl"])
@pytest.mark.parametrize("lb_L", [0.0, 2.0])
def test_radial_steele_wall(coord, lb_L):
    """steele.jl:111-143 on a radial grid: lb = 0 a pore wall at ub, lb > 0 a solid core
    of radius lb; the package's V_ext against the oracle's, the clamp of the wall distance
    at 0.5 sigma, and a finite potential everywhere."""
    import cdft_b200 as cd
    pm, om = S.models(["methane"])
    T, p = 150.0, 1e7
    rb = pb.density(om, p, T, [1.0])
    L = om.length_scale()
    lb, ub, N = lb_L * L, 10 * L, 151
    make = cd.Uniform1DSphr if coord == "sphr" else cd.Uniform1DCyl
    st = make((p, T), [rb], [lb, ub], N)
    r = st.coords(0)
    V = cd.Steele(["graphite"]).potential_radial(pm, r, T, *st.bounds[0])
    so = rd.RadialDFTSystem(om, rd.RadialStructure((p, T), [rb], ub, N, coord, lb=lb),
                            walls=[fn.SteeleWall.graphite()])
    np.testing.assert_allclose(V, so.vext, rtol=1e-12)
    assert np.all(np.isfinite(V))
    zw = (r - lb) if lb > 0 else (ub - r)
    clamped = zw <= 0.5 * om.sigma[0]
    assert clamped.any() and (~clamped).any()
    assert np.ptp(V[0, clamped]) == 0.0          # one value over the clamped points
    far = np.argmax(zw)                           # the point farthest from the wall
    assert abs(V[0, far]) < abs(V[0, clamped][0])


@pytest.mark.parametrize("coord", ["sphr", "cyl"])
@pytest.mark.parametrize("lb_L", [0.0, 2.0])
def test_radial_steele_equals_planar_wall_at_wall_distance(coord, lb_L):
    """Independent of both restatements: on a radial grid the Steele potential is the
    planar single-wall 10-4-3 value (steele.jl:49-81, graphite: sigma_s 3.40 A, eps_s 28 K,
    rho_s 0.114 A^-3, Delta 3.35 A; Lorentz-Berthelot fluid-solid pair) evaluated at the
    wall distance r - lb (solid core, lb > 0) or ub - r (pore, lb = 0), with the distance
    clamped below at half the smallest fluid sigma (steele.jl:125-126)."""
    import cdft_b200 as cd
    pm, om = S.models(["methane"])
    T, p = 150.0, 1e7
    rb = pb.density(om, p, T, [1.0])
    L = om.length_scale()
    lb, ub, N = lb_L * L, 10 * L, 151
    make = cd.Uniform1DSphr if coord == "sphr" else cd.Uniform1DCyl
    st = make((p, T), [rb], [lb, ub], N)
    r = st.coords(0)
    V = cd.Steele(["graphite"]).potential_radial(pm, r, T, *st.bounds[0])

    sig_s, eps_s, rho_s, delta = 3.40e-10, 28.0, 0.114e30, 3.35e-10
    sig_f, eps_f = 3.7039e-10, 150.03
    s, e = 0.5 * (sig_s + sig_f), np.sqrt(eps_s * eps_f)

    def planar(z):
        return (2 * np.pi * rho_s * e * delta * s * s
                * (0.4 * (s / z) ** 10 - (s / z) ** 4 - s ** 4 / (3 * delta * (z + 0.61 * delta) ** 3)) / T)

    zw = (r - lb) if lb > 0 else (ub - r)
    zc = np.maximum(zw, 0.5 * sig_f)
    np.testing.assert_allclose(V[0], planar(zc), rtol=1e-12)
    clamped = zw <= 0.5 * sig_f
    assert clamped.any()
    np.testing.assert_allclose(V[0, clamped], planar(0.5 * sig_f), rtol=1e-12)


@pytest.mark.parametrize("width", [0.0, 3.2e-9])
def test_steele_parameter_derivative_matches_central_differences(width):
    """Steele.potential_dtheta (the wall's dependence on the fluid's sigma_i and eps_i,
    steele.jl:36-41,49-81) against central differences of the potential."""
    import cdft_b200 as cd
    pm, _ = S.models(["methane"])
    z = np.linspace(2e-10, 3e-9, 50)
    wall = cd.Steele(["graphite"], width)
    d = wall.potential_dtheta(pm, z, 150.0)
    th = pm.theta()
    for t in range(3):
        h = 1e-6 * abs(th[t])
        e = np.where(np.arange(3) == t, h, 0.0)
        fd = (wall.potential(pm.with_theta(th + e), z, 150.0) - wall.potential(pm.with_theta(th - e), z, 150.0)) / (2 * h)
        assert np.max(np.abs(fd - d[t])) <= 1e-8 * max(np.max(np.abs(fd)), 1e-300) + (0.0 if t < 2 else 0.0)
