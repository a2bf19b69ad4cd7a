"""Exact zeros and non-finite values on the device path.

- Phi and dPhi/dn at vanishing weighted densities: the dispersion composition
  mbar = sum r_i m_i / sum r_i, the chain log(y lambda / rho) and the association
  xi = 1 - |nv2|^2 / n2^2 are 0/0 there.  In
  FP32 the FFT noise inside hard solutes rounds to exactly 0.0 at some grid points,
  so these points occur in ordinary runs; the functional is finite and zero there.
- A non-finite evaluation: the Euler-Lagrange clamp keeps a NaN (Julia's clamp,
  converge.jl:150) and aasol stops with errcode -2 instead of running on a profile
  that a clamped NaN moved.  A mixed-precision run whose FP32 phase stops that way
  is converged again in FP64 from its initial profile."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["methane", "water_octane"])
def test_phi_pointwise_at_zero_densities(case):
    import cdft_b200 as cd
    sp, so = S.methane_wall(N=64) if case == "methane" else S.water_octane_lle(N=64)
    nc, NF = sp.nc, so.NF
    n = np.zeros((nc, NF, 4))
    # point 0: all zero; point 1: only the dispersion density left; point 2: rho > 0
    # with lambda = 0; point 3: a dilute isotropic state (vector field 0) next to the zeros
    n[:, NF - 1, 1] = 1e-3
    n[:, 0, 2] = 1e-3
    n[:, :, 3] = 1e-3
    n[:, 3, 3] = 0.0
    f, g = cd.phi_pointwise(sp, n)
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(g))
    assert f[0] == 0.0


class _NaNField:
    """An external field with one non-finite value (at the middle grid point)."""

    def potential(self, model, z, T):
        V = np.zeros((len(model), z.size))
        V[0, z.size // 2] = np.nan
        return V


@pytest.mark.parametrize("engine", ["grid", "persistent"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_evaluation_is_divergence(engine, precision):
    import cdft_b200 as cd
    from oracle import pcsaft_bulk as pb
    pm, om = S.models(["methane"])
    rb = pb.density(om, 1e7, 150.0, [1.0])
    s = om.sigma[0]
    st = cd.Uniform1DCart((1e7, 150.0), [rb], (0.5 * s, 4.5 * s), 101)
    sp = cd.DFTSystem(pm, st, [cd.Steele(["graphite"], 0.0), _NaNField()], cd.DFTOptions(precision))
    rho = cd.initialize_profiles(sp)
    rho[~np.isfinite(rho)] = rb
    r0 = rho.copy()
    res = cd.converge(sp, rho, beta=0.1, tol=1e-10, anderson_m=5, maxit=100, engine=engine)
    assert res.idid == 0 and res.errcode == -2
    # one evaluation per phase: FP64 stops at once; mixed on the grid engine stops its FP32
    # phase and its FP64 restart from the initial profile at once (on the persistent engine a
    # 1D mixed plan converges in FP64 directly)
    two_phase = precision == "mixed" and engine == "grid"
    assert res.evaluations == (2 if two_phase else 1)
    assert not np.isfinite(res.resnorm)
    np.testing.assert_allclose(rho, r0, rtol=1e-14)
    sp.close()
