"""Batched bulk densities on the device (cdft_bulk_density) against the host bulk
PC-SAFT (cdft_b200.thermo, itself pinned to the oracle's bulk equations): the stable
root of every isotherm state point, liquid and vapour roots of n-octane and water
(2B association), and a water + n-octane liquid.  Roots to 1e-12 relative."""
import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def test_isotherm_stable_densities():
    import bench
    import cdft_b200 as cd
    model = cd.PCSAFT(["methane"], **bench.METHANE)
    ps = np.array([p for _, p, _ in bench.isotherm_specs()])
    got = cd.bulk_density(model, ps, bench.T_ISO, [1.0])
    want = np.array([model.stable_density(p, bench.T_ISO, [1.0]) for p in ps])
    np.testing.assert_allclose(got, want, rtol=1e-12)


@pytest.mark.parametrize("names,T,x", [(["octane"], 298.15, [1.0]), (["water"], 298.15, [1.0]),
                                       (["water", "octane"], 298.15, [0.3, 0.7])])
def test_liquid_and_vapour_roots(names, T, x):
    import cdft_b200 as cd
    pm, _ = S.models(names)
    ps = np.logspace(2, 6, 9)
    for phase in ("liquid", "vapour", "stable"):
        try:
            want = np.array([pm.molar_density(p, T, x, phase) if phase != "stable" else pm.stable_density(p, T, x)
                             for p in ps])
        except ValueError:
            continue
        got = cd.bulk_density(pm, ps, T, x, phase)
        np.testing.assert_allclose(got, want, rtol=1e-12, err_msg=phase)


def test_cross_association_is_refused():
    import cdft_b200 as cd
    from cdft_b200._lib import CDFTError
    pm, _ = S.models(["water", "ethanol"])
    with pytest.raises(CDFTError):
        cd.bulk_density(pm, [1e5], 298.15, [0.5, 0.5], "liquid")
