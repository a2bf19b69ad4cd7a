"""The reference-structured FP64 comparison path of bench.py (C2C FFT pair per
convolution, autograd dPhi/dn, aasol with a host-side small solve), run with torch on
the CPU against the oracle at 16^3: one fixed-point map and a whole converge."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "cdft.jl_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def _oracle_system(N=16):
    from golden import make_fixtures as mf
    from oracle import functional as fn, pcsaft_bulk as pb
    om = mf.oracle_model(["argon"])
    s = om.sigma[0]
    box = 16.0 * s
    rb = 0.021e30 / pb.N_A
    centres = mf.solute_centres(27, 1.5 * s, box, 2 * box / 128, seed=0)   # the 128^3 box's solutes
    V = mf.solute_vext(N, box, centres, 1.5 * s)
    return fn.DFTSystem(om, fn.Structure((1e5, 100.0), [rb], [(0.0, box)] * 3, (N, N, N)), vext=V)


def _params(so):
    st = so.structure
    return dict(N=st.ngrid[0], box=st.bounds[0][1] - st.bounds[0][0], L=so.L, d=float(so.hsd_red[0]),
                m=float(so.m[0]), s=float(so.sigma_red[0, 0]), eps=float(so.eps_ij[0, 0]), T=st.T,
                vext=np.ascontiguousarray(so.vext[0]), cprd=float(so.chem_pot_res_dens[0]))


def test_plain_fixed_point_map_equals_oracle():
    import torch
    import bench
    so = _oracle_system()
    gfix = bench.plain3d_functional(_params(so), "cpu")
    rng = np.random.default_rng(3)
    rho = so.initialize_profiles() * (1 + 0.05 * rng.standard_normal(so.structure.grid_shape))
    with np.errstate(all="ignore"):
        want = so.get_new_profile(rho)[0]
    got = gfix(torch.from_numpy(np.log(rho[0]))).numpy()
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10)


def test_plain_converge_equals_oracle():
    import torch
    import bench
    so = _oracle_system()
    gfix = bench.plain3d_functional(_params(so), "cpu")
    rho0 = so.initialize_profiles()
    kw = dict(beta=0.1, tol=1e-10, anderson_m=10, maxit=300)
    with np.errstate(all="ignore"):
        want, out = so.converge(rho0, **kw)
    x, evals, ok = bench.plain_aasol(gfix, torch.from_numpy(np.log(rho0[0])), m=10, beta=0.1, tol=1e-10,
                                     maxit=300)
    assert out.errcode == 0 and ok
    assert abs(evals - len(out.history)) <= 2
    np.testing.assert_allclose(np.exp(x.numpy()), want[0], rtol=1e-8)


@pytest.mark.gpu
def test_plain_gpu_path_converges_to_ours():
    import bench
    r = bench.plain_fp64_gpu_3d(32)
    assert r["converged"]
    assert r["omega_ex_rel_diff_vs_ours"] < 1e-8 and r["rho_max_rel_diff_vs_ours"] < 1e-7
